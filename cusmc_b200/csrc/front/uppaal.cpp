// UPPAAL flat-system reader: declarations, templates, locations, branchpoints
// and transitions, with the reference front end's text conventions.
//
// Reference behaviour followed here (paths relative to the reference repo):
//   declarations            automata_parser/declaration_parser.cpp:9-104
//   constant arithmetic     automata_parser/arithmetic-expression-evaluator.h:18-297
//   variable expressions    automata_parser/variable_expression_evaluator.cpp:17-302
//   string helpers          automata_parser/helper_methods.h:16-103,
//                           automata_parser/string_extractor.cpp:21-84
//   locations/transitions   automata_parser/uppaal_xml_parser.cpp:133-694
#include "front.h"
#include "xml.h"

#include <cctype>
#include <cmath>
#include <cstring>
#include <list>
#include <sstream>
#include <stdexcept>

namespace csmc {

Node *Network::node(int id) {
    for (auto &n : nodes)
        if (n.id == id) return &n;
    return nullptr;
}

namespace {

[[noreturn]] void fail(const std::string &m) { throw std::runtime_error(m); }

// ---- string helpers (helper_methods.h / string_extractor.cpp) -------------

std::string replace_all(std::string s, const std::string &from, const std::string &to) {
    if (from.empty()) return s;
    size_t p = 0;
    while ((p = s.find(from, p)) != std::string::npos) {
        s.replace(p, from.size(), to);
        p += to.size();
    }
    return s;
}

std::string remove_spaces(const std::string &s) { return replace_all(s, " ", ""); }

std::string take_while(const std::string &s, const std::string &w) { return s.substr(0, s.find(w)); }

std::string take_after(const std::string &s, const std::string &w) {
    // find() + length in unsigned arithmetic: a missing one-character
    // separator wraps to position 0, i.e. the whole string (helper_methods.h:34-37)
    const size_t start = s.find(w) + w.size();
    if (start > s.size()) fail("substring start out of range in '" + s + "'");
    return s.substr(start);
}

bool contains(const std::string &s, const std::string &t) { return s.find(t) != std::string::npos; }

// std::getline splitting: no trailing empty segment after a final separator.
std::vector<std::string> getline_split(const std::string &s, char sep) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string seg;
    while (std::getline(ss, seg, sep)) out.push_back(seg);
    return out;
}

// The two regex rewrites of helper::split_expr around parenthesis stripping:
// "random\((.*)\)" -> "random|$1|" and back.  ECMAScript '.' stops at line
// ends, '.*' is greedy, and every non-overlapping match is replaced.
std::string regex_wrap(const std::string &s, const std::string &open, char close, const std::string &rep_open,
                       char rep_close) {
    std::string out;
    size_t pos = 0;
    for (;;) {
        size_t p = s.find(open, pos);
        if (p == std::string::npos) break;
        size_t body = p + open.size();
        size_t line_end = s.find_first_of("\n\r", body);
        if (line_end == std::string::npos) line_end = s.size();
        size_t last = std::string::npos;
        for (size_t i = body; i < line_end; ++i)
            if (s[i] == close) last = i;
        if (last == std::string::npos) {
            out.append(s, pos, p + 1 - pos);
            pos = p + 1;
            continue;
        }
        out.append(s, pos, p - pos);
        out += rep_open;
        out.append(s, body, last - body);
        out.push_back(rep_close);
        pos = last + 1;
    }
    out.append(s, pos, std::string::npos);
    return out;
}

std::vector<std::string> split_guard(const std::string &e) {
    std::vector<std::string> out;
    for (std::string seg : getline_split(e, '&')) {
        seg = replace_all(seg, "&", "");
        seg = regex_wrap(seg, "random(", ')', "random|", '|');
        seg = replace_all(seg, "(", "");
        seg = replace_all(seg, ")", "");
        seg = regex_wrap(seg, "random|", '|', "random(", ')');
        out.push_back(seg);
    }
    return out;
}

std::string constraint_op_text(const std::string &e) {
    if (contains(e, "<=")) return "<=";
    if (contains(e, ">=")) return ">=";
    if (contains(e, "==")) return "==";
    if (contains(e, "!=")) return "!=";
    if (contains(e, "<")) return "<";
    if (contains(e, ">")) return ">";
    fail("Operand in " + e + " not found");
}

COp constraint_op(const std::string &e) {
    const std::string t = constraint_op_text(e);
    if (t == "<=") return COp::Le;
    if (t == ">=") return COp::Ge;
    if (t == "==") return COp::Eq;
    if (t == "!=") return COp::Ne;
    if (t == "<") return COp::Lt;
    return COp::Gt;
}

Op expr_cmp_op(const std::string &e) {  // uppaal_xml_parser.cpp:55-85
    const std::string t = constraint_op_text(e);
    if (t == "<=") return Op::Le;
    if (t == ">=") return Op::Ge;
    if (t == "==") return Op::Eq;
    if (t == "!=") return Op::Ne;
    if (t == "<") return Op::Lt;
    return Op::Gt;
}

std::string float_text(float f) {  // std::to_string(float): "%f" of the promoted value
    char b[512];
    std::snprintf(b, sizeof b, "%f", static_cast<double>(f));
    return b;
}

// ---- constant evaluator used for declaration initialisers -----------------
// Double arithmetic, one-letter-variable legacy slots, degree trigonometry;
// the result is narrowed to float (arithmetic-expression-evaluator.h:292-297).
class ConstEval {
  public:
    ConstEval(const std::unordered_map<std::string, double> *local,
              const std::unordered_map<std::string, double> *global)
        : local_(local), global_(global) {}

    float eval(const std::string &text) {
        buf_ = text;
        p_ = 0;
        double result = 0.0;
        get_token();
        if (tok_.empty()) return 0.0f;
        exp1(result);
        return static_cast<float>(result);
    }

  private:
    enum { DELIM = 1, VARIABLE, NUMBER, FUNCTION };
    const std::unordered_map<std::string, double> *local_, *global_;
    std::string buf_, tok_;
    size_t p_ = 0;
    int type_ = 0;

    static bool stop(char c) { return c == 0 || std::strchr(" +-/*%^=()\t\r", c) != nullptr; }

    char at(size_t i) const { return i < buf_.size() ? buf_[i] : '\0'; }

    void get_token() {
        type_ = 0;
        tok_.clear();
        if (!at(p_)) return;
        while (std::isspace(static_cast<unsigned char>(at(p_)))) ++p_;
        char c = at(p_);
        if (c && std::strchr("+-*/%^=()", c)) {
            type_ = DELIM;
            tok_.push_back(c);
            ++p_;
        } else if (std::isalpha(static_cast<unsigned char>(c))) {
            while (!stop(at(p_))) tok_.push_back(buf_[p_++]);
            while (std::isspace(static_cast<unsigned char>(at(p_)))) ++p_;
            type_ = at(p_) == '(' ? FUNCTION : VARIABLE;
        } else if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
            while (!stop(at(p_))) tok_.push_back(buf_[p_++]);
            type_ = NUMBER;
        }
    }

    void exp1(double &r) {
        if (type_ == VARIABLE) {
            size_t save = p_;
            std::string t = tok_;
            get_token();
            if (tok_ != "=") {
                p_ = save;
                tok_ = t;
                type_ = VARIABLE;
            } else {
                get_token();
                exp2(r);
                return;
            }
        }
        exp2(r);
    }
    void exp2(double &r) {
        exp3(r);
        char op;
        while (!tok_.empty() && ((op = tok_[0]) == '+' || op == '-')) {
            double t = 0;
            get_token();
            exp3(t);
            r = op == '-' ? r - t : r + t;
        }
    }
    void exp3(double &r) {
        exp4(r);
        char op;
        while (!tok_.empty() && ((op = tok_[0]) == '*' || op == '/' || op == '%')) {
            double t = 0;
            get_token();
            exp4(t);
            if (op == '*') r = r * t;
            else if (op == '/') r = r / t;
            else {
                int a = static_cast<int>(r), b = static_cast<int>(t);
                if (b == 0) fail("integer modulo by zero in a declaration");
                r = a % b;
            }
        }
    }
    void exp4(double &r) {
        exp5(r);
        while (tok_ == "^") {
            double t = 0;
            get_token();
            exp5(t);
            r = std::pow(r, t);
        }
    }
    void exp5(double &r) {
        char op = 0;
        if ((type_ == DELIM && tok_ == "+") || tok_ == "-") {
            op = tok_[0];
            get_token();
        }
        exp6(r);
        if (op == '-') r = -r;
    }
    void exp6(double &r) {
        const double kPi = 3.14159265358979323846;
        bool isfunc = type_ == FUNCTION;
        std::string fname;
        if (isfunc) {
            fname = tok_;
            get_token();
        }
        if (tok_ == "(") {
            get_token();
            exp2(r);
            if (isfunc) {
                if (fname == "SIN") r = std::sin(kPi / 180 * r);
                else if (fname == "COS") r = std::cos(kPi / 180 * r);
                else if (fname == "TAN") r = std::tan(kPi / 180 * r);
                else if (fname == "ASIN") r = 180 / kPi * std::asin(r);
                else if (fname == "ACOS") r = 180 / kPi * std::acos(r);
                else if (fname == "ATAN") r = 180 / kPi * std::atan(r);
                else if (fname == "SINH") r = std::sinh(r);
                else if (fname == "COSH") r = std::cosh(r);
                else if (fname == "TANH") r = std::tanh(r);
                else if (fname == "ASINH") r = std::asinh(r);
                else if (fname == "ACOSH") r = std::acosh(r);
                else if (fname == "ATANH") r = std::atanh(r);
                else if (fname == "LN") r = std::log(r);
                else if (fname == "LOG") r = std::log10(r);
                else if (fname == "EXP") r = std::exp(r);
                else if (fname == "SQRT") r = std::sqrt(r);
                else if (fname == "SQR") r = r * r;
                else if (fname == "ROUND") r = std::round(r);
                else if (fname == "INT") r = std::floor(r);
            }
            get_token();
            return;
        }
        if (type_ == VARIABLE) {
            auto it = local_->find(tok_);
            if (it != local_->end()) r = it->second;
            else {
                auto g = global_->find(tok_);
                if (g == global_->end()) fail("VAR NOT DECLARED: " + tok_);
                r = g->second;
            }
            get_token();
            return;
        }
        if (type_ == NUMBER) {
            r = std::atof(tok_.c_str());
            get_token();
            return;
        }
        // syntax error: the reference leaves the result unset; we keep it
    }
};

// ---- declaration parser ----------------------------------------------------
enum DeclType { kClock, kConstBool, kBool, kConstDouble, kConstInt, kChan, kDouble, kInt };

struct Decl {
    DeclType type;
    std::string name;
    double value;
};

class DeclParser {
  public:
    std::vector<Decl> parse(const std::string &decl, const std::unordered_map<std::string, double> *const_global) {
        const_global_ = const_global;
        std::vector<Decl> out;
        for (const std::string &line : getline_split(decl, '\n')) {
            if (line.empty()) continue;
            std::string t = strip_leading(line, ' ');
            t = strip_leading(line, '\t');
            if (t.compare(0, 2, "//") == 0) continue;
            if (starts(t, "clock")) {
                keyword(t, kClock, out);
            } else if (starts(t, "const")) {
                std::string c = strip_leading(t.substr(5), ' ');
                numbers(c, out, true);
            } else if (starts(t, "broadcastchan")) {
                keyword(t, kChan, out);
            }
            numbers(t, out, false);
        }
        return out;
    }

  private:
    std::unordered_map<std::string, double> local_;  // persists across calls, first definition wins
    const std::unordered_map<std::string, double> *const_global_ = nullptr;

    static bool starts(const std::string &s, const std::string &k) { return s.compare(0, k.size(), k) == 0; }

    // helper::remove_while: throws when every character is the one removed
    static std::string strip_leading(const std::string &s, char c) {
        for (size_t i = 0; i < s.size(); ++i)
            if (s[i] != c) return s.substr(i);
        fail("declaration line consists only of '" + std::string(1, c) + "'");
    }

    void numbers(const std::string &s, std::vector<Decl> &out, bool is_const) {
        if (starts(s, "double")) keyword(s, is_const ? kConstDouble : kDouble, out);
        if (starts(s, "bool")) keyword(s, is_const ? kConstBool : kBool, out);
        if (starts(s, "int")) keyword(s, is_const ? kConstInt : kInt, out);
    }

    static const char *kw(DeclType t) {
        switch (t) {
        case kClock: return "clock";
        case kChan: return "broadcastchan";
        case kConstBool: case kBool: return "bool";
        case kConstDouble: case kDouble: return "double";
        default: return "int";
        }
    }

    void keyword(const std::string &lines, DeclType type, std::vector<Decl> &out) {
        const std::string key = kw(type);
        for (const std::string &raw : getline_split(lines, ',')) {
            std::string in = remove_spaces(raw);
            in = replace_all(in, key, "");
            in = replace_all(in, ";", "");
            std::string left = contains(in, ":=") ? take_while(in, ":=") : contains(in, "=") ? take_while(in, "=") : in;
            std::string right = contains(in, "=") ? take_after(in, "=") : "";
            right = replace_all(right, "true", "1");
            right = replace_all(right, "false", "0");
            std::string text;
            if (!right.empty()) {
                ConstEval ev(&local_, const_global_);
                text = float_text(ev.eval(right));
            }
            std::vector<std::string> names;
            {   // helper::split_all on ","
                std::string s = left;
                size_t p;
                while ((p = s.find(',')) != std::string::npos) {
                    names.push_back(s.substr(0, p));
                    s.erase(0, p + 1);
                }
                names.push_back(s);
            }
            for (const std::string &n : names) {
                const std::string v = text.empty() ? "0" : text;
                out.push_back(Decl{type, n, std::stod(v)});
                local_.emplace(n, text.empty() ? 0.0 : static_cast<double>(std::stof(text)));
            }
        }
    }
};

// ---- expression parser producing IR trees -----------------------------------
class ExprParser {
  public:
    ExprParser(Network &net, const std::unordered_map<std::string, int> *local,
               const std::unordered_map<std::string, int> *global,
               const std::unordered_map<std::string, double> *const_local,
               const std::unordered_map<std::string, double> *const_global)
        : net_(net), local_(local), global_(global), clocal_(const_local), cglobal_(const_global) {}

    Expr *parse(const std::string &text) {
        buf_ = text;
        p_ = 0;
        get_token();
        if (tok_.empty()) fail("No Expression Present");
        Expr *e = exp1();
        if (!tok_.empty()) fail("Syntax Error in expression '" + text + "'");
        return e;
    }

  private:
    enum { DELIM = 1, VARIABLE, NUMBER, FUNCTION };
    Network &net_;
    const std::unordered_map<std::string, int> *local_, *global_;
    const std::unordered_map<std::string, double> *clocal_, *cglobal_;
    std::string buf_, tok_;
    size_t p_ = 0;
    int type_ = 0;

    char at(size_t i) const { return i < buf_.size() ? buf_[i] : '\0'; }
    static bool stop(char c) { return c == 0 || std::strchr(" +-/*%^=()!\t\r", c) != nullptr; }

    void get_token() {
        type_ = 0;
        tok_.clear();
        if (!at(p_)) return;
        while (std::isspace(static_cast<unsigned char>(at(p_)))) ++p_;
        char c = at(p_);
        if (c && std::strchr("+-*/%^=()!", c)) {
            type_ = DELIM;
            tok_.push_back(c);
            ++p_;
        } else if (std::isalpha(static_cast<unsigned char>(c))) {
            while (!stop(at(p_))) tok_.push_back(buf_[p_++]);
            while (std::isspace(static_cast<unsigned char>(at(p_)))) ++p_;
            type_ = at(p_) == '(' ? FUNCTION : VARIABLE;
        } else if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
            while (!stop(at(p_))) tok_.push_back(buf_[p_++]);
            type_ = NUMBER;
        }
    }

    Expr *bin(Op op, Expr *l, Expr *r) {
        Expr *e = net_.make(op);
        e->l = l;
        e->r = r;
        return e;
    }

    Expr *exp1() {
        if (type_ == VARIABLE) {
            size_t save = p_;
            std::string t = tok_;
            get_token();
            if (tok_ != "=") {
                p_ = save;
                tok_ = t;
                type_ = VARIABLE;
            } else {
                get_token();
                return exp2();
            }
        }
        return exp2();
    }
    Expr *exp2() {
        Expr *r = exp3();
        while (tok_ == "+" || tok_ == "-") {
            Op op = tok_ == "+" ? Op::Plus : Op::Minus;
            get_token();
            r = bin(op, r, exp3());
        }
        return r;
    }
    Expr *exp3() {
        Expr *r = exp4();
        while (tok_ == "*" || tok_ == "/" || tok_ == "%") {
            Op op = tok_ == "*" ? Op::Mul : tok_ == "/" ? Op::Div : Op::Mod;
            get_token();
            r = bin(op, r, exp4());
        }
        return r;
    }
    Expr *exp4() {
        Expr *r = exp5();
        while (tok_ == "^") {
            get_token();
            r = bin(Op::Pow, r, exp5());
        }
        return r;
    }
    Expr *exp5() {
        char op = 0;
        if ((type_ == DELIM && tok_ == "!") || tok_ == "-") {
            op = tok_[0];
            get_token();
        }
        Expr *r = exp6();
        if (op == '-') return bin(Op::Neg, r, nullptr);
        if (op == '!') return bin(Op::Not, r, nullptr);
        return r;
    }
    Expr *exp6() {
        const bool isfunc = type_ == FUNCTION;
        std::string fname;
        if (isfunc) {
            fname = tok_;
            get_token();
        }
        if (tok_ == "(") {
            get_token();
            Expr *r = exp2();
            if (tok_ != ")") fail("Unbalanced Parentheses");
            if (isfunc) {
                if (fname == "random") r = bin(Op::Random, r, nullptr);
                else if (fname == "sqrt") r = bin(Op::Sqrt, r, nullptr);
                else fail("Unknown Function " + fname);
            }
            get_token();
            return r;
        }
        if (type_ == VARIABLE) {
            Expr *e = net_.make(Op::Lit);
            auto cl = clocal_->find(tok_);
            auto cg = cglobal_->find(tok_);
            auto l = local_->find(tok_);
            auto g = global_->find(tok_);
            if (cl != clocal_->end()) e->value = cl->second;
            else if (cg != cglobal_->end()) e->value = cg->second;
            else if (l != local_->end()) { e->op = Op::Var; e->var = l->second; }
            else if (g != global_->end()) { e->op = Op::Var; e->var = g->second; }
            else fail("VAR NOT DECLARED. VAR:" + tok_ + ":");
            get_token();
            return e;
        }
        if (type_ == NUMBER) {
            Expr *e = net_.make(Op::Lit);
            e->value = std::stod(tok_);
            get_token();
            return e;
        }
        fail("Syntax Error, not known token:" + tok_ + ":");
    }
};

// ---- the model reader --------------------------------------------------------
class UppaalReader {
  public:
    explicit UppaalReader(Network &net) : net_(net) {}

    void read(const XmlNode &doc) {
        const XmlNode *nta = doc.child("nta");
        if (!nta) fail("model has no <nta> element");
        init_globals(*nta);
        net_.system_text = nta->child_text("system");
        int system = 0;
        for (const XmlNode *t : nta->children_named("template")) {
            const std::string init_ref = remove_spaces(t->child(("init")) ? t->child("init")->attr("ref") : "");
            init_node_id_ = node_id(init_ref);
            cur_template_ = t->child_text("name");
            init_locals(*t);
            net_.template_names.emplace(system, t->child_text("name"));
            for (const XmlNode *l : t->children_named("location")) location(*l, system);
            for (const XmlNode *b : t->children_named("branchpoint")) branchpoint(*b, system);
            for (const XmlNode *tr : t->children_named("transition")) transition(*tr);
            vars_.clear();
            timers_.clear();
            ++system;
        }
        net_.n_templates = system;
    }

  private:
    Network &net_;
    DeclParser dp_;
    int vars_id_ = 0, chan_id_ = 1, init_node_id_ = 0;
    std::string cur_template_;
    std::unordered_map<std::string, double> const_local_, const_global_;
    std::unordered_map<std::string, int> timers_, global_timers_, vars_, global_vars_;

    static int node_id(const std::string &ref) {  // "idN" -> N+1
        std::string s = remove_spaces(ref);
        if (s.size() < 2) fail("malformed location reference '" + ref + "'");
        s.replace(0, 2, "");
        size_t used = 0;
        int v = 0;
        try {
            v = std::stoi(s, &used);
        } catch (const std::exception &) {
            fail("malformed location reference '" + ref + "'");
        }
        return v + 1;
    }

    Expr *expr(const std::string &text) {
        ExprParser p(net_, &vars_, &global_vars_, &const_local_, &const_global_);
        return p.parse(text);
    }

    void add_var(const std::string &name, bool clock, double value, bool global) {
        (global ? global_vars_ : vars_)[name] = vars_id_;
        if (clock) (global ? global_timers_ : timers_)[name] = vars_id_;
        net_.vars.push_back(VarDecl{vars_id_, clock ? 1 : 0, value});
        net_.var_names.push_back(global ? name : remove_spaces(cur_template_) + "." + name);
        ++vars_id_;
    }

    void init_globals(const XmlNode &nta) {
        const std::string decl = remove_spaces(nta.child_text("declaration"));
        std::vector<Decl> ds = dp_.parse(decl, &const_global_);
        const_global_["true"] = 1.0;
        const_global_["false"] = 0.0;
        for (const Decl &d : ds) {
            if (d.type == kClock) add_var(d.name, true, d.value, true);
            else if (d.type == kChan) global_vars_[d.name] = chan_id_++;
            else if (d.type == kConstDouble || d.type == kConstInt || d.type == kConstBool) const_global_[d.name] = d.value;
            else add_var(d.name, false, d.value, true);
        }
    }

    void init_locals(const XmlNode &t) {
        const std::string decl = remove_spaces(t.child_text("declaration"));
        for (const Decl &d : dp_.parse(decl, &const_global_)) {
            if (d.type == kClock) add_var(d.name, true, d.value, false);
            else if (d.type == kChan) vars_[d.name] = chan_id_++;
            else if (d.type == kConstDouble || d.type == kConstInt || d.type == kConstBool) const_local_[d.name] = d.value;
            else add_var(d.name, false, d.value, false);
        }
    }

    // uppaal_xml_parser.cpp:133-163: the variable named left of the first
    // comparison character.
    int timer_id(const std::string &e) const {
        const std::string w = replace_all(remove_spaces(e), "\n", "");
        size_t index = 0;
        while (index != e.size()) {
            ++index;
            char c = index < w.size() ? w[index] : '\0';
            if (c == '<' || c == '>' || c == '=' || c == '!') break;
        }
        const std::string sub = w.substr(0, index);
        auto l = vars_.find(sub);
        if (l != vars_.end()) return l->second;
        auto g = global_vars_.find(sub);
        if (g != global_vars_.end()) return g->second;
        fail("unknown variable in '" + e + "'");
    }

    void fill_constraints(const std::vector<std::string> &exprs, std::vector<Constraint> &out) {
        for (const std::string &ex : exprs) {
            if (ex.empty()) continue;
            const std::string in = remove_spaces(ex);
            if (in.empty()) continue;
            const std::string op = constraint_op_text(in);
            const std::string left = take_while(in, op), right = take_after(in, op);
            Constraint c;
            c.op = constraint_op(in);
            if (timers_.count(left) || global_timers_.count(left)) {
                c.uses_variable = true;
                c.var = timer_id(in);
                c.expression = expr(right);
            } else {
                c.uses_variable = false;
                c.value = expr(left);
                c.expression = expr(right);
            }
            out.push_back(c);
        }
    }

    Expr *if_statement(const std::string &input) {  // uppaal_xml_parser.cpp:496-547
        const std::string in = remove_spaces(input);
        const std::string cond = take_while(in, "?");
        const std::string if_true = take_while(take_after(in, "?"), ":");
        const std::string if_false = replace_all(take_after(in, ":"), ";", "");
        std::vector<Expr *> conds;
        for (const std::string &ex : split_guard(cond)) {
            if (ex.empty()) continue;
            const std::string c = remove_spaces(ex);
            if (c.empty()) continue;
            const std::string op = constraint_op_text(c);
            const std::string left = take_while(c, op), right = take_after(c, op);
            Expr *e = net_.make(expr_cmp_op(c));
            if (timers_.count(left) || global_timers_.count(left) || vars_.count(left) || global_vars_.count(left)) {
                Expr *v = net_.make(Op::Var);
                v->var = timer_id(c);
                e->l = v;
            } else {
                e->l = expr(left);
            }
            e->r = expr(right);
            conds.push_back(e);
        }
        if (conds.empty()) fail("empty condition in '" + input + "'");
        if (conds.size() > 2)
            fail("conditional with more than two conjuncts in '" + input +
                 "' (the reference builds a cyclic expression for it)");
        Expr *c = conds[0];
        if (conds.size() == 2) {
            c = net_.make(Op::And);
            c->l = conds[0];
            c->r = conds[1];
        }
        Expr *w = net_.make(Op::Cond);
        w->l = c;
        w->r = expr(if_true);
        w->els = expr(if_false);
        return w;
    }

    std::vector<Update> assignment(const std::string &input) {  // uppaal_xml_parser.cpp:549-583
        std::vector<Update> out;
        for (const std::string &seg : getline_split(input, ',')) {
            const std::string in = remove_spaces(seg);
            if (in.empty()) continue;
            const std::string left = contains(in, ":=") ? take_while(in, ":=") : take_while(in, "=");
            std::string right = take_after(in, "=");
            right = replace_all(right, "true", "1");
            right = replace_all(right, "false", "0");
            Update u;
            u.expr = (contains(right, "?") && contains(right, ":")) ? if_statement(right) : expr(right);
            u.var = timer_id(left);
            out.push_back(u);
        }
        return out;
    }

    int sync(const std::string &input) const {  // uppaal_xml_parser.cpp:585-601
        const std::string in = remove_spaces(input);
        const bool listener = contains(in, "?");
        const std::string key = replace_all(in, listener ? "?" : "!", "");
        auto l = vars_.find(key);
        int ec;
        if (l != vars_.end()) ec = l->second;
        else {
            auto g = global_vars_.find(key);
            if (g == global_vars_.end()) fail(key + " is not a declared channel");
            ec = g->second;
        }
        return listener ? -ec : ec;
    }

    void location(const XmlNode &loc, int system) {  // uppaal_xml_parser.cpp:377-431
        const int id = node_id(loc.attr("id"));
        const std::string name = loc.child_text("name");
        const bool committed = loc.child("committed") != nullptr;
        const bool urgent = loc.child("urgent") != nullptr;
        Expr *rate = net_.make(Op::Lit);
        rate->value = 1.0;
        net_.edges[id] = {};
        bool goal = false;
        if (!name.empty()) {
            goal = name == "Goal";
            if (net_.node_names.emplace(id, name).second) net_.node_name_order.emplace_back(id, name);
        }
        const XmlNode *label = loc.child("label");  // only the first label is read
        const std::string kind = label ? label->attr("kind") : "";
        const std::string text = label ? label->child_value() : "";
        Node n;
        n.id = id;
        n.system = system;
        if (kind == "exponentialrate") {
            const std::string w = remove_spaces(text);
            size_t p = w.find('=');
            rate = expr(p == std::string::npos ? w : w.substr(p + 1));
        }
        if (kind == "invariant") fill_constraints(split_guard(text), n.invariants);
        if (init_node_id_ == id) net_.start_nodes.push_back(id);
        n.type = goal ? kGoal : committed ? kCommitted : urgent ? kUrgent : kLocation;
        n.lambda = rate;
        net_.nodes.push_back(std::move(n));
    }

    void branchpoint(const XmlNode &b, int system) {  // uppaal_xml_parser.cpp:653-671
        const int id = node_id(b.attr("id"));
        net_.edges[id] = {};
        Node n;
        n.id = id;
        n.system = system;
        n.type = kBranch;
        n.lambda = net_.make(Op::Lit);
        n.lambda->value = 1.0;
        net_.nodes.push_back(std::move(n));
    }

    void transition(const XmlNode &t) {  // uppaal_xml_parser.cpp:433-489
        const XmlNode *s = t.child("source"), *d = t.child("target");
        const int src = node_id(s ? s->attr("ref") : "");
        const int dst = node_id(d ? d->attr("ref") : "");
        Edge e;
        for (const XmlNode *label : t.children_named("label")) {
            const std::string kind = label->attr("kind");
            const std::string text = label->child_value();
            if (kind == "guard") fill_constraints(split_guard(text), e.guards);
            else if (kind == "assignment") e.updates = assignment(text);
            else if (kind == "synchronisation") e.channel = sync(text);
            else if (kind == "probability") e.weight = expr(remove_spaces(text));
        }
        if (!e.weight) {
            e.weight = net_.make(Op::Lit);
            e.weight->value = 1.0;
        }
        // a target that is not a known node resolves to the first node read
        e.dest_id = net_.node(dst) ? dst : (net_.nodes.empty() ? dst : net_.nodes.front().id);
        auto it = net_.edges.find(src);
        if (it == net_.edges.end()) fail("transition source id" + std::to_string(src - 1) + " is not a location");
        it->second.push_back(std::move(e));
    }
};

}  // namespace

std::unique_ptr<Network> parse_uppaal_text(const std::string &text) {
    auto doc = xml_parse(text);
    auto net = std::make_unique<Network>();
    UppaalReader r(*net);
    r.read(*doc);
    return net;
}

std::unique_ptr<Network> parse_uppaal_file(const std::string &path) {
    auto doc = xml_parse_file(path);
    auto net = std::make_unique<Network>();
    UppaalReader r(*net);
    r.read(*doc);
    return net;
}

}  // namespace csmc
