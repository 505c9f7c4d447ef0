// UPPAAL query formulas (the <queries> of the reference's model files) ->
// the simulation query.  The reference ignores these formulas and takes the
// query from its command line (main.cu:39-110); this reader accepts the SMC
// subset its models use:
//   Pr[<=T](<> Process.location)           location reachability (a template
//                                            name, or a process instantiated
//                                            as "name = Template(...)")
//   Pr[<=T](<> var OP k)   OP in >= > <= <  variable reachability (max or min)
//   Pr[<=T; N](...)                          the same with a run count
//   E[<=T; N](max: var), E[<=T; N](min: var) expected extreme value
// Variables are named as declared: globals by name, template locals as
// "Template.name".  Everything else (A[], E<>, -->, simulate, sum(...),
// parameterised templates) is rejected with a message.
#include "front.h"

#include <cctype>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>

namespace csmc {

namespace {

[[noreturn]] void bad(const std::string &f, const std::string &why) {
    throw std::runtime_error("query \"" + f + "\": " + why);
}

std::string strip(const std::string &s) {
    std::string o;
    for (char c : s)
        if (c != ' ' && c != '\t' && c != '\n' && c != '\r') o += c;
    return o;
}

double number(const std::string &f, const std::string &s) {
    size_t used = 0;
    double v = 0;
    try {
        v = std::stod(s, &used);
    } catch (const std::exception &) {
        bad(f, "'" + s + "' is not a number");
    }
    if (used != s.size()) bad(f, "'" + s + "' is not a number");
    return v;
}

// A number the query can use: finite (stod also reads "nan" and "inf").
double finite_number(const std::string &f, const std::string &s, const char *what) {
    const double v = number(f, s);
    if (!std::isfinite(v)) bad(f, std::string(what) + " must be a finite number, not '" + s + "'");
    return v;
}

int var_id(const Network &net, const std::string &f, const std::string &name) {
    for (size_t i = 0; i < net.var_names.size(); ++i)
        if (net.var_names[i] == name) return static_cast<int>(i);
    bad(f, "no variable named '" + name + "' (locals are written Template.name)");
}

// Template of a process name: the template itself, or the template of an
// instantiation "name = Template(...)" in the <system> block.
std::string template_of(const Network &net, const std::string &name) {
    for (const auto &kv : net.template_names)
        if (strip(kv.second) == name) return name;
    const std::string sys = strip(net.system_text);
    const std::string pat = name + "=";
    for (size_t p = sys.find(pat); p != std::string::npos; p = sys.find(pat, p + 1)) {
        if (p > 0 && (std::isalnum(static_cast<unsigned char>(sys[p - 1])) || sys[p - 1] == '_')) continue;
        const size_t open = sys.find('(', p + pat.size());
        if (open == std::string::npos) break;
        return sys.substr(p + pat.size(), open - p - pat.size());
    }
    return name;
}

bool is_location(const Network &net, const std::string &tpl, const std::string &loc) {
    int sys = -1;
    for (const auto &kv : net.template_names)
        if (strip(kv.second) == tpl) sys = kv.first;
    if (sys < 0) return false;
    for (const Node &n : net.nodes) {
        if (n.system != sys) continue;
        auto it = net.node_names.find(n.id);
        if (it != net.node_names.end() && strip(it->second) == loc) return true;
    }
    return false;
}

}  // namespace

QueryText parse_formula(const Network &net, const std::string &formula) {
    const std::string f = strip(formula);
    QueryText q;
    auto close = [&](size_t open) {
        int depth = 0;
        for (size_t i = open; i < f.size(); ++i) {
            if (f[i] == '(') ++depth;
            if (f[i] == ')' && --depth == 0) return i;
        }
        bad(formula, "unbalanced parentheses");
    };
    const bool pr = f.rfind("Pr[", 0) == 0, ex = f.rfind("E[", 0) == 0;
    if (!pr && !ex) bad(formula, "only Pr[<=T](<> ...) and E[<=T;N](max|min: var) are supported");
    const size_t lb = f.find('['), rb = f.find(']');
    if (rb == std::string::npos || f.compare(lb + 1, 2, "<=") != 0) bad(formula, "expected a time bound [<=T]");
    std::string bound = f.substr(lb + 3, rb - lb - 3);
    const size_t semi = bound.find(';');
    if (semi != std::string::npos) {
        const double n = finite_number(formula, bound.substr(semi + 1), "the run count");
        if (!(n >= 1) || n != std::floor(n)) bad(formula, "the run count must be a positive integer");
        if (n > 9007199254740992.0) bad(formula, "the run count must be at most 2^53");
        q.sims = static_cast<uint64_t>(n);
        bound = bound.substr(0, semi);
    }
    q.horizon = finite_number(formula, bound, "the time bound");
    if (q.horizon < 0) bad(formula, "the time bound must not be negative");
    if (rb + 1 >= f.size() || f[rb + 1] != '(') bad(formula, "expected '(' after the bound");
    const size_t end = close(rb + 1);
    if (end != f.size() - 1) bad(formula, "unexpected text after the formula");
    std::string body = f.substr(rb + 2, end - rb - 2);
    if (ex) {
        if (q.sims == 0) bad(formula, "E[...] needs a run count: E[<=T; N](max: var)");
        const size_t colon = body.find(':');
        if (colon == std::string::npos) bad(formula, "expected max: or min:");
        const std::string agg = body.substr(0, colon);
        if (agg != "max" && agg != "min") bad(formula, "expected max: or min:");
        q.kind = 1;
        q.is_max = agg == "max";
        q.is_estimate = 1;
        q.var_id = var_id(net, formula, body.substr(colon + 1));
        q.threshold = 0;
        return q;
    }
    if (body.rfind("<>", 0) != 0) bad(formula, "only eventually-formulas Pr[...](<> ...) are supported");
    body = body.substr(2);
    if (body.find("sum(") != std::string::npos || body.find("forall") != std::string::npos)
        bad(formula, "quantified formulas are not supported");
    static const char *ops[] = {">=", "<=", ">", "<"};
    for (const char *op : ops) {
        const size_t p = body.find(op);
        if (p == std::string::npos) continue;
        const std::string lhs = body.substr(0, p), rhs = body.substr(p + std::string(op).size());
        const double k = finite_number(formula, rhs, "the threshold");
        q.kind = 1;
        q.is_estimate = 0;
        q.var_id = var_id(net, formula, lhs);
        const std::string o = op;
        const double inf = std::numeric_limits<double>::infinity();
        if (o == ">=") { q.is_max = 1; q.threshold = std::nextafter(k, -inf); }
        else if (o == ">") { q.is_max = 1; q.threshold = k; }
        else if (o == "<=") { q.is_max = 0; q.threshold = std::nextafter(k, inf); }
        else { q.is_max = 0; q.threshold = k; }
        return q;
    }
    if (body.find("==") != std::string::npos || body.find("!=") != std::string::npos)
        bad(formula, "equality goals are not supported (use >=, >, <=, <)");
    const size_t dot = body.find('.');
    if (dot == std::string::npos) bad(formula, "expected Template.location or a variable comparison");
    const std::string proc = body.substr(0, dot), loc = body.substr(dot + 1);
    if (proc.find('(') != std::string::npos) bad(formula, "parameterised templates are not supported");
    const std::string tpl = template_of(net, proc);
    if (!is_location(net, tpl, loc)) bad(formula, "no location '" + loc + "' in template '" + tpl + "'");
    q.kind = 0;
    q.var_id = -1;
    q.is_max = 1;
    q.is_estimate = 0;
    q.loc_query = tpl + "." + loc;
    return q;
}

}  // namespace csmc
