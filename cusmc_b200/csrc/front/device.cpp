// Reference passes that shape what the kernel receives, the canonical dump,
// and the packer.
//
//   optimizer visit order, goal marking, constraint-set reduction and
//   top-level constant folding:
//       automata_parser/network/domain_optimization_visitor.cpp:4-107,151-441
//       automata_parser/network/visitor.cpp:109-197
//   PN layout:  automata_parser/network/pn_compile_visitor.cpp:3-68
//   location-query goal by name:  smc.cu:407-436
//   device layout choices:  simulation/state/shared_model_state.cu:164-614
#include "front.h"
#include "../include/csmc_net.h"
#include "../include/csmc_numeric.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <stdexcept>
#include <limits>
#include <unordered_set>

namespace csmc {
namespace {

[[noreturn]] void fail(const std::string &m) { throw std::runtime_error(m); }

constexpr double kEps = 0.00001;  // DBL_EPSILON of include/common_macros.h:72

bool is_leaf(const Expr *e) { return e->op == Op::Lit || e->op == Op::Var; }

// ---- constant evaluation (domain_optimization_visitor.cpp:292-369) -----------
// sub: variables replaced by update expressions (compound constraints).
using Subst = std::function<const Expr *(int)>;

bool is_const(const Expr *e, const Subst &sub) {
    if (e->op == Op::Lit) return true;
    if (e->op == Op::Var) {
        const Expr *s = sub ? sub(e->var) : nullptr;
        return s ? is_const(s, nullptr) : false;
    }
    if (e->op == Op::Random) return false;
    const bool l = e->l ? is_const(e->l, sub) : true;
    const bool r = e->r ? is_const(e->r, sub) : true;
    const bool c = e->op == Op::Cond ? (e->els ? is_const(e->els, sub) : true) : true;
    return c && l && r;
}

double eval_const(const Expr *e, const Subst &sub) {
    auto L = [&] { return eval_const(e->l, sub); };
    auto R = [&] { return eval_const(e->r, sub); };
    switch (e->op) {
    case Op::Lit: return e->value;
    case Op::Var: {
        const Expr *s = sub ? sub(e->var) : nullptr;
        if (!s) fail("variable in constant expression");
        return eval_const(s, nullptr);
    }
    case Op::Plus: return L() + R();
    case Op::Minus: return L() - R();
    case Op::Mul: return L() * R();
    case Op::Div: {
        const double t = R();
        if (t == 0.0) fail("Found division by zero in const expression, while running optimizer.");
        return L() / t;
    }
    case Op::Pow: return std::pow(L(), R());
    case Op::Neg: return -L();
    case Op::Sqrt: return std::sqrt(L());
    case Op::Mod: {
        const int a = static_cast<int>(L()), b = static_cast<int>(R());
        if (b == 0) fail("integer modulo by zero in a constant expression");
        return a % b;
    }
    case Op::And: return std::abs(L()) > kEps && std::abs(R()) > kEps;
    case Op::Or: return std::abs(L()) > kEps || std::abs(R()) > kEps;
    case Op::Le: return L() <= R();
    case Op::Ge: return L() >= R();
    case Op::Lt: return L() < R();
    case Op::Gt: return L() > R();
    case Op::Eq: return std::abs(L() - R()) <= kEps;
    case Op::Ne: return std::abs(L() - R()) > kEps;
    case Op::Not: return std::abs(L()) <= kEps;
    case Op::Cond: return std::abs(L()) > kEps ? R() : eval_const(e->els, sub);
    default: fail("unsupported operator in constant expression");
    }
}

void fold(Expr *e) {  // reduce_expr: whole expression only, in place
    if (!e || e->op == Op::Lit) return;
    if (!is_const(e, nullptr)) return;
    const double v = eval_const(e, nullptr);
    e->value = v;
    e->op = Op::Lit;
    e->l = e->r = e->els = nullptr;
}

// A constraint as the optimizer sees it, possibly with substituted sides.
struct CCon {
    const Constraint *orig = nullptr;  // original guard (nullptr for compound/invariant copies)
    COp op;
    bool uses_variable;
    const Expr *value, *expression;
    Subst sub_value, sub_expr;
};

bool ccon_eval(const CCon &c) {
    const double l = eval_const(c.value, c.sub_value), r = eval_const(c.expression, c.sub_expr);
    switch (c.op) {
    case COp::Le: return l <= r;
    case COp::Lt: return l < r;
    case COp::Ge: return l >= r;
    case COp::Gt: return l > r;
    case COp::Eq: return std::abs(l - r) <= kEps;
    case COp::Ne: return std::abs(l - r) > kEps;
    }
    return false;
}

bool ccon_is_const(const CCon &c) {
    if (c.uses_variable) return false;
    return is_const(c.value, c.sub_value) && is_const(c.expression, c.sub_expr);
}

class Optimizer {
  public:
    Optimizer(Network &net, const std::unordered_set<std::string> &query) : net_(net), query_(query) {
        for (auto &n : net_.nodes) by_id_[n.id] = &n;
        for (const auto &v : net_.vars) var_ids_.insert(v.id);
    }

    void run() {
        for (int sid : net_.start_nodes) visit_node(by_id_.at(sid));
        for (auto &n : net_.nodes)
            if (!visited_nodes_.count(n.id))
                fail("location id" + std::to_string(n.id - 1) +
                     " is not reachable from an initial location (the reference front end cannot upload it)");
    }

  private:
    Network &net_;
    const std::unordered_set<std::string> &query_;
    std::unordered_map<int, Node *> by_id_;
    std::set<int> var_ids_;
    std::set<int> visited_nodes_;
    std::set<const Edge *> visited_edges_;

    void check_clock_refs(const Expr *e) {  // validate_invariants -> expr_contains_clock
        if (!e || e->op == Op::Lit) return;
        if (e->op == Op::Var) {
            if (!var_ids_.count(e->var)) fail("invariant refers to unknown variable id " + std::to_string(e->var));
            return;
        }
        check_clock_refs(e->l);
        check_clock_refs(e->r);
        if (e->op == Op::Cond) check_clock_refs(e->els);
    }

    bool is_goal(const Node &n) const {
        auto nn = net_.node_names.find(n.id);
        if (nn == net_.node_names.end()) return false;
        auto tn = net_.template_names.find(n.system);
        if (tn == net_.template_names.end()) fail("template of location not found");
        return query_.count(tn->second + "." + nn->second) > 0;
    }

    // reduce_constraint_set on a node's invariants (in place)
    void reduce_invariants(Node &n) {
        std::vector<Constraint> kept;
        for (const Constraint &c : n.invariants) {
            CCon cc{&c, c.op, c.uses_variable, c.value, c.expression, nullptr, nullptr};
            if (c.uses_variable || !ccon_is_const(cc)) {
                kept.push_back(c);
                continue;
            }
            if (!ccon_eval(cc)) {  // create_false_constraint_set: "0 < 1"
                Constraint f;
                f.op = COp::Lt;
                f.uses_variable = false;
                f.value = net_.make(Op::Lit);
                f.value->value = 0.0;
                f.expression = net_.make(Op::Lit);
                f.expression->value = 1.0;
                n.invariants.assign(1, f);
                return;
            }
        }
        if (kept.size() < n.invariants.size()) n.invariants = kept;
    }

    void visit_node(Node *n) {
        if (visited_nodes_.count(n->id)) return;
        visited_nodes_.insert(n->id);
        for (const Constraint &c : n->invariants)
            if (c.uses_variable) check_clock_refs(c.expression);
        reduce_invariants(*n);
        if (is_goal(*n)) n->type = kGoal;
        for (Constraint &c : n->invariants) {
            if (!c.uses_variable) fold(c.value);
            fold(c.expression);
        }
        auto &edges = net_.edges[n->id];
        for (Edge &e : edges) visit_edge(e);
        for (Edge &e : edges) visit_node(by_id_.at(e.dest_id));
        fold(n->lambda);
    }

    void visit_edge(Edge &e) {
        if (visited_edges_.count(&e)) return;
        visited_edges_.insert(&e);
        // compound_optimize_constraints: guards + destination invariants
        // rewritten through the updates, as they stand at this point
        std::vector<CCon> list;
        for (const Constraint &g : e.guards)
            list.push_back(CCon{&g, g.op, g.uses_variable, g.value, g.expression, nullptr, nullptr});
        const Node *dest = by_id_.at(e.dest_id);
        const std::vector<Update> *ups = &e.updates;
        Subst sub = [ups](int var) -> const Expr * {
            for (const Update &u : *ups)
                if (u.var == var) return u.expr;
            return nullptr;
        };
        for (const Constraint &inv : dest->invariants) {
            if (!inv.uses_variable) {
                list.push_back(CCon{nullptr, inv.op, false, inv.value, inv.expression, sub, sub});
                continue;
            }
            bool any = false;
            for (const Update &u : e.updates) {
                if (u.var != inv.var) continue;
                list.push_back(CCon{nullptr, inv.op, false, u.expr, inv.expression, nullptr, sub});
                any = true;
            }
            if (!any) list.push_back(CCon{nullptr, inv.op, true, nullptr, inv.expression, nullptr, sub});
        }
        // reduce_constraint_set: the first constant-false entry replaces the
        // whole set (so the original guards are not visited below)
        std::vector<const CCon *> kept;
        bool early_false = false;
        for (const CCon &c : list) {
            if (c.uses_variable || !ccon_is_const(c)) {
                kept.push_back(&c);
                continue;
            }
            if (!ccon_eval(c)) {
                early_false = true;
                break;
            }
        }
        if (!early_false) {
            for (const CCon *c : kept) {
                if (!c->orig) continue;  // compound copies are not uploaded
                Constraint *g = const_cast<Constraint *>(c->orig);
                if (!g->uses_variable) fold(g->value);
                fold(g->expression);
            }
        }
        for (Update &u : e.updates) fold(u.expr);
        fold(e.weight);
    }
};

// ---- PN compilation (pn_compile_visitor.cpp) ---------------------------------
int pn_len(const Expr *e) {
    if (is_leaf(e)) return 1;
    const int l = e->l ? pn_len(e->l) : 0;
    const int r = e->r ? pn_len(e->r) : 0;
    if (e->op == Op::Cond) return l + 1 + pn_len(e->els) + 2 + r;
    return l + r + 1;
}

void pn_emit(const Expr *e, std::vector<Expr> &out) {
    if (!e) return;
    if (e->op == Op::Cond) {
        Expr skip;
        skip.op = Op::PnSkip;
        skip.var = pn_len(e->els) + 2;
        pn_emit(e->l, out);
        out.push_back(skip);
        pn_emit(e->els, out);
        Expr t;
        t.op = Op::Lit;
        t.value = 1.0;
        out.push_back(t);
        skip.var = pn_len(e->r);
        out.push_back(skip);
        pn_emit(e->r, out);
        return;
    }
    pn_emit(e->l, out);
    pn_emit(e->r, out);
    Expr rec = *e;
    rec.l = rec.r = rec.els = nullptr;
    out.push_back(rec);
}

DevExpr dev_pn(const Expr *e) {
    DevExpr d;
    if (!e) fail("missing expression");
    if (e->op == Op::Lit) { d.kind = 0; d.value = e->value; return d; }
    if (e->op == Op::Var) { d.kind = 1; d.var = e->var; return d; }
    d.kind = 2;
    pn_emit(e, d.pn);
    if (static_cast<int>(d.pn.size()) + 1 != pn_len(e) + 1) fail("internal: PN length mismatch");
    return d;
}

DevExpr dev_tree(const Expr *e) {
    DevExpr d;
    if (!e) fail("missing expression");
    if (e->op == Op::Lit) { d.kind = 0; d.value = e->value; return d; }
    if (e->op == Op::Var) { d.kind = 1; d.var = e->var; return d; }
    d.kind = 3;
    d.tree = e;
    return d;
}

DevGuard dev_guard(const Constraint &c, const DevModel &m) {
    DevGuard g;
    g.op = c.op;
    int var = -2;
    if (c.uses_variable) var = c.var;
    else if (c.value && c.value->op == Op::Var) var = c.value->var;
    if (var == -2) return g;  // ignored by the kernel
    g.var_based = true;
    const int nv = static_cast<int>(m.var_kind_clock.size());
    if (var < 0 || var >= nv) {
        g.var = -1;
        g.var_is_clock = false;
    } else {
        g.var = var;
        g.var_is_clock = m.var_kind_clock[var] != 0;
    }
    return g;
}

}  // namespace

DevModel build_device_model(Network &net, const std::string &loc_query, bool loc_mode) {
    std::unordered_set<std::string> query{loc_query};
    Optimizer opt(net, query);
    opt.run();

    std::unordered_map<int, Node *> by_id;
    for (auto &n : net.nodes) by_id[n.id] = &n;

    if (loc_mode) {  // smc.cu:407-436, with the same container operations
        std::string nodename;
        bool dot = false;
        for (char c : loc_query) {
            if (c == '.') { dot = true; continue; }
            if (dot) nodename.push_back(c);
        }
        std::unordered_map<int, std::string> names;
        for (const auto &p : net.node_name_order) names.emplace(p.first, p.second);
        const std::unordered_map<int, std::string> names_copy(names);
        std::unordered_map<std::string, int> by_name;
        for (auto it = names_copy.cbegin(); it != names_copy.cend(); ++it) by_name.insert({it->second, it->first});
        auto t = by_name.find(nodename);
        if (t != by_name.end()) {
            auto nm = by_id.find(t->second);
            if (nm != by_id.end()) nm->second->type = kGoal;
        }
    }

    DevModel m;
    for (const auto &v : net.vars) {
        m.var_kind_clock.push_back(v.rate > 0 ? 1 : 0);
        double iv = v.value;
        int ii;
        if (std::isnan(iv)) ii = 0;
        else if (iv >= 2147483647.0) ii = 2147483647;
        else if (iv <= -2147483648.0) ii = -2147483647 - 1;
        else ii = static_cast<int>(iv);
        m.var_init.push_back(ii);
    }

    int max_comp = -1;
    for (const auto &n : net.nodes) max_comp = std::max(max_comp, n.system);
    m.comps.resize(max_comp + 1);
    for (int c = 0; c <= max_comp; ++c) {
        auto tn = net.template_names.find(c);
        m.comps[c].name = tn == net.template_names.end() ? "" : tn->second;
        m.comps[c].init_id = c < static_cast<int>(net.start_nodes.size()) ? net.start_nodes[c] : -1;
    }
    std::vector<std::vector<int>> ids(max_comp + 1);
    for (const auto &n : net.nodes) ids[n.system].push_back(n.id);
    for (int c = 0; c <= max_comp; ++c) {
        auto &v = ids[c];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        DevComp &dc = m.comps[c];
        for (int id : v) {
            const Node &n = *by_id.at(id);
            DevLoc L;
            L.id = id;
            auto nn = net.node_names.find(id);
            L.named = nn != net.node_names.end();
            if (L.named) L.name = nn->second;
            L.type = n.type;
            L.lambda = dev_pn(n.lambda);
            for (const Constraint &inv : n.invariants) {
                DevGuard g = dev_guard(inv, m);
                if (g.var_based) g.rhs = dev_pn(inv.expression);
                L.invariants.push_back(g);
            }
            for (const Edge &e : net.edges[id]) {
                DevEdge de;
                de.dest_id = e.dest_id;
                de.channel = e.channel;
                de.weight = dev_tree(e.weight);
                for (const Constraint &gc : e.guards) {
                    DevGuard g = dev_guard(gc, m);
                    if (g.var_based) g.rhs = dev_tree(gc.expression);
                    de.guards.push_back(g);
                }
                for (const Update &u : e.updates) de.updates.push_back(DevUpdate{u.var, dev_pn(u.expr)});
                L.edges.push_back(std::move(de));
            }
            dc.locs.push_back(std::move(L));
        }
        for (size_t i = 0; i < dc.locs.size(); ++i) {
            if (dc.locs[i].id == dc.init_id) dc.init_local = static_cast<int>(i);
            for (DevEdge &e : dc.locs[i].edges)
                for (size_t j = 0; j < dc.locs.size(); ++j)
                    if (dc.locs[j].id == e.dest_id) { e.dest_local = static_cast<int>(j); break; }
        }
    }
    return m;
}

// ---- canonical dump ------------------------------------------------------------
namespace {

const char *op_name(Op op) {
    switch (op) {
    case Op::Lit: return "lit";
    case Op::Var: return "var";
    case Op::Random: return "random";
    case Op::Plus: return "+";
    case Op::Minus: return "-";
    case Op::Mul: return "*";
    case Op::Div: return "/";
    case Op::Pow: return "^";
    case Op::Neg: return "neg";
    case Op::Sqrt: return "sqrt";
    case Op::Mod: return "%";
    case Op::And: return "&&";
    case Op::Or: return "||";
    case Op::Le: return "<=";
    case Op::Ge: return ">=";
    case Op::Lt: return "<";
    case Op::Gt: return ">";
    case Op::Eq: return "==";
    case Op::Ne: return "!=";
    case Op::Not: return "!";
    case Op::Cond: return "?:";
    case Op::Compiled: return "compiled";
    case Op::PnCompiled: return "pn";
    case Op::PnSkip: return "skip";
    }
    return "?";
}

std::string num(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

std::string dump_tree(const Expr *e) {
    if (!e) return "-";
    if (e->op == Op::Lit) return "L" + num(e->value);
    if (e->op == Op::Var) return "V" + std::to_string(e->var);
    // the device copy of a tree keeps only left/right (shared_model_state.cu:112-124)
    return std::string("(") + op_name(e->op) + " " + dump_tree(e->l) + " " + dump_tree(e->r) + ")";
}

std::string dump_dev(const DevExpr &d) {
    switch (d.kind) {
    case 0: return "L" + num(d.value);
    case 1: return "V" + std::to_string(d.var);
    case 2: {
        std::string s = "P" + std::to_string(d.pn.size() + 1) + "{";
        for (size_t i = 0; i < d.pn.size(); ++i) {
            const Expr &r = d.pn[i];
            if (i) s += ",";
            if (r.op == Op::Lit) s += "L" + num(r.value);
            else if (r.op == Op::Var) s += "V" + std::to_string(r.var);
            else if (r.op == Op::PnSkip) s += "S" + std::to_string(r.var);
            else s += op_name(r.op);
        }
        return s + "}";
    }
    default: return "T" + dump_tree(d.tree);
    }
}

const char *cop_name(COp op) {
    switch (op) {
    case COp::Le: return "<=";
    case COp::Lt: return "<";
    case COp::Ge: return ">=";
    case COp::Gt: return ">";
    case COp::Eq: return "==";
    case COp::Ne: return "!=";
    }
    return "?";
}

std::string dump_guard(const DevGuard &g) {
    if (!g.var_based) return std::string("ignored ") + cop_name(g.op);
    return std::string(cop_name(g.op)) + " V" + std::to_string(g.var) + " " + (g.var_is_clock ? "CLOCK" : "INT") +
           " " + dump_dev(g.rhs);
}

}  // namespace

std::string quote_dump(const std::string &s) {
    std::string o = "\"";
    for (char c : s) {
        if (c == '\n') o += "\\n";
        else if (c == '\t') o += "\\t";
        else if (c == '\r') o += "\\r";
        else if (c == '"') o += "\\\"";
        else if (c == '\\') o += "\\\\";
        else o += c;
    }
    return o + "\"";
}

std::string dump_device_model(const DevModel &m) {
    std::string o = "csmc-dump 1\n";
    char b[256];
    std::snprintf(b, sizeof b, "vars %zu\n", m.var_kind_clock.size());
    o += b;
    for (size_t i = 0; i < m.var_kind_clock.size(); ++i) {
        std::snprintf(b, sizeof b, "var %zu %s %d\n", i, m.var_kind_clock[i] ? "CLOCK" : "INT", m.var_init[i]);
        o += b;
    }
    std::snprintf(b, sizeof b, "components %zu\n", m.comps.size());
    o += b;
    for (size_t c = 0; c < m.comps.size(); ++c) {
        const DevComp &dc = m.comps[c];
        o += "comp " + std::to_string(c) + " " + quote_dump(dc.name) + " nlocs " + std::to_string(dc.locs.size()) +
             " init " + std::to_string(dc.init_id) + "\n";
        for (const DevLoc &L : dc.locs) {
            o += "loc " + std::to_string(L.id) + " " + quote_dump(L.named ? L.name : "") + " type " +
                 std::to_string(L.type) + " lambda " + dump_dev(L.lambda) + " inv " +
                 std::to_string(L.invariants.size()) + " edges " + std::to_string(L.edges.size()) + "\n";
            for (const DevGuard &g : L.invariants) o += "  inv " + dump_guard(g) + "\n";
            for (const DevEdge &e : L.edges) {
                o += "  edge dst " + std::to_string(e.dest_id) + " chan " + std::to_string(e.channel) + " weight " +
                     dump_dev(e.weight) + " guards " + std::to_string(e.guards.size()) + " updates " +
                     std::to_string(e.updates.size()) + "\n";
                for (const DevGuard &g : e.guards) o += "    guard " + dump_guard(g) + "\n";
                for (const DevUpdate &u : e.updates)
                    o += "    update V" + std::to_string(u.var) + " " + dump_dev(u.expr) + "\n";
            }
        }
    }
    o += "end\n";
    return o;
}

// ---- packer ----------------------------------------------------------------------
namespace {

class Packer {
  public:
    explicit Packer(const DevModel &m) : m_(m) {}

    std::vector<uint8_t> pack() {
        const uint32_t nv = static_cast<uint32_t>(m_.var_kind_clock.size());
        if (m_.comps.empty()) fail("network has no components");
        csmc_net_header h;
        std::memset(&h, 0, sizeof h);
        for (const DevComp &c : m_.comps) {
            if (c.locs.empty()) fail("component '" + c.name + "' has no locations");
            if (c.init_local < 0) fail("component '" + c.name + "' has no initial location");
            if (c.locs.size() > 65535) fail("too many locations in one component");
            csmc_comp pc;
            pc.loc_begin = static_cast<uint32_t>(locs_.size());
            pc.n_locs = static_cast<uint16_t>(c.locs.size());
            pc.init_local = static_cast<uint16_t>(c.init_local);
            comps_.push_back(pc);
            h.max_locs_per_comp = std::max<uint32_t>(h.max_locs_per_comp, pc.n_locs);
            for (const DevLoc &L : c.locs) {
                csmc_loc pl;
                std::memset(&pl, 0, sizeof pl);
                pl.edge_begin = static_cast<uint32_t>(edges_.size());
                pl.inv_begin = static_cast<uint32_t>(guards_.size());
                pl.rate = handle(L.lambda, nv);
                pl.type = static_cast<uint8_t>(L.type);
                // invariants the delay computation acts on: variable-based,
                // upper bound (< or <=), on a clock (simulation.cu:461-511)
                uint32_t ninv = 0;
                for (const DevGuard &g : L.invariants) {
                    if (!g.var_based || g.var < 0 || !g.var_is_clock) continue;
                    if (g.op != COp::Lt && g.op != COp::Le) continue;
                    csmc_guard pg;
                    pg.var = static_cast<uint16_t>(g.var);
                    pg.op = g.op == COp::Lt ? CSMC_G_LT : CSMC_G_LE;
                    pg.clock = 1;
                    pg.rhs = handle(g.rhs, nv);
                    guards_.push_back(pg);
                    ++ninv;
                }
                if (ninv > 255) fail("too many invariants on one location");
                pl.n_inv = static_cast<uint8_t>(ninv);
                h.max_inv_per_loc = std::max(h.max_inv_per_loc, ninv);
                if (L.edges.size() > CSMC_MAX_EDGES_PER_LOC)
                    fail("location id" + std::to_string(L.id - 1) + " has more than " +
                         std::to_string(CSMC_MAX_EDGES_PER_LOC) + " outgoing edges");
                pl.n_edges = static_cast<uint8_t>(L.edges.size());
                h.max_edges_per_loc = std::max<uint32_t>(h.max_edges_per_loc, pl.n_edges);
                uint32_t nrecv = 0;
                for (const DevEdge &e : L.edges) {
                    if (e.channel < 0) ++nrecv;
                    if (e.channel > 32767 || e.channel < -32767) fail("channel id out of range");
                    h.n_channels_max = std::max<uint32_t>(h.n_channels_max, static_cast<uint32_t>(std::abs(e.channel)));
                }
                pl.n_recv = static_cast<uint8_t>(nrecv);
                for (const DevEdge &e : L.edges) {
                    if (e.channel >= 0) continue;
                    const uint32_t ch = static_cast<uint32_t>(-e.channel);
                    if (ch < 32) h.recv_chan_lo |= 1u << ch;
                    else if (ch < 63) h.recv_chan_hi |= 1u << (ch - 32);
                    else h.recv_chan_hi |= 1u << 31;
                }
                locs_.push_back(pl);
                // edges are appended after all locations of the component so
                // that a location's edges stay contiguous
                for (const DevEdge &e : L.edges) pending_.push_back(&e);
                pending_loc_.push_back(static_cast<uint32_t>(locs_.size() - 1));
                pending_cnt_.push_back(static_cast<uint32_t>(L.edges.size()));
                flush_edges(nv, h);
            }
        }
        if (nv > 65535) fail("too many variables");
        std::vector<uint16_t> clocks;
        for (uint32_t i = 0; i < nv; ++i) {
            csmc_var v;
            v.init = static_cast<float>(m_.var_init[i]);
            v.kind = m_.var_kind_clock[i] ? 1u : 0u;
            if (v.kind) {
                ++h.n_clocks;
                clocks.push_back(static_cast<uint16_t>(i));
            }
            vars_.push_back(v);
        }
        // rate slots: literal rates pre-inverted on the host, other rate
        // expressions deduplicated into a per-step program table
        std::vector<uint16_t> loc_rate;
        std::vector<float> inv_lit;
        std::vector<uint32_t> rate_prog;
        {
            std::map<uint32_t, uint16_t> lit_slot, prog_slot;
            for (const csmc_loc &pl : locs_) {
                const uint32_t hdl = pl.rate;
                if (CSMC_H_TAG(hdl) == CSMC_H_LIT) {
                    const float inv = csmc::inv_rate(consts_[CSMC_H_PAYLOAD(hdl)]);
                    uint32_t bits;
                    std::memcpy(&bits, &inv, 4);
                    auto it = lit_slot.find(bits);
                    if (it == lit_slot.end()) {
                        it = lit_slot.emplace(bits, static_cast<uint16_t>(inv_lit.size())).first;
                        inv_lit.push_back(inv);
                    }
                    loc_rate.push_back(it->second);
                } else {
                    auto it = prog_slot.find(hdl);
                    if (it == prog_slot.end()) {
                        it = prog_slot.emplace(hdl, static_cast<uint16_t>(rate_prog.size())).first;
                        rate_prog.push_back(hdl);
                    }
                    loc_rate.push_back(static_cast<uint16_t>(it->second | CSMC_RATE_PROG_BIT));
                }
            }
            if (inv_lit.size() >= CSMC_RATE_PROG_BIT) fail("too many distinct rates");
            h.n_rate_prog = static_cast<uint32_t>(rate_prog.size());
            h.n_inv_lit = static_cast<uint32_t>(inv_lit.size());
            if (h.n_rate_prog <= CSMC_MAX_RATE_PROGS) h.flags |= CSMC_NET_RATE_TABLE;
            // whether some rate program reads a clock (then its value changes
            // with every race step, not only with transitions)
            bool reads_clock = false;
            auto is_clock = [&](uint32_t v) { return v < nv && m_.var_kind_clock[v]; };
            for (uint32_t hdl : rate_prog) {
                const uint32_t tag = CSMC_H_TAG(hdl), pl = CSMC_H_PAYLOAD(hdl);
                if (tag == CSMC_H_VAR) {
                    reads_clock |= is_clock(pl);
                } else if (tag == CSMC_H_PN || tag == CSMC_H_TREE) {
                    for (size_t ip = pl + 1; ip < code_.size() && CSMC_INS_OP(code_[ip]) != CSMC_OP_END; ++ip)
                        if (CSMC_INS_OP(code_[ip]) == CSMC_OP_PUSH_V) reads_clock |= is_clock(CSMC_INS_A(code_[ip]));
                }
            }
            if (!reads_clock) h.flags |= CSMC_NET_RATE_NO_CLOCK;
        }
        std::vector<uint64_t> loc_desc;
        std::vector<uint32_t> loc_inv1(locs_.size(), 0u);
        for (size_t i = 0; i < locs_.size(); ++i) {
            const csmc_loc &pl = locs_[i];
            uint32_t flags = 0, lo = 0;
            if (pl.type > 1) flags |= CSMC_DESC_ZERO;
            if (pl.n_inv) flags |= CSMC_DESC_INV;
            if (pl.n_inv == 1) {  // one clock bound by a literal: inline in the kernels
                const csmc_guard &g = guards_[pl.inv_begin];
                const uint32_t k = CSMC_H_PAYLOAD(g.rhs);
                if (CSMC_H_TAG(g.rhs) == CSMC_H_LIT && k < 0x8000u && g.var <= 0xffffu) {
                    flags |= CSMC_DESC_INV1;
                    loc_inv1[i] = (static_cast<uint32_t>(g.var) << 16) | ((g.op == CSMC_G_LT ? 1u : 0u) << 15) | k;
                }
            }
            const uint16_t slot = loc_rate[i];
            if (slot & CSMC_RATE_PROG_BIT) {
                if (h.flags & CSMC_NET_RATE_TABLE) {
                    flags |= CSMC_DESC_PROG;
                    lo = slot & ~CSMC_RATE_PROG_BIT;
                } else {
                    flags |= CSMC_DESC_EVAL;
                }
            } else {
                std::memcpy(&lo, &inv_lit[slot], 4);
            }
            if (flags & CSMC_DESC_EVAL) {  // the inline invariant path reads the rate from the descriptor
                flags &= ~CSMC_DESC_INV1;
                loc_inv1[i] = 0u;
            }
            loc_desc.push_back(static_cast<uint64_t>(lo) | (static_cast<uint64_t>(flags) << 32));
        }
        // race classes: always-exponential locations sharing the source of
        // their 1/rate (a literal of finite positive value, or one per-step
        // rate program) of at least two locations.  With more than
        // CSMC_RACE_CLASSES such sources, the ones with the most locations
        // get classes (ids in order of first appearance) and the other
        // locations race through their descriptor.
        {
            auto class_key = [](uint64_t d, uint64_t &key) {
                const uint32_t fl = static_cast<uint32_t>(d >> 32), lo = static_cast<uint32_t>(d);
                float inv;
                std::memcpy(&inv, &lo, 4);
                const bool lit_ok = (fl & CSMC_DESC_PROG) || (inv > 0.0f && inv <= std::numeric_limits<float>::max());
                key = d & (0xffffffffull | (static_cast<uint64_t>(CSMC_DESC_PROG) << 32));
                return !(fl & (CSMC_DESC_ZERO | CSMC_DESC_INV | CSMC_DESC_EVAL)) && lit_ok;
            };
            std::vector<uint64_t> order;  // keys in order of first appearance
            std::map<uint64_t, uint32_t> count;
            for (uint64_t d : loc_desc) {
                uint64_t key;
                if (!class_key(d, key)) continue;
                if (!count[key]++) order.push_back(key);
            }
            // a source shared by a single location gains nothing from a class
            std::vector<uint64_t> ranked;
            for (uint64_t key : order)
                if (count[key] >= 2) ranked.push_back(key);
            std::stable_sort(ranked.begin(), ranked.end(),
                             [&](uint64_t a, uint64_t b) { return count[a] > count[b]; });
            if (ranked.size() > CSMC_RACE_CLASSES) ranked.resize(CSMC_RACE_CLASSES);
            std::map<uint64_t, uint32_t> cls;
            for (uint64_t key : order)
                if (std::find(ranked.begin(), ranked.end(), key) != ranked.end())
                    cls.emplace(key, static_cast<uint32_t>(cls.size()));
            for (uint64_t &d : loc_desc) {
                uint64_t key;
                uint32_t c = CSMC_DESC_NO_CLASS;
                if (class_key(d, key)) {
                    auto it = cls.find(key);
                    if (it != cls.end()) c = it->second;
                }
                d |= static_cast<uint64_t>(c << 8) << 32;
            }
            if (comps_.size() <= 256 && !cls.empty()) {
                h.flags |= CSMC_NET_RACE_CLASSES;
                h.n_classes = static_cast<uint32_t>(cls.size());
            }
        }
        h.magic = CSMC_NET_MAGIC;
        h.version = CSMC_NET_VERSION;
        h.header_bytes = sizeof(csmc_net_header);
        h.n_comps = static_cast<uint32_t>(comps_.size());
        h.n_locs = static_cast<uint32_t>(locs_.size());
        h.n_edges = static_cast<uint32_t>(edges_.size());
        h.n_guards = static_cast<uint32_t>(guards_.size());
        h.n_updates = static_cast<uint32_t>(updates_.size());
        h.n_vars = nv;
        h.n_consts = static_cast<uint32_t>(consts_.size());
        h.n_code = static_cast<uint32_t>(code_.size());
        h.max_stack = max_stack_;
        std::vector<uint8_t> out(sizeof(csmc_net_header), 0);
        auto section = [&](const void *p, size_t bytes) {
            while (out.size() % 16) out.push_back(0);
            const uint32_t off = static_cast<uint32_t>(out.size());
            out.insert(out.end(), static_cast<const uint8_t *>(p), static_cast<const uint8_t *>(p) + bytes);
            return off;
        };
        h.off_comp = section(comps_.data(), comps_.size() * sizeof(csmc_comp));
        h.off_loc = section(locs_.data(), locs_.size() * sizeof(csmc_loc));
        h.off_edge = section(edges_.data(), edges_.size() * sizeof(csmc_edge));
        h.off_guard = section(guards_.data(), guards_.size() * sizeof(csmc_guard));
        h.off_update = section(updates_.data(), updates_.size() * sizeof(csmc_update));
        h.off_var = section(vars_.data(), vars_.size() * sizeof(csmc_var));
        h.off_const = section(consts_.data(), consts_.size() * sizeof(double));
        h.off_code = section(code_.data(), code_.size() * sizeof(uint64_t));
        h.off_loc_rate = section(loc_rate.data(), loc_rate.size() * sizeof(uint16_t));
        h.off_inv_lit = section(inv_lit.data(), inv_lit.size() * sizeof(float));
        h.off_rate_prog = section(rate_prog.data(), rate_prog.size() * sizeof(uint32_t));
        h.off_clock = section(clocks.data(), clocks.size() * sizeof(uint16_t));
        h.off_loc_desc = section(loc_desc.data(), loc_desc.size() * sizeof(uint64_t));
        h.off_loc_inv1 = section(loc_inv1.data(), loc_inv1.size() * sizeof(uint32_t));
        while (out.size() % 16) out.push_back(0);
        h.total_bytes = static_cast<uint32_t>(out.size());
        std::memcpy(out.data(), &h, sizeof h);
        return out;
    }

  private:
    const DevModel &m_;
    std::vector<csmc_comp> comps_;
    std::vector<csmc_loc> locs_;
    std::vector<csmc_edge> edges_;
    std::vector<csmc_guard> guards_;
    std::vector<csmc_update> updates_;
    std::vector<csmc_var> vars_;
    std::vector<double> consts_;
    std::vector<uint64_t> code_;
    std::map<uint64_t, uint32_t> const_index_;
    std::map<std::vector<uint64_t>, uint32_t> program_index_;  // identical programs share code
    uint32_t max_stack_ = 1;
    std::vector<const DevEdge *> pending_;
    std::vector<uint32_t> pending_loc_, pending_cnt_;

    void flush_edges(uint32_t nv, csmc_net_header &h) {
        for (size_t k = 0; k < pending_loc_.size(); ++k) {
            locs_[pending_loc_[k]].edge_begin = static_cast<uint32_t>(edges_.size());
            for (uint32_t j = 0; j < pending_cnt_[k]; ++j) {
                const DevEdge &e = *pending_[j];
                csmc_edge pe;
                pe.dst_local = static_cast<int16_t>(e.dest_local);
                pe.channel = static_cast<int16_t>(e.channel);
                pe.weight = handle(e.weight, nv);
                const uint32_t gb = static_cast<uint32_t>(guards_.size());
                uint32_t ng = 0;
                for (const DevGuard &g : e.guards) {
                    if (!g.var_based) continue;  // ignored by the kernel
                    if (g.var < 0) fail("guard on a variable unknown to the registry");
                    csmc_guard pg;
                    pg.var = static_cast<uint16_t>(g.var);
                    switch (g.op) {
                    case COp::Le: pg.op = CSMC_G_LE; break;
                    case COp::Lt: pg.op = CSMC_G_LT; break;
                    case COp::Ge: pg.op = CSMC_G_GE; break;
                    case COp::Gt: pg.op = CSMC_G_GT; break;
                    case COp::Eq: pg.op = CSMC_G_EQ; break;
                    default: pg.op = CSMC_G_FALSE; break;  // "!=" disables the edge (simulation.cu:249-251)
                    }
                    pg.clock = g.var_is_clock ? 1 : 0;
                    pg.rhs = handle(g.rhs, nv);
                    guards_.push_back(pg);
                    ++ng;
                }
                const uint32_t ub = static_cast<uint32_t>(updates_.size());
                for (const DevUpdate &u : e.updates) {
                    if (u.var < 0 || static_cast<uint32_t>(u.var) >= nv)
                        fail("update of variable id " + std::to_string(u.var) + " which is not a variable");
                    csmc_update pu;
                    pu.var = static_cast<uint32_t>(u.var);
                    pu.expr = handle(u.expr, nv);
                    updates_.push_back(pu);
                }
                if (ng > 255 || e.updates.size() > 255) fail("too many guards or updates on one edge");
                if (gb > 0xffffff || ub > 0xffffff) fail("network too large");
                pe.guard_begin = gb | (ng << 24);
                pe.upd = ub | (static_cast<uint32_t>(e.updates.size()) << 24);
                h.max_guards_per_edge = std::max(h.max_guards_per_edge, ng);
                h.max_updates_per_edge = std::max<uint32_t>(h.max_updates_per_edge, static_cast<uint32_t>(e.updates.size()));
                edges_.push_back(pe);
            }
            pending_.erase(pending_.begin(), pending_.begin() + pending_cnt_[k]);
        }
        pending_loc_.clear();
        pending_cnt_.clear();
    }

    uint32_t konst(double v) {
        uint64_t bits;
        std::memcpy(&bits, &v, 8);
        auto it = const_index_.find(bits);
        if (it != const_index_.end()) return it->second;
        const uint32_t i = static_cast<uint32_t>(consts_.size());
        consts_.push_back(v);
        const_index_[bits] = i;
        return i;
    }

    uint32_t var_ref(int var, uint32_t nv) {
        if (var < 0 || static_cast<uint32_t>(var) >= nv)
            fail("expression refers to id " + std::to_string(var) + " which is not a variable");
        return static_cast<uint32_t>(var);
    }

    uint32_t program(std::vector<uint64_t> p, uint32_t tag, uint32_t flags, uint32_t depth) {
        auto push = [](uint64_t i) {
            const uint32_t o = CSMC_INS_OP(i);
            return o == CSMC_OP_PUSH_C || o == CSMC_OP_PUSH_V;
        };
        auto binop = [](uint64_t i) {
            const uint32_t o = CSMC_INS_OP(i);
            return o == CSMC_OP_ADD || o == CSMC_OP_SUB || o == CSMC_OP_MUL || o == CSMC_OP_DIV ||
                   o == CSMC_OP_TADD || o == CSMC_OP_TSUB || o == CSMC_OP_TMUL;
        };
        if ((p.size() == 3 && push(p[0]) && push(p[1]) && binop(p[2])) ||
            (p.size() == 5 && push(p[0]) && push(p[1]) && binop(p[2]) && push(p[3]) && binop(p[4])))
            flags |= CSMC_PROG_CHAIN;
        p.insert(p.begin(), CSMC_INS(CSMC_OP_HDR, flags | (depth << 8)));
        p.push_back(CSMC_INS(CSMC_OP_END, 0));
        std::vector<uint64_t> key = p;
        key.push_back(tag);
        auto it = program_index_.find(key);
        if (it != program_index_.end()) return it->second;
        const uint32_t start = static_cast<uint32_t>(code_.size());
        code_.insert(code_.end(), p.begin(), p.end());
        program_index_[key] = start;
        return start;
    }

    // PN records -> instructions; stack depth bound = number of pushes on the
    // longest path (the reference stack grows by one per record).
    uint32_t pn_program(const std::vector<Expr> &pn, uint32_t nv) {
        std::vector<uint64_t> p;
        uint32_t pushes = 0;
        bool window = true;
        for (const Expr &r : pn) {
            uint32_t op;
            uint32_t a = 0;
            switch (r.op) {
            case Op::Lit: op = CSMC_OP_PUSH_C; a = konst(r.value); break;
            case Op::Var: op = CSMC_OP_PUSH_V; a = var_ref(r.var, nv); break;
            case Op::Random: op = CSMC_OP_RANDOM; break;
            case Op::Plus: op = CSMC_OP_ADD; break;
            case Op::Minus: op = CSMC_OP_SUB; break;
            case Op::Mul: op = CSMC_OP_MUL; break;
            case Op::Div: op = CSMC_OP_DIV; break;
            case Op::Pow: op = CSMC_OP_POW; break;
            case Op::Neg: op = CSMC_OP_NEG; break;
            case Op::Sqrt: op = CSMC_OP_SQRT; break;
            case Op::Mod: op = CSMC_OP_MOD; break;
            case Op::And: op = CSMC_OP_AND; break;
            case Op::Or: op = CSMC_OP_OR; break;
            case Op::Le: op = CSMC_OP_LE; break;
            case Op::Ge: op = CSMC_OP_GE; break;
            case Op::Lt: op = CSMC_OP_LT; break;
            case Op::Gt: op = CSMC_OP_GT; break;
            case Op::Eq: op = CSMC_OP_EQ; break;
            case Op::Ne: op = CSMC_OP_NE; break;
            case Op::Not: op = CSMC_OP_NOT; break;
            case Op::Cond: op = CSMC_OP_DUP; break;
            case Op::PnSkip: op = CSMC_OP_SKIP; a = static_cast<uint32_t>(r.var); break;
            default: op = CSMC_OP_ZERO; break;
            }
            if (op != CSMC_OP_SKIP) ++pushes;
            else window = false;
            p.push_back(CSMC_INS(op, a));
        }
        if (pushes > CSMC_MAX_STACK)
            fail("expression needs " + std::to_string(pushes) + " stack entries (limit " +
                 std::to_string(CSMC_MAX_STACK) + "; the reference kernel overflows beyond 10)");
        max_stack_ = std::max(max_stack_, pushes);
        return program(p, CSMC_H_PN, window ? CSMC_PROG_WINDOW : 0u, pushes);
    }

    // Tree -> postfix with the recursive evaluator's semantics.
    void tree_emit(const Expr *e, std::vector<uint64_t> &p, uint32_t nv, uint32_t depth, uint32_t &maxd) {
        maxd = std::max(maxd, depth + 1);
        if (e->op == Op::Lit) { p.push_back(CSMC_INS(CSMC_OP_PUSH_C, konst(e->value))); return; }
        if (e->op == Op::Var) { p.push_back(CSMC_INS(CSMC_OP_PUSH_V, var_ref(e->var, nv))); return; }
        uint32_t op = 0;
        switch (e->op) {
        case Op::Plus: op = CSMC_OP_TADD; break;
        case Op::Minus: op = CSMC_OP_TSUB; break;
        case Op::Mul: op = CSMC_OP_TMUL; break;
        case Op::Div: op = CSMC_OP_TDIV; break;
        default: break;
        }
        if (op == 0 || !e->l || !e->r) {  // unsupported by the tree evaluator: 0.0
            p.push_back(CSMC_INS(CSMC_OP_PUSH_C, konst(0.0)));
            return;
        }
        tree_emit(e->l, p, nv, depth, maxd);
        tree_emit(e->r, p, nv, depth + 1, maxd);
        p.push_back(CSMC_INS(op, 0));
    }

    uint32_t handle(const DevExpr &d, uint32_t nv) {
        switch (d.kind) {
        case 0: return CSMC_H_MAKE(CSMC_H_LIT, konst(d.value));
        case 1: return CSMC_H_MAKE(CSMC_H_VAR, var_ref(d.var, nv));
        case 2: return CSMC_H_MAKE(CSMC_H_PN, pn_program(d.pn, nv));
        default: {
            std::vector<uint64_t> p;
            uint32_t maxd = 0;
            tree_emit(d.tree, p, nv, 0, maxd);
            if (maxd > CSMC_MAX_STACK) fail("expression tree too deep");
            max_stack_ = std::max(max_stack_, maxd);
            return CSMC_H_MAKE(CSMC_H_TREE, program(p, CSMC_H_TREE, maxd <= 2 ? CSMC_PROG_WINDOW : 0u, maxd));
        }
        }
    }
};

}  // namespace

std::vector<uint8_t> pack_device_model(const DevModel &m) {
    Packer p(m);
    return p.pack();
}

}  // namespace csmc
