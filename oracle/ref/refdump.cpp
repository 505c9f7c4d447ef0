/*
 * refdump: runs the REFERENCE front end on one UPPAAL model and prints the
 * network exactly as the reference's simulation kernel receives it, in the
 * canonical text format that cusmc_b200's own front end also prints
 * (csmc_dump_model).  Test infrastructure only: it links the reference's
 * parser objects (built by oracle/ref/Makefile) and is used by
 * tests/golden/make_frontend_golden.py to pin the new front end.
 *
 *   refdump <model.xml> <loc_query> <loc|var>
 *
 * The pipeline is the one in smc.cu:283-436 of the reference (parse,
 * populate_properties, domain_optimization_visitor, pn_compile_visitor,
 * VariableTrackingVisitor, and for location queries the by-name goal marking
 * of smc.cu:407-436).  The walk over nodes/edges/guards/updates/invariants
 * follows init_shared_model_state (simulation/state/shared_model_state.cu:
 * 164-689): components are the parser's subsystems, locations are sorted by
 * node id within a component, edges come from the parser's node->edge map
 * copy taken before optimisation, a guard or invariant is "variable-based"
 * when its constraint uses a variable directly or its left side is a single
 * variable expression (shared_model_state.cu:355-441), and initial values are
 * truncated to int (shared_model_state.cu:282-297).
 */
#include "automata_parser/uppaal_xml_parser.h"
#include "automata_parser/network/domain_optimization_visitor.h"
#include "automata_parser/network/pn_compile_visitor.h"
#include "automata_parser/variable_usage_visitor.h"
#include "automata_parser/network/network_props.h"

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

static const char *op_name(int op) {
    switch (op) {
    case expr::literal_ee: return "lit";
    case expr::clock_variable_ee: return "var";
    case expr::random_ee: return "random";
    case expr::plus_ee: return "+";
    case expr::minus_ee: return "-";
    case expr::multiply_ee: return "*";
    case expr::division_ee: return "/";
    case expr::power_ee: return "^";
    case expr::negation_ee: return "neg";
    case expr::sqrt_ee: return "sqrt";
    case expr::modulo_ee: return "%";
    case expr::and_ee: return "&&";
    case expr::or_ee: return "||";
    case expr::less_equal_ee: return "<=";
    case expr::greater_equal_ee: return ">=";
    case expr::less_ee: return "<";
    case expr::greater_ee: return ">";
    case expr::equal_ee: return "==";
    case expr::not_equal_ee: return "!=";
    case expr::not_ee: return "!";
    case expr::conditional_ee: return "?:";
    case expr::compiled_ee: return "compiled";
    case expr::pn_compiled_ee: return "pn";
    case expr::pn_skips_ee: return "skip";
    }
    return "?";
}

static std::string num(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

// Device form of an expression: what copy_expression_to_device would upload.
static std::string dump_tree(const expr *e) {
    if (!e) return "-";
    if (e->operand == expr::literal_ee) return "L" + num(e->value);
    if (e->operand == expr::clock_variable_ee) return "V" + std::to_string(e->variable_id);
    std::string s = "(";
    s += op_name(e->operand);
    s += " " + dump_tree(e->left) + " " + dump_tree(e->right) + ")";
    return s;
}

static std::string dump_expr(const expr *e) {
    if (!e) return "-";
    if (e->operand == expr::pn_compiled_ee) {
        std::string s = "P" + std::to_string(e->length) + "{";
        for (int i = 1; i < e->length; ++i) {
            const expr &r = e[i];
            if (i > 1) s += ",";
            if (r.operand == expr::literal_ee) s += "L" + num(r.value);
            else if (r.operand == expr::clock_variable_ee) s += "V" + std::to_string(r.variable_id);
            else if (r.operand == expr::pn_skips_ee) s += "S" + std::to_string(r.length);
            else s += op_name(r.operand);
        }
        return s + "}";
    }
    if (e->operand == expr::literal_ee || e->operand == expr::clock_variable_ee) return dump_tree(e);
    return "T" + dump_tree(e);
}

static const char *cop(int op) {
    switch (op) {
    case constraint::less_equal_c: return "<=";
    case constraint::less_c: return "<";
    case constraint::greater_equal_c: return ">=";
    case constraint::greater_c: return ">";
    case constraint::equal_c: return "==";
    case constraint::not_equal_c: return "!=";
    }
    return "compiled";
}

static std::string quote(const std::string &s) {
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

// One guard or invariant in device form (create_variable_guard and the
// non-variable branch of init_shared_model_state).
static std::string dump_constraint(
    const constraint &g,
    const std::unordered_map<int, VariableTrackingVisitor::VariableUsage> &reg) {
    int var = -2;
    if (g.uses_variable) var = g.variable_id;
    else if (g.value != nullptr && g.value->operand == expr::clock_variable_ee) var = g.value->variable_id;
    if (var == -2) return std::string("ignored ") + cop(g.operand);
    std::string kind = "INT";
    auto it = reg.find(var);
    if (it == reg.end()) var = -1;
    else kind = it->second.kind == VariableKind::CLOCK ? "CLOCK" : "INT";
    return std::string(cop(g.operand)) + " V" + std::to_string(var) + " " + kind + " " +
           dump_expr(g.expression);
}

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: refdump model.xml loc_query loc|var\n");
        return 2;
    }
    const std::string file = argv[1];
    const std::string loc_query = argv[2];
    const bool loc_mode = std::string(argv[3]) == "loc";
    try {
        abstract_parser *parser = new uppaal_xml_parser();
        network model = parser->parse(file);
        network_props properties = {};
        populate_properties(properties, parser);

        auto *query_set = new std::unordered_set<std::string>();
        query_set->insert(loc_query);
        domain_optimization_visitor optimizer(query_set, properties.node_network,
                                              properties.node_names, properties.template_names);
        optimizer.optimize(&model);
        pn_compile_visitor pn_compiler;
        pn_compiler.visit(&model);
        VariableTrackingVisitor var_tracker;
        var_tracker.visit(&model);
        const auto &registry = var_tracker.get_variable_registry();
        const int num_vars = static_cast<int>(registry.size());

        std::unordered_map<int, node *> node_map = optimizer.get_node_map();
        if (loc_mode) {  // smc.cu:407-436
            std::string comp, nodename;
            bool dot = false;
            for (char c : loc_query) {
                if (c == '.') { dot = true; continue; }
                (dot ? nodename : comp).push_back(c);
            }
            auto t = properties.node_name_int_map.find(nodename);
            if (t != properties.node_name_int_map.cend()) {
                auto nm = node_map.find(t->second);
                if (nm != node_map.end()) nm->second->type = node::goal;
            }
        }

        const auto &subsys = *optimizer.get_node_subsystems_map();
        const auto &nem = *properties.node_edge_map;
        int max_comp = -1;
        for (const auto &p : subsys) max_comp = std::max(max_comp, p.second);
        std::vector<std::vector<std::pair<int, const std::list<edge> *>>> comps(max_comp + 1);
        for (const auto &p : nem) comps[subsys.at(p.first)].push_back({p.first, &p.second});
        for (auto &c : comps)
            std::sort(c.begin(), c.end(), [](const auto &a, const auto &b) { return a.first < b.first; });

        std::printf("csmc-dump 1\n");
        std::printf("vars %d\n", num_vars);
        for (int i = 0; i < num_vars; ++i) {
            double init = 0.0;
            for (int k = 0; k < model.variables.size; ++k)
                if (model.variables.store[k].id == i) { init = model.variables.store[k].value; break; }
            std::printf("var %d %s %d\n", i,
                        registry.at(i).kind == VariableKind::CLOCK ? "CLOCK" : "INT",
                        static_cast<int>(init));
        }
        std::printf("components %d\n", static_cast<int>(comps.size()));
        for (size_t c = 0; c < comps.size(); ++c) {
            const int init_id = c < static_cast<size_t>(model.automatas.size) ? model.automatas.store[c]->id : -1;
            auto tn = properties.template_names->find(static_cast<int>(c));
            std::printf("comp %zu %s nlocs %zu init %d\n", c,
                        quote(tn == properties.template_names->end() ? "" : tn->second).c_str(),
                        comps[c].size(), init_id);
            for (size_t l = 0; l < comps[c].size(); ++l) {
                const int nid = comps[c][l].first;
                const node *n = node_map.at(nid);
                auto nn = properties.node_names->find(nid);
                std::printf("loc %d %s type %d lambda %s inv %d edges %zu\n", nid,
                            quote(nn == properties.node_names->end() ? "" : nn->second).c_str(),
                            static_cast<int>(n->type), dump_expr(n->lamda).c_str(), n->invariants.size,
                            comps[c][l].second->size());
                for (int i = 0; i < n->invariants.size; ++i)
                    std::printf("  inv %s\n", dump_constraint(n->invariants.store[i], registry).c_str());
                for (const edge &e : *comps[c][l].second) {
                    std::printf("  edge dst %d chan %d weight %s guards %d updates %d\n", e.dest->id,
                                e.channel, dump_expr(e.weight).c_str(), e.guards.size, e.updates.size);
                    for (int g = 0; g < e.guards.size; ++g)
                        std::printf("    guard %s\n", dump_constraint(e.guards.store[g], registry).c_str());
                    for (int u = 0; u < e.updates.size; ++u) {
                        const update &up = e.updates.store[u];
                        std::printf("    update V%d %s\n", up.variable_id, dump_expr(up.expression).c_str());
                    }
                }
            }
        }
        std::printf("end\n");
    } catch (const std::exception &ex) {
        std::printf("csmc-dump 1\nerror %s\n", ex.what());
        return 1;
    }
    return 0;
}
