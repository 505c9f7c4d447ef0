// Front end: UPPAAL XML (the subset the reference accepts) -> model IR ->
// device form -> packed network blob.
//
// The IR keeps the reference's observable semantics, quirks included, because
// the drop-in promise is "same model file, same numbers":
//   * variable ids: globals first, then each template's locals, in
//     declaration order (automata_parser/uppaal_xml_parser.cpp:228-317);
//   * node ids: XML "idN" -> N+1 (automata_parser/string_extractor.cpp:66-70);
//   * constant initialisers folded through float and "%f" text
//     (automata_parser/declaration_parser.cpp:18,33,
//      automata_parser/arithmetic-expression-evaluator.h:292-297);
//   * guards split on '&' with parentheses stripped (helper_methods.h:74-91);
//   * the device form of every expression: guards and edge weights are
//     uploaded as expression trees, invariants, rates and updates as postfix
//     programs (the PN compiler rewrites only the optimizer's copies of the
//     guards and weights, automata_parser/network/pn_compile_visitor.cpp:75-102
//     vs simulation/state/shared_model_state.cu:536-593), with the optimizer's
//     top-level constant folding applied in place
//     (automata_parser/network/domain_optimization_visitor.cpp:432-441).
#pragma once
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

namespace csmc {

// Expression operators; the numbering is the reference's expr::operators
// (include/engine/domain.h:39-75) so dumps can be compared record by record.
enum class Op : uint8_t {
    Lit = 0, Var = 1, Random, Plus, Minus, Mul, Div, Pow, Neg, Sqrt, Mod,
    And, Or, Le, Ge, Lt, Gt, Eq, Ne, Not, Cond, Compiled, PnCompiled, PnSkip
};

struct Expr {
    Op op = Op::Lit;
    double value = 1.0;  // literal value (Lit)
    int var = 0;         // variable id (Var)
    Expr *l = nullptr, *r = nullptr, *els = nullptr;  // els: false branch of Cond
};

// Constraint operators (include/engine/domain.h:100-108).
enum class COp : uint8_t { Le = 0, Lt = 1, Ge = 2, Gt = 3, Eq = 4, Ne = 5 };

struct Constraint {
    COp op = COp::Le;
    bool uses_variable = false;  // left side resolved to a clock by name
    int var = -1;                // when uses_variable
    Expr *value = nullptr;       // left side when !uses_variable
    Expr *expression = nullptr;  // right side
};

struct Update {
    int var = 0;
    Expr *expr = nullptr;
};

struct Edge {
    int channel = 0;  // 0 tau, >0 sender c!, <0 receiver c?
    Expr *weight = nullptr;
    int dest_id = 0;
    std::vector<Constraint> guards;
    std::vector<Update> updates;
};

enum NodeType : int { kLocation = 0, kGoal = 1, kBranch = 2, kUrgent = 3, kCommitted = 4 };

struct Node {
    int id = 0;
    int type = kLocation;
    Expr *lambda = nullptr;
    std::vector<Constraint> invariants;
    int system = 0;  // template index
};

struct VarDecl {
    int id = 0;
    int rate = 0;  // 1 = clock
    double value = 0.0;
};

// A parsed network in the reference's IR shape.
struct Network {
    std::deque<Expr> arena;  // stable addresses
    std::vector<Node> nodes;                           // document order
    std::unordered_map<int, std::vector<Edge>> edges;  // source node id -> edges, document order
    std::vector<VarDecl> vars;                         // id order
    std::vector<std::string> var_names;                // id order: "name" (global), "Template.name" (local)
    std::vector<int> start_nodes;                      // init node id per template (document order)
    std::unordered_map<int, std::string> node_names;   // only named locations
    std::vector<std::pair<int, std::string>> node_name_order;  // insertion order of node_names
    std::unordered_map<int, std::string> template_names;
    std::string system_text;  // the <system> block (process instantiations)
    int n_templates = 0;
    Expr *make(Op op) {
        arena.emplace_back();
        arena.back().op = op;
        return &arena.back();
    }
    Node *node(int id);
};

// Parses a model file; throws std::runtime_error on anything the reference
// front end would reject.
std::unique_ptr<Network> parse_uppaal_file(const std::string &path);
std::unique_ptr<Network> parse_uppaal_text(const std::string &text);

// ---------------------------------------------------------------------------
// Device form: what the simulation kernel receives.

// One compiled expression, as uploaded.  kind: 0 literal, 1 variable,
// 2 postfix program (PN records), 3 expression tree.
struct DevExpr {
    int kind = 0;
    double value = 0.0;
    int var = 0;
    std::vector<Expr> pn;        // kind 2: records 1..len-1 of the PN array (header excluded)
    const Expr *tree = nullptr;  // kind 3
};

struct DevGuard {          // a guard or an invariant as the kernel sees it
    bool var_based = false;  // false: ignored by the kernel
    COp op = COp::Le;
    int var = -1;            // -1 when the variable is unknown to the registry
    bool var_is_clock = false;
    DevExpr rhs;
};

struct DevUpdate {
    int var = 0;
    DevExpr expr;
};

struct DevEdge {
    int dest_id = 0;
    int dest_local = -1;  // index among the component's locations, -1 if absent
    int channel = 0;
    DevExpr weight;
    std::vector<DevGuard> guards;
    std::vector<DevUpdate> updates;
};

struct DevLoc {
    int id = 0;
    std::string name;
    bool named = false;
    int type = kLocation;
    DevExpr lambda;
    std::vector<DevGuard> invariants;
    std::vector<DevEdge> edges;
};

struct DevComp {
    std::string name;
    int init_id = -1;
    int init_local = -1;
    std::vector<DevLoc> locs;  // sorted by node id
};

struct DevModel {
    std::vector<int> var_kind_clock;  // 1 clock, 0 int
    std::vector<int> var_init;        // initial value truncated to int
    std::vector<DevComp> comps;
};

// Runs the reference's passes (goal marking from the query, constant folding,
// PN compilation, the by-name location-query fallback when loc_mode) and
// returns the device form.  Throws std::runtime_error where the reference
// would fail (e.g. a location unreachable from the initial locations).
DevModel build_device_model(Network &net, const std::string &loc_query, bool loc_mode);

// Canonical text dump of the device form (same format as oracle/ref/refdump).
std::string dump_device_model(const DevModel &m);

// Packs the device form into the binary network blob (see csmc_net.h).
std::vector<uint8_t> pack_device_model(const DevModel &m);

// Helpers shared with the CLI.
std::string quote_dump(const std::string &s);

// A query formula of the reference's model files, resolved against a network
// (front/query.cpp).  kind: 0 location, 1 variable; sims: the formula's run
// count (0: none given).
struct QueryText {
    int kind = 0, var_id = -1, is_max = 1, is_estimate = 0;
    double threshold = 0.0, horizon = 0.0;
    uint64_t sims = 0;
    std::string loc_query;
};
QueryText parse_formula(const Network &net, const std::string &formula);

}  // namespace csmc
