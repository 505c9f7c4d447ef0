// cusmc: drop-in command line for the reference cuSMC binary.
//
// Same grammar, defaults, messages and exit codes as the reference's main()
// and HandleCommandLineArguments (main.cu:10-110):
//   -m|--model PATH   -s|--seed INT
//   -q|--query SIMS T THRESHOLD VAR_ID IS_MAX IS_ESTIMATE LOC_QUERY
//   -h|--help
// Exit code 1 after a simulation, 0 after -h or a command-line error.
// Options of this build that the reference does not have use the --csmc-
// prefix so the reference grammar stays intact:
//   --csmc-formula TEXT    the query as an UPPAAL formula (Pr[<=T](<> P.loc),
//                          Pr[<=T](<> v >= k), E[<=T; N](max: v)); replaces the
//                          -q fields except SIMS, which the formula's N overrides
//   --csmc-json PATH       JSON summary (estimate, 95% CI, Chernoff-Hoeffding eps)
//   --csmc-runs-csv PATH   every run's flag and tracked value
//   --csmc-is              learned importance sampling for a variable
//                          probability query: CE training of the proposal on
//                          the GPU, then SIMS weighted runs (csmc_smc_is)
//   --csmc-is-ce R,N,S,LR  its CE configuration: at most R rounds of N runs,
//                          S Adam steps per round at step size LR
//                          (default 12,10000,40,0.03)
#include "../../../include/csmc.h"

#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <string>

namespace {

struct Extras {  // the --csmc- options
    std::string formula, json, runs_csv;
    bool is = false;
    csmc_ce_config ce{12, 40, 10000, 1000000, 0.1, 0.03, 1, 0};
};

bool parse_ce(const std::string &v, csmc_ce_config *ce) {
    int r = 0, st = 0;
    unsigned long long n = 0;
    double lr = 0.0;
    char tail = 0;
    if (std::sscanf(v.c_str(), "%d,%llu,%d,%lf%c", &r, &n, &st, &lr, &tail) != 4 || r < 1 || n < 1 || st < 1 ||
        !(lr > 0.0))
        return false;
    ce->rounds = r;
    ce->runs_per_round = n;
    ce->adam_steps = st;
    ce->lr = lr;
    return true;
}

struct StatConfig {  // statistics_Configuration, main.cuh:46-58
    int simulations = 16384;
    int time_bound = 100;
    int threshold = -1;
    int var_id = 1;
    bool is_max = true;
    bool is_estimate = true;
    std::string loc_query;
};

bool handle_args(int argc, char **argv, std::string *filename, int *seed, StatConfig *stats, Extras *ex) {
    for (int i = 1; i < argc; i++) {
        std::string arg = argv[i];
        if (arg == "--csmc-is") {
            ex->is = true;
        } else if (arg == "--csmc-is-ce") {
            if (i + 1 >= argc || !parse_ce(argv[i + 1], &ex->ce)) {
                std::cerr << "Error: --csmc-is-ce requires ROUNDS,RUNS,ADAM_STEPS,LR" << std::endl;
                return false;
            }
            ++i;
        } else if (arg == "--csmc-formula" || arg == "--csmc-json" || arg == "--csmc-runs-csv") {
            if (i + 1 >= argc) {
                std::cerr << "Error: " << arg << " requires a value" << std::endl;
                return false;
            }
            std::string &dst = arg == "--csmc-formula" ? ex->formula : (arg == "--csmc-json" ? ex->json : ex->runs_csv);
            dst = argv[++i];
        } else if (arg == "-m" || arg == "--model") {
            if (i + 1 < argc) {
                *filename = argv[++i];
            } else {
                std::cerr << "Error: -i option requires a value" << std::endl;
                return false;
            }
        } else if (arg == "-s" || arg == "--seed") {
            if (i + 1 < argc) {
                const std::string str = argv[++i];
                try {
                    *seed = std::stoi(str);
                } catch (const std::invalid_argument &e) {
                    std::cerr << "Error: invalid argument: " << e.what() << std::endl;
                    return false;
                } catch (const std::out_of_range &e) {
                    std::cerr << "Error: number too big: " << e.what() << std::endl;
                    return false;
                }
            } else {
                std::cerr << "Error: -s option requires a value" << std::endl;
                return false;
            }
        } else if (arg == "-q" || arg == "--query") {
            if (i + 7 < argc) {
                const std::string sims = argv[++i], tb = argv[++i], thr = argv[++i], vid = argv[++i],
                                  mx = argv[++i], est = argv[++i];
                stats->loc_query = argv[++i];
                try {
                    stats->simulations = std::stoi(sims);
                    stats->time_bound = std::stoi(tb);
                    stats->threshold = std::stoi(thr);
                    stats->var_id = std::stoi(vid);
                    stats->is_max = static_cast<bool>(std::stoi(mx));
                    stats->is_estimate = static_cast<bool>(std::stoi(est));
                } catch (const std::invalid_argument &e) {
                    std::cerr << "Error: invalid argument: " << e.what() << std::endl;
                    return false;
                } catch (const std::out_of_range &e) {
                    std::cerr << "Error: number too big: " << e.what() << std::endl;
                    return false;
                }
            } else {
                std::cerr << "Error: -r option requires a value" << std::endl;
                return false;
            }
        } else if (arg == "-h" || arg == "--help") {
            std::cout << "Use -m or --model, followed by a path, for inputting a path the the model XML file."
                      << std::endl;
            std::cout << "Use -s or --seed, followed by a number, to initialize curand with a constant seed. "
                         "(0 = random seed)"
                      << std::endl;
            std::cout << "Use -q or --query, followed by : number of simulation, time bound, a variable threshold, "
                         "a variable name (id), Max=1 or Min=0, Estimate=1 or Probability=0."
                      << std::endl;
            return false;
        } else {
            std::cerr << "Error: unknown option: " << arg << std::endl;
            return false;
        }
    }
    return true;
}

}  // namespace

int main(int argc, char *argv[]) {
    std::string filename = "../xml_files/LargeModels/aloha_50.xml";
    int seed = 1235;
    StatConfig st;
    Extras ex;
    if (!handle_args(argc, argv, &filename, &seed, &st, &ex)) return 0;
    int rc;
    if (ex.is) {
        csmc_query q{};
        int sims = st.simulations;
        if (!ex.formula.empty()) {
            char buf[512];
            uint64_t n = 0;
            rc = csmc_query_parse(filename.c_str(), ex.formula.c_str(), &q, buf, sizeof buf, &n);
            if (rc != CSMC_OK) {
                std::cerr << "Error: " << csmc_last_error() << std::endl;
                return 0;
            }
            if (n > static_cast<uint64_t>(INT32_MAX)) {
                std::cerr << "Error: the formula's run count " << n << " exceeds " << INT32_MAX << std::endl;
                return 0;
            }
            if (n) sims = static_cast<int>(n);
        } else {
            q.kind = st.var_id == -1 ? CSMC_QUERY_LOCATION : CSMC_QUERY_VARIABLE;
            q.var_id = st.var_id;
            q.is_max = st.is_max ? 1 : 0;
            q.is_estimate = st.is_estimate ? 1 : 0;
            q.threshold = st.threshold;
            q.horizon = st.time_bound;
        }
        rc = csmc_smc_is(filename.c_str(), seed, sims, &q, &ex.ce, ex.json.empty() ? nullptr : ex.json.c_str());
        if (rc != CSMC_OK) std::cerr << "Error: " << csmc_last_error() << std::endl;
        return 1;
    }
    if (ex.formula.empty() && ex.json.empty() && ex.runs_csv.empty()) {
        rc = csmc_smc(filename.c_str(), seed, st.simulations, st.time_bound, st.threshold, st.var_id,
                      st.is_max ? 1 : 0, st.is_estimate ? 1 : 0, st.loc_query.c_str());
    } else {
        csmc_query q{};
        std::string loc = st.loc_query;
        int sims = st.simulations;
        if (!ex.formula.empty()) {
            char buf[512];
            uint64_t n = 0;
            rc = csmc_query_parse(filename.c_str(), ex.formula.c_str(), &q, buf, sizeof buf, &n);
            if (rc != CSMC_OK) {
                std::cerr << "Error: " << csmc_last_error() << std::endl;
                return 0;
            }
            loc = buf;
            if (n > static_cast<uint64_t>(INT32_MAX)) {
                // the report and the timing CSV carry the run count as int
                // (the reference's statistics_Configuration::simulations)
                std::cerr << "Error: the formula's run count " << n << " exceeds " << INT32_MAX << std::endl;
                return 0;
            }
            if (n) sims = static_cast<int>(n);
        } else {
            q.kind = st.var_id == -1 ? CSMC_QUERY_LOCATION : CSMC_QUERY_VARIABLE;
            q.var_id = st.var_id;
            q.is_max = st.is_max ? 1 : 0;
            q.is_estimate = st.is_estimate ? 1 : 0;
            q.threshold = st.threshold;
            q.horizon = st.time_bound;
        }
        rc = csmc_smc_ex(filename.c_str(), seed, sims, &q, loc.c_str(), ex.json.empty() ? nullptr : ex.json.c_str(),
                         ex.runs_csv.empty() ? nullptr : ex.runs_csv.c_str());
    }
    if (rc != CSMC_OK) std::cerr << "Error: " << csmc_last_error() << std::endl;
    return 1;
}
