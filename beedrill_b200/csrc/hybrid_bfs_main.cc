// hybrid_bfs -- command line driver with the reference's flags
// (hybrid_bfs_main.cc:10-27, 65-132) and output lines (:175-306), running the
// B200 BFS through the C++ facade.
//
// Added flags (not in the reference):
//   --rmat_scale N     generate a seeded RMAT graph on the device instead of
//                      loading --graph_filename (edge factor --edge_factor,
//                      seed --seed)
//   --min_parent       deterministic parents: smallest neighbour one level up
//   --dump_depths F    write the int32 depth array of the last trial to F
//   --root_seed S      lcg(S) instead of lcg(0) for the root picker
//   --policy_file F    trained direction policy for --algorithm learned
//                      (default: ../policy/learned_policy.json, or
//                      learned_policy_batched.json with --batched, beside
//                      this binary's directory)
//   --batched          run all trials' roots together (64 per group, one
//                      captured launch); per-root lines report the batch
//                      time divided evenly
//   --degree_order     neighbour lists ordered by neighbour degree, highest
//                      first (results are unchanged)
//   --hub_layout       --degree_order, and the traversal runs on vertices
//                      renumbered by degree (results in the file's ids)
//   --tuning_file F    launch parameters from the autotuner (default:
//                      ../tuning/b200.json beside this binary's directory,
//                      when present)
// Algorithms: the reference's four names plus top_down, bottom_up, learned.
#include <getopt.h>
#include <unistd.h>

#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "beedrill/hybrid_bfs.hpp"

namespace {

const struct option long_options[] = {
    {"graph_filename", required_argument, nullptr, 0},
    {"distributed_load", no_argument, nullptr, 0},
    {"heavy_threshold", required_argument, nullptr, 0},
    {"num_trials", required_argument, nullptr, 0},
    {"source_vertex", required_argument, nullptr, 0},
    {"algorithm", required_argument, nullptr, 0},
    {"alpha", required_argument, nullptr, 0},
    {"beta", required_argument, nullptr, 0},
    {"sort_edge_blocks", no_argument, nullptr, 0},
    {"dump_edge_list", no_argument, nullptr, 0},
    {"check_graph", no_argument, nullptr, 0},
    {"dump_graph", no_argument, nullptr, 0},
    {"check_results", no_argument, nullptr, 0},
    {"version", no_argument, nullptr, 0},
    {"help", no_argument, nullptr, 0},
    {"rmat_scale", required_argument, nullptr, 0},
    {"edge_factor", required_argument, nullptr, 0},
    {"seed", required_argument, nullptr, 0},
    {"root_seed", required_argument, nullptr, 0},
    {"min_parent", no_argument, nullptr, 0},
    {"dump_depths", required_argument, nullptr, 0},
    {"policy_file", required_argument, nullptr, 0},
    {"batched", no_argument, nullptr, 0},
    {"degree_order", no_argument, nullptr, 0},
    {"hub_layout", no_argument, nullptr, 0},
    {"tuning_file", required_argument, nullptr, 0},
    {nullptr, 0, nullptr, 0},
};

void print_help(const char *argv0)
{
    printf("Usage: %s [OPTIONS]\n", argv0);
    printf("\t--graph_filename     Path to graph file to load\n");
    printf("\t--distributed_load   Accepted for compatibility (single GPU: same as a normal load)\n");
    printf("\t--heavy_threshold    Accepted for compatibility (degree binning is automatic)\n");
    printf("\t--num_trials         Run BFS this many times.\n");
    printf("\t--source_vertex      Use this as the source vertex. If unspecified, pick random vertices.\n");
    printf("\t--algorithm          beamer_hybrid | remote_writes_hybrid | migrating_threads |\n"
           "\t                     remote_writes | top_down | bottom_up | learned | none\n");
    printf("\t--alpha              Alpha parameter for direction-optimizing BFS\n");
    printf("\t--beta               Beta parameter for direction-optimizing BFS\n");
    printf("\t--sort_edge_blocks   Sort each neighbour list by vertex id\n");
    printf("\t--dump_edge_list     Print the edge list to stdout after loading (slow)\n");
    printf("\t--check_graph        Validate the constructed graph against the edge list\n");
    printf("\t--dump_graph         Print the graph to stdout after construction (slow)\n");
    printf("\t--check_results      Validate the BFS results (slow)\n");
    printf("\t--rmat_scale N       Generate a seeded RMAT graph of 2^N vertices on the GPU\n");
    printf("\t--edge_factor K      Generated edges per vertex (default 16)\n");
    printf("\t--seed S             Generator seed (default 0)\n");
    printf("\t--root_seed S        Root picker seed (default 0, as the reference)\n");
    printf("\t--min_parent         Deterministic parents (smallest neighbour one level up)\n");
    printf("\t--dump_depths FILE   Write the depth array (int32) of the last trial\n");
    printf("\t--policy_file FILE   Trained direction policy for --algorithm learned\n");
    printf("\t--batched            Run all trials' roots together (64 per group)\n");
    printf("\t--degree_order       Order neighbour lists by neighbour degree\n");
    printf("\t--hub_layout         Traverse with vertices renumbered by degree\n");
    printf("\t--tuning_file FILE   Launch parameters from the autotuner\n");
    printf("\t--version            Print version info\n");
    printf("\t--help               Print command line help\n");
}

struct bfs_args {
    const char *graph_filename = nullptr;
    long num_trials = 1;
    long source_vertex = -1;
    const char *algorithm = "beamer_hybrid";
    long alpha = 15;
    long beta = 18;
    bool sort_edge_blocks = false;
    bool dump_edge_list = false;
    bool check_graph = false;
    bool dump_graph = false;
    bool check_results = false;
    int rmat_scale = 0;
    long edge_factor = 16;
    unsigned long seed = 0;
    unsigned long root_seed = 0;
    bool min_parent = false;
    const char *dump_depths = nullptr;
    const char *policy_file = nullptr;
    bool batched = false;
    bool degree_order = false;
    bool hub_layout = false;
    const char *tuning_file = nullptr;
};

bfs_args parse(int argc, char **argv)
{
    bfs_args a;
    int idx = 0;
    while (true) {
        int c = getopt_long(argc, argv, "", long_options, &idx);
        if (c == -1) { break; }
        if (c == '?') {
            printf("Invalid arguments\n");
            print_help(argv[0]);
            exit(1);
        }
        const std::string name = long_options[idx].name;
        if (name == "graph_filename") { a.graph_filename = optarg; }
        else if (name == "num_trials") { a.num_trials = atol(optarg); }
        else if (name == "source_vertex") { a.source_vertex = atol(optarg); }
        else if (name == "algorithm") { a.algorithm = optarg; }
        else if (name == "alpha") { a.alpha = atol(optarg); }
        else if (name == "beta") { a.beta = atol(optarg); }
        else if (name == "sort_edge_blocks") { a.sort_edge_blocks = true; }
        else if (name == "dump_edge_list") { a.dump_edge_list = true; }
        else if (name == "check_graph") { a.check_graph = true; }
        else if (name == "dump_graph") { a.dump_graph = true; }
        else if (name == "check_results") { a.check_results = true; }
        else if (name == "rmat_scale") { a.rmat_scale = atoi(optarg); }
        else if (name == "edge_factor") { a.edge_factor = atol(optarg); }
        else if (name == "seed") { a.seed = strtoul(optarg, nullptr, 10); }
        else if (name == "root_seed") { a.root_seed = strtoul(optarg, nullptr, 10); }
        else if (name == "min_parent") { a.min_parent = true; }
        else if (name == "dump_depths") { a.dump_depths = optarg; }
        else if (name == "policy_file") { a.policy_file = optarg; }
        else if (name == "batched") { a.batched = true; }
        else if (name == "degree_order") { a.degree_order = true; }
        else if (name == "hub_layout") { a.hub_layout = true; }
        else if (name == "tuning_file") { a.tuning_file = optarg; }
        else if (name == "version") {
            printf("%s\n", bd_version());
            exit(0);
        } else if (name == "help") {
            print_help(argv[0]);
            exit(1);
        }
    }
    if (a.graph_filename == nullptr && a.rmat_scale <= 0) {
        printf("Missing graph filename\n");
        exit(1);
    }
    if (a.num_trials <= 0) { printf("num_trials must be > 0\n"); exit(1); }
    if (a.alpha <= 0) { printf("alpha must be > 0\n"); exit(1); }
    if (a.beta <= 0) { printf("beta must be > 0\n"); exit(1); }
    return a;
}

int alg_code(const char *name)
{
    if (!strcmp(name, "beamer_hybrid") || !strcmp(name, "remote_writes_hybrid")) { return BD_ALG_BEAMER; }
    if (!strcmp(name, "migrating_threads") || !strcmp(name, "remote_writes") ||
        !strcmp(name, "top_down")) {
        return BD_ALG_TOP_DOWN;
    }
    if (!strcmp(name, "bottom_up")) { return BD_ALG_BOTTOM_UP; }
    if (!strcmp(name, "learned")) { return BD_ALG_LEARNED; }
    return -1;
}

// Directory of this binary (beedrill_b200/bin).
std::string binary_dir()
{
    char exe[4096];
    const ssize_t len = readlink("/proc/self/exe", exe, sizeof(exe) - 1);
    if (len <= 0) { return "."; }
    exe[len] = '\0';
    std::string dir = exe;
    const size_t slash = dir.rfind('/');
    return slash == std::string::npos ? "." : dir.substr(0, slash);
}

// The autotuner's launch parameters for a graph of n vertices, if any.
bool find_tuning(const bfs_args &args, long n, beedrill::tuning *t)
{
    const std::string path =
        args.tuning_file ? args.tuning_file : binary_dir() + "/../tuning/b200.json";
    if (access(path.c_str(), R_OK) != 0) {
        if (args.tuning_file) { throw beedrill::error(BD_ERR_IO, "tuning file " + path); }
        return false;
    }
    *t = beedrill::load_tuning(path, n);
    return true;
}

// The trained policy beside this binary (beedrill_b200/bin -> beedrill_b200/policy).
std::string default_policy(bool batched)
{
    return binary_dir() +
           (batched ? "/../policy/learned_policy_batched.json" : "/../policy/learned_policy.json");
}

// Loads the policy for --algorithm learned; without a file the rule decides.
bool find_policy(const bfs_args &args, beedrill::policy *pol)
{
    const std::string path = args.policy_file ? args.policy_file : default_policy(args.batched);
    if (access(path.c_str(), R_OK) != 0) {
        if (args.policy_file) { throw beedrill::error(BD_ERR_IO, "policy file " + path); }
        printf("No policy file %s: the rule decides every step\n", path.c_str());
        return false;
    }
    *pol = beedrill::load_policy(path);
    return true;
}

void report(long edges, double ms, const std::string &dirs, long *edges_all, double *ms_all,
            double *inv_sum)
{
    *edges_all += edges;
    *ms_all += ms;
    const double mteps = (1e-6 * edges) / (ms / 1000);
    *inv_sum += 1.0 / mteps;
    // the reference's line, character for character (hybrid_bfs_main.cc:297)
    printf("Traversed %li edges in %3.2f ms, %3.2f MTEPS \n", edges, ms, mteps);
    printf("Directions: %s\n", dirs.c_str());
}

bool write_depths(const char *path, const std::vector<int32_t> &d)
{
    FILE *fp = fopen(path, "wb");
    const bool ok = fp && fwrite(d.data(), sizeof(int32_t), d.size(), fp) == d.size();
    if (!ok) { printf("Cannot write %s\n", path); }
    if (fp) { fclose(fp); }
    return ok;
}

// --batched: every trial's root in one call of the batched traversal.
bool run_batched(const bfs_args &args, beedrill::graph &g, int alg, const std::vector<int64_t> &roots)
{
    bool success = true;
    bd_msbfs_opts opts;
    bd_msbfs_default_opts(&opts);
    beedrill::tuning tn;
    if (find_tuning(args, g.num_vertices(), &tn)) { tn.apply(&opts); }
    if (alg == BD_ALG_TOP_DOWN) { opts.force_dir = 0; }
    if (alg == BD_ALG_BOTTOM_UP) { opts.force_dir = 1; }
    // every root's parent_ complete when the run ends, as in the reference
    opts.materialize = 1;
    opts.min_parent = args.min_parent ? 1 : 0;
    beedrill::batched_bfs bfs(g, (int32_t)roots.size(), &opts);
    beedrill::policy pol;
    if (alg == BD_ALG_LEARNED && find_policy(args, &pol)) { bfs.set_policy(pol); }
    printf("Doing breadth-first search from %zu vertices in one batch\n", roots.size());
    bfs.run(roots);
    const double ms = bfs.last_stats().ms / (double)roots.size();
    long edges_all = 0;
    double ms_all = 0, inv_sum = 0;
    for (size_t s = 0; s < roots.size(); ++s) {
        if (args.check_results) {
            const bool ok = bfs.check((int32_t)s);
            printf("Checking results...\n%s\n", ok ? "PASS" : "FAIL");
            success = success && ok;
        }
        report(bfs.count_num_traversed_edges((int32_t)s), ms, "batched", &edges_all, &ms_all,
               &inv_sum);
    }
    if (args.dump_depths) {
        success = write_depths(args.dump_depths, bfs.depths((int32_t)roots.size() - 1)) && success;
    }
    printf("Mean performance over all trials: %3.2f MTEPS \n", (1e-6 * edges_all) / (ms_all / 1000));
    printf("Harmonic mean over all trials: %3.2f MTEPS \n", roots.size() / inv_sum);
    return success;
}

// The reference's load line (hybrid_bfs_main.cc:175-178, components_main.cc:
// 133-136): edges, time, and MB/s of 16-byte edges; here the time covers
// reading or generating the edges and building the CSR on the device.
void print_loaded(const beedrill::graph &g, std::chrono::steady_clock::time_point t0)
{
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const long m = g.num_edges();
    printf("Loaded %li edges in %3.2f ms, %3.2f MB/s\n", m, ms, (1e-6 * m * 16) / (1e-3 * ms));
    printf("Graph has %li vertices\n", g.num_vertices());
}

}  // namespace

int main(int argc, char **argv)
{
    bool success = true;
    bfs_args args = parse(argc, argv);
    try {
        const int32_t order = args.hub_layout         ? BD_ORDER_HUB
                              : args.degree_order     ? BD_ORDER_DEGREE
                              : args.sort_edge_blocks ? BD_ORDER_SORTED
                                                      : BD_ORDER_INSERTION;
        const auto t_load = std::chrono::steady_clock::now();
        beedrill::graph g = args.rmat_scale > 0
                                ? beedrill::graph::rmat(args.rmat_scale, args.edge_factor, args.seed,
                                                        0.57, 0.19, 0.19, 0.05, order)
                                : beedrill::graph::from_el64(args.graph_filename, order);
        print_loaded(g, t_load);
        if (args.dump_edge_list || args.dump_graph) {
            std::vector<int64_t> off;
            std::vector<uint32_t> adj;
            g.csr(off, adj);
            for (long v = 0; v < g.num_vertices(); ++v) {
                if (off[v + 1] == off[v]) { continue; }
                printf("%li ->", v);
                for (int64_t e = off[v]; e < off[v + 1]; ++e) { printf(" %u", adj[e]); }
                printf("\n");
            }
        }
        if (args.check_graph) {
            printf("Checking graph...");
            if (g.check()) {
                printf("PASS\n");
            } else {
                printf("FAIL\n");
                success = false;
            }
        }
        if (args.source_vertex >= g.num_vertices()) {
            printf("Source vertex %li out of range.\n", args.source_vertex);
            exit(1);
        }
        if (!strcmp(args.algorithm, "none")) { return !success; }
        const int alg = alg_code(args.algorithm);
        if (alg < 0) {
            printf("Algorithm '%s' not implemented!\n", args.algorithm);
            exit(1);
        }
        printf("Initializing BFS data structures...\n");
        std::vector<int64_t> roots;
        if (args.source_vertex < 0) {
            roots = g.pick_roots(args.root_seed, args.num_trials);
        } else {
            roots.assign(args.num_trials, args.source_vertex);
        }
        if (args.batched) { return run_batched(args, g, alg, roots) && success ? 0 : 1; }
        bd_bfs_opts opts;
        bd_bfs_default_opts(&opts);
        opts.alg = alg;
        opts.alpha = args.alpha;
        opts.beta = args.beta;
        opts.min_parent = args.min_parent ? 1 : 0;
        beedrill::tuning tn;
        if (find_tuning(args, g.num_vertices(), &tn)) { tn.apply(&opts); }
        beedrill::hybrid_bfs bfs(g, &opts);
        beedrill::policy pol;
        if (alg == BD_ALG_LEARNED && find_policy(args, &pol)) { bfs.set_policy(pol); }
        long edges_all = 0;
        double ms_all = 0, inv_sum = 0;
        for (long s = 0; s < args.num_trials; ++s) {
            const long source = (long)roots[s];
            bfs.clear();
            printf("Doing breadth-first search from vertex %li (sample %li of %li)\n", source, s + 1,
                   args.num_trials);
            bfs.run(source);
            const double ms = bfs.last_stats().ms;
            if (args.check_results) {
                printf("Checking results...\n");
                if (bfs.check(source)) {
                    printf("PASS\n");
                } else {
                    printf("FAIL\n");
                    success = false;
                }
            }
            std::string dirs;
            for (const bd_step &st : bfs.steps()) { dirs += st.dir ? 'B' : 'T'; }
            report(bfs.count_num_traversed_edges(), ms, dirs, &edges_all, &ms_all, &inv_sum);
            if (args.dump_depths && s == args.num_trials - 1) {
                success = write_depths(args.dump_depths, bfs.depths()) && success;
            }
        }
        printf("Mean performance over all trials: %3.2f MTEPS \n",
               (1e-6 * edges_all) / (ms_all / 1000));
        printf("Harmonic mean over all trials: %3.2f MTEPS \n", args.num_trials / inv_sum);
    } catch (const beedrill::error &e) {
        printf("%s\n", e.what());
        return 1;
    }
    return !success;
}
