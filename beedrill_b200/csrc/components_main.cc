// components -- command line driver with the reference's flags
// (components_main.cc:8-103) and output lines (:105-196), running connected
// components on the device through the C++ facade.
//
// Added flags (not in the reference):
//   --rmat_scale N     generate a seeded RMAT graph on the device instead of
//                      loading --graph_filename (edge factor --edge_factor,
//                      seed --seed)
// GTEPS is printed as the reference computes it: iterations x edges / time
// (one iteration here: a single pass over the arcs).
#include <getopt.h>

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
    {"num_trials", required_argument, nullptr, 0},
    {"dump_edge_list", no_argument, nullptr, 0},
    {"check_graph", no_argument, nullptr, 0},
    {"dump_graph", no_argument, nullptr, 0},
    {"check_results", no_argument, nullptr, 0},
    {"dump_results", no_argument, nullptr, 0},
    {"version", no_argument, nullptr, 0},
    {"help", no_argument, nullptr, 0},
    {"rmat_scale", required_argument, nullptr, 0},
    {"edge_factor", required_argument, nullptr, 0},
    {"seed", required_argument, nullptr, 0},
    {nullptr, 0, nullptr, 0},
};

void print_help(const char *argv0)
{
    printf("Usage: %s [OPTIONS]\n", argv0);
    printf("\t--graph_filename     Path to graph file to load\n");
    printf("\t--distributed_load   Accepted for compatibility (single GPU: same as a normal load)\n");
    printf("\t--num_trials         Run the algorithm this many times.\n");
    printf("\t--dump_edge_list     Print the edge list to stdout after loading (slow)\n");
    printf("\t--check_graph        Validate the constructed graph against the edge list\n");
    printf("\t--dump_graph         Print the graph to stdout after construction (slow)\n");
    printf("\t--check_results      Validate the results\n");
    printf("\t--dump_results       Print the results to stdout (slow)\n");
    printf("\t--rmat_scale N       Generate a seeded RMAT graph of 2^N vertices on the GPU\n");
    printf("\t--edge_factor K      Generated edges per vertex (default 16)\n");
    printf("\t--seed S             Generator seed (default 0)\n");
    printf("\t--version            Print version info\n");
    printf("\t--help               Print command line help\n");
}

struct components_args {
    const char *graph_filename = nullptr;
    long num_trials = 1;
    bool dump_edge_list = false;
    bool check_graph = false;
    bool dump_graph = false;
    bool check_results = false;
    bool dump_results = false;
    int rmat_scale = 0;
    long edge_factor = 16;
    unsigned long seed = 0;
};

components_args parse(int argc, char **argv)
{
    components_args a;
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
        else if (name == "dump_edge_list") { a.dump_edge_list = true; }
        else if (name == "check_graph") { a.check_graph = true; }
        else if (name == "dump_graph") { a.dump_graph = true; }
        else if (name == "check_results") { a.check_results = true; }
        else if (name == "dump_results") { a.dump_results = true; }
        else if (name == "rmat_scale") { a.rmat_scale = atoi(optarg); }
        else if (name == "edge_factor") { a.edge_factor = atol(optarg); }
        else if (name == "seed") { a.seed = strtoul(optarg, nullptr, 10); }
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
    return a;
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
    const components_args args = parse(argc, argv);
    try {
        const auto t_load = std::chrono::steady_clock::now();
        beedrill::graph g = args.rmat_scale > 0
                                ? beedrill::graph::rmat(args.rmat_scale, args.edge_factor, args.seed)
                                : beedrill::graph::from_el64(args.graph_filename);
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
        printf("Initializing data structures...\n");
        beedrill::components cc(g);
        for (long trial = 0; trial < args.num_trials; ++trial) {
            cc.clear();
            printf("Finding connected components...\n");
            const beedrill::components::stats s = cc.run();
            const double teps = (double)s.num_iters * g.num_edges() / (1e-3 * s.ms);
            printf("Found %li components in %li iterations (%3.2f ms, %3.2f GTEPS)\n",
                   (long)s.num_components, (long)s.num_iters, s.ms, 1e-9 * teps);
        }
        if (args.check_results) {
            printf("Checking results...");
            if (cc.check()) {
                printf("PASS\n");
            } else {
                printf("FAIL\n");
                success = false;
            }
        }
        if (args.dump_results) { cc.dump(); }
    } catch (const beedrill::error &e) {
        printf("%s\n", e.what());
        return 1;
    }
    return !success;
}
