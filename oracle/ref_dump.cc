// ref_dump: runs the UNMODIFIED reference BFS (hybrid_bfs.cc, graph_base.h,
// dist_edge_list.cc, edge_list.cc, lcg.h) on an el64 file and writes its
// results in a binary form the parity tests read.
//
// Test infrastructure only.  It is compiled against the reference sources
// where they lie (oracle/Makefile) and never shipped or called by the product.
//
// The reference class exposes no accessor for its parent array, so this
// driver opens the private members of hybrid_bfs / sliding_queue for reading
// (the "#define private public" below, applied only to the reference's own
// headers, after every standard header they use has been included).  It reads:
//   * parent_     (hybrid_bfs.h:15)  -> the reference's own BFS tree
//   * new_parent_ (hybrid_bfs.h:17)  -> >= 0 exactly for vertices that a
//                                       bottom-up step discovered
//                                       (hybrid_bfs.cc:111-143), which pins the
//                                       direction of every non-empty level
//   * queue_.head_ptr_[0..window_)   -> level boundaries of the sliding queue
//                                       (sliding_queue.h:77-84)
//
// Output file layout (little endian):
//   char[8] "BDREF001"
//   int64 n, num_edges, num_roots, has_graph
//   if has_graph: int64 offsets[n+1], int64 adjacency[2*num_edges]
//   per root:
//     int64 root, check_ok, m_c; double time_ms; int64 num_windows,
//     int64 heads[num_windows], int64 parent[n], uint8 bottom_up_flag[n]
#include <algorithm>
#include <atomic>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <getopt.h>
#include <iterator>
#include <memory>
#include <numeric>
#include <queue>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "graph.h"
#include "dist_edge_list.h"
#include "hybrid_bfs.h"
#include "lcg.h"
#undef private
#undef protected

static void die(const char *msg)
{
    fprintf(stderr, "ref_dump: %s\n", msg);
    exit(2);
}

static void put(FILE *f, const void *p, size_t bytes)
{
    if (bytes && fwrite(p, 1, bytes, f) != bytes) { die("write failed"); }
}

static void put64(FILE *f, int64_t v) { put(f, &v, 8); }

int main(int argc, char **argv)
{
    const char *graph_path = nullptr;
    const char *out_path = nullptr;
    const char *alg = "beamer_hybrid";
    long alpha = 15, beta = 18, num_roots = 8, seed = 0;
    bool dump_graph = false;
    std::vector<long> explicit_roots;

    static const struct option opts[] = {
        {"graph_filename", required_argument, nullptr, 'g'},
        {"out", required_argument, nullptr, 'o'},
        {"algorithm", required_argument, nullptr, 'a'},
        {"alpha", required_argument, nullptr, 'A'},
        {"beta", required_argument, nullptr, 'B'},
        {"num_trials", required_argument, nullptr, 'n'},
        {"seed", required_argument, nullptr, 's'},
        {"source_vertex", required_argument, nullptr, 'v'},
        {"dump_graph", no_argument, nullptr, 'd'},
        {nullptr, 0, nullptr, 0},
    };
    int c, idx;
    while ((c = getopt_long(argc, argv, "", opts, &idx)) != -1) {
        switch (c) {
            case 'g': graph_path = optarg; break;
            case 'o': out_path = optarg; break;
            case 'a': alg = optarg; break;
            case 'A': alpha = atol(optarg); break;
            case 'B': beta = atol(optarg); break;
            case 'n': num_roots = atol(optarg); break;
            case 's': seed = atol(optarg); break;
            case 'v': explicit_roots.push_back(atol(optarg)); break;
            case 'd': dump_graph = true; break;
            default: die("bad arguments");
        }
    }
    if (!graph_path || !out_path) { die("need --graph_filename and --out"); }

    auto dist_el = dist_edge_list::load_binary(graph_path);
    auto g = create_graph_from_edge_list<graph>(*dist_el);
    const long n = g->num_vertices();
    const long m = g->num_edges();

    std::vector<long> roots = explicit_roots;
    if (roots.empty()) {
        // Same picker as hybrid_bfs_main.cc:136-144,159.
        lcg rng((unsigned long)seed);
        for (long s = 0; s < num_roots; ++s) {
            long source;
            do { source = rng() % n; } while (g->out_degree(source) == 0);
            roots.push_back(source);
        }
    }

    FILE *f = fopen(out_path, "wb");
    if (!f) { die("cannot open output"); }
    put(f, "BDREF001", 8);
    put64(f, n);
    put64(f, m);
    put64(f, (int64_t)roots.size());
    put64(f, dump_graph ? 1 : 0);
    if (dump_graph) {
        int64_t off = 0;
        put64(f, off);
        for (long v = 0; v < n; ++v) { off += g->out_degree(v); put64(f, off); }
        for (long v = 0; v < n; ++v) {
            auto *e = g->out_neighbors(v);
            for (long k = 0; k < g->out_degree(v); ++k) { put64(f, e[k].dst); }
        }
    }

    auto bfs = emu::make_repl_shallow<hybrid_bfs>(*g);
    std::vector<uint8_t> flag(n);
    for (long source : roots) {
        if (source < 0 || source >= n) { die("root out of range"); }
        bfs->clear();
        hooks_region_begin("bfs");
        if (!strcmp(alg, "beamer_hybrid")) {
            bfs->run_beamer(source, alpha, beta);
        } else if (!strcmp(alg, "migrating_threads")) {
            bfs->run_with_migrating_threads(source);
        } else if (!strcmp(alg, "remote_writes")) {
            bfs->run_with_remote_writes(source);
        } else if (!strcmp(alg, "remote_writes_hybrid")) {
            bfs->run_with_remote_writes_hybrid(source, alpha, beta);
        } else {
            die("unknown algorithm");
        }
        double ms = hooks_region_end();
        int64_t ok = bfs->check(source) ? 1 : 0;
        int64_t mc = bfs->count_num_traversed_edges();
        put64(f, source);
        put64(f, ok);
        put64(f, mc);
        put(f, &ms, 8);
        sliding_queue &q = bfs->queue_;
        put64(f, q.window_);
        for (long w = 0; w < q.window_; ++w) { put64(f, q.head_ptr_[w]); }
        for (long v = 0; v < n; ++v) { put64(f, bfs->parent_[v]); }
        for (long v = 0; v < n; ++v) { flag[v] = bfs->new_parent_[v] >= 0 ? 1 : 0; }
        put(f, flag.data(), (size_t)n);
    }
    fclose(f);
    return 0;
}
