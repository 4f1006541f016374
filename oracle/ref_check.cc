// ref_check: runs the UNMODIFIED reference hybrid_bfs::check
// (hybrid_bfs.cc:281-379) on parent arrays read from a file, so the
// oracle's restatement of check() -- its verdict and the vertex at which it
// stops -- can be compared with the reference on wrong trees too.
//
// Test infrastructure only.  It is compiled against the reference sources
// where they lie (oracle/Makefile) and never shipped or called by the product.
// The class keeps its parent array private (hybrid_bfs.h:15), so, as in
// ref_dump.cc, the reference's headers are included with `private` opened
// for writing the array before check() runs.
//
//   ref_check --graph_filename G --parents P [--print_tree]
//
// P (little endian): int64 k, int64 n, then k records of int64 source and
// int64 parent[n].  For record i the output is the line "BEGIN i", whatever
// the reference's check() logs (its LOG lines name the vertex it stops at),
// then "VERDICT i <0|1>".  With --print_tree, print_tree()
// (hybrid_bfs.cc:381-399) runs instead of check(): "BEGIN i", the tree's
// text, "END i".
#include <getopt.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <queue>
#include <string>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "dist_edge_list.h"
#include "graph.h"
#include "hybrid_bfs.h"
#undef private
#undef protected

static void die(const char *msg)
{
    fprintf(stderr, "ref_check: %s\n", msg);
    exit(2);
}

int main(int argc, char **argv)
{
    const char *graph_path = nullptr;
    const char *parents_path = nullptr;
    bool tree = false;
    static const struct option opts[] = {
        {"graph_filename", required_argument, nullptr, 'g'},
        {"parents", required_argument, nullptr, 'p'},
        {"print_tree", no_argument, nullptr, 't'},
        {nullptr, 0, nullptr, 0},
    };
    int c, idx;
    while ((c = getopt_long(argc, argv, "", opts, &idx)) != -1) {
        switch (c) {
            case 'g': graph_path = optarg; break;
            case 'p': parents_path = optarg; break;
            case 't': tree = true; break;
            default: die("bad arguments");
        }
    }
    if (!graph_path || !parents_path) { die("need --graph_filename and --parents"); }

    auto dist_el = dist_edge_list::load_binary(graph_path);
    auto g = create_graph_from_edge_list<graph>(*dist_el);
    const long n = g->num_vertices();

    FILE *f = fopen(parents_path, "rb");
    if (!f) { die("cannot open parents"); }
    int64_t k = 0, pn = 0;
    if (fread(&k, 8, 1, f) != 1 || fread(&pn, 8, 1, f) != 1) { die("short parents header"); }
    if (pn != n) { die("parent count differs from the graph's vertex count"); }
    std::vector<int64_t> parent(n);

    auto bfs = emu::make_repl_shallow<hybrid_bfs>(*g);
    for (int64_t i = 0; i < k; ++i) {
        int64_t source = 0;
        if (fread(&source, 8, 1, f) != 1 || fread(parent.data(), 8, n, f) != (size_t)n) {
            die("short parents body");
        }
        if (source < 0 || source >= n) { die("source out of range"); }
        for (long v = 0; v < n; ++v) { bfs->parent_[v] = parent[v]; }
        printf("BEGIN %ld\n", (long)i);
        fflush(stdout);
        if (tree) {
            bfs->print_tree();
            printf("END %ld\n", (long)i);
            fflush(stdout);
            continue;
        }
        const bool ok = bfs->check(source);
        printf("VERDICT %ld %d\n", (long)i, ok ? 1 : 0);
        fflush(stdout);
    }
    fclose(f);
    return 0;
}
