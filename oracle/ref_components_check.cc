// ref_components_check: runs the UNMODIFIED reference components::check
// (components.cc:155-200) on labellings read from a file, so the oracle's
// restatement of that rule can be compared with the reference on wrong
// labellings too, not only on the reference's own results.
//
// Test infrastructure only.  It is compiled against the reference sources
// where they lie (oracle/Makefile) and never shipped or called by the product.
// component_ is a public member of the reference class (components.h:13), so
// each labelling is written into it before check() runs.
//
//   ref_components_check --graph_filename G --labels L
//
// L (little endian): int64 k, int64 n, then k x n int64 labels.  Prints one
// line "VERDICT <0|1>" per labelling, in order.
#include <getopt.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "components.h"
#include "dist_edge_list.h"
#include "graph.h"

static void die(const char *msg)
{
    fprintf(stderr, "ref_components_check: %s\n", msg);
    exit(2);
}

int main(int argc, char **argv)
{
    const char *graph_path = nullptr;
    const char *labels_path = nullptr;
    static const struct option opts[] = {
        {"graph_filename", required_argument, nullptr, 'g'},
        {"labels", required_argument, nullptr, 'l'},
        {nullptr, 0, nullptr, 0},
    };
    int c, idx;
    while ((c = getopt_long(argc, argv, "", opts, &idx)) != -1) {
        switch (c) {
            case 'g': graph_path = optarg; break;
            case 'l': labels_path = optarg; break;
            default: die("bad arguments");
        }
    }
    if (!graph_path || !labels_path) { die("need --graph_filename and --labels"); }

    auto dist_el = dist_edge_list::load_binary(graph_path);
    auto g = create_graph_from_edge_list<graph>(*dist_el);
    const long n = g->num_vertices();

    FILE *f = fopen(labels_path, "rb");
    if (!f) { die("cannot open labels"); }
    int64_t k = 0, ln = 0;
    if (fread(&k, 8, 1, f) != 1 || fread(&ln, 8, 1, f) != 1) { die("short labels header"); }
    if (ln != n) { die("label count differs from the graph's vertex count"); }
    std::vector<int64_t> labels(n);

    auto cc = emu::make_repl_shallow<components>(*g);
    for (int64_t i = 0; i < k; ++i) {
        if (fread(labels.data(), 8, n, f) != (size_t)n) { die("short labels body"); }
        for (long v = 0; v < n; ++v) { cc->component_[v] = labels[v]; }
        const bool ok = cc->check();
        printf("VERDICT %d\n", ok ? 1 : 0);
        fflush(stdout);
    }
    fclose(f);
    return 0;
}
