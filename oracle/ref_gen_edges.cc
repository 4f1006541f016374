// ref_gen_edges: runs the UNMODIFIED reference RMAT generator
// (generator/rmat_generator.h: sitmo::prng_engine stream, next_edge,
// rmat_fill with its serial self-loop re-roll) and the first three
// post-processing steps of generator/rmat_dataset_dump.cc:48-53 (flip_edges,
// sort_edges, dedup_edges from generator/edge_list_utils.h), and writes the
// edge lists the parity tests read.  The vertex relabel and the edge shuffle
// that follow in rmat_dataset_dump.cc:55-57 use std::random_shuffle, whose
// output depends on the thread count under the parallel libstdc++ mode, so
// they are left out: the deduplicated, sorted list is the reproducible part.
//
// Test infrastructure only.  Compiled serially (no OpenMP: rmat_fill's
// parallel loop runs as OMP_NUM_THREADS=1 would) against the reference
// sources where they lie (oracle/Makefile); never shipped or called by the
// product.
//
//   ref_gen_edges <scale> <edge_factor> <a> <b> <c> <d> <seed> <out>
//
// Output (little endian): char[8] "BDGEN001", int64 num_vertices,
// int64 generated edges E, int64 E x {src, dst} in generation order (after
// the self-loop re-roll), int64 deduplicated edges m, int64 m x {src, dst}.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "generator/edge_list_utils.h"
#include "generator/rmat_generator.h"

int main(int argc, char **argv)
{
    if (argc != 9) {
        fprintf(stderr, "usage: %s scale edge_factor a b c d seed out\n", argv[0]);
        return 2;
    }
    const int scale = atoi(argv[1]);
    const int64_t edge_factor = atoll(argv[2]);
    const double a = atof(argv[3]), b = atof(argv[4]), c = atof(argv[5]), d = atof(argv[6]);
    const uint32_t seed = (uint32_t)strtoul(argv[7], nullptr, 10);
    const int64_t nv = (int64_t)1 << scale;
    const int64_t num_edges = edge_factor * nv;

    rmat_edge_generator generator(nv, a, b, c, d, seed);
    pvector<edge> edges(num_edges);
    rmat_fill(generator, edges.begin(), edges.end());
    std::vector<edge> generated(edges.begin(), edges.end());
    flip_edges(edges.begin(), edges.end());
    sort_edges(edges.begin(), edges.end());
    edge *new_end = dedup_edges(edges.begin(), edges.end());
    const int64_t m = new_end - edges.begin();

    FILE *fp = fopen(argv[8], "wb");
    if (!fp) { return 1; }
    fwrite("BDGEN001", 1, 8, fp);
    fwrite(&nv, 8, 1, fp);
    fwrite(&num_edges, 8, 1, fp);
    fwrite(generated.data(), sizeof(edge), generated.size(), fp);
    fwrite(&m, 8, 1, fp);
    fwrite(edges.begin(), sizeof(edge), (size_t)m, fp);
    fclose(fp);
    return 0;
}
