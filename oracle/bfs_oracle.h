/* bfs_oracle.h -- CPU restatement of the reference's BFS path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (beedrill_b200/, the
 * C-ABI library, the CLI) links, loads or calls this code.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the
 * checker.
 *
 * Each function cites the reference file:line it restates.  Parity of this
 * restatement is pinned against the reference itself: oracle/ref_dump.cc runs
 * the unmodified reference sources and tests/golden/ holds its outputs.
 *
 * Conventions: n vertices, m undirected edges, 2m arcs.  CSR offsets are
 * int64[n+1], adjacency uint32[2m].  Depth is int32 with -1 = unreached.
 * Parents use the reference encoding (hybrid_bfs.cc:433-443 and :152-160):
 * parent[source] = source, a reached vertex holds its parent id (>= 0), an
 * unreached vertex holds -deg(v), or -1 when deg(v) == 0.
 */
#ifndef BD_ORACLE_H
#define BD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- el64 edge-list files (edge_list.cc:20-89, dist_edge_list.cc:63-76) -- */
/* Returns 0 on success, <0 on a malformed header (the reference exits(1)). */
int or_el64_header(const char *path, int64_t *num_vertices, int64_t *num_edges,
                   int64_t *header_bytes);
int or_el64_load(const char *path, int64_t *src, int64_t *dst, int64_t num_edges);
int or_el64_write(const char *path, int64_t num_vertices, int64_t num_edges,
                  const int64_t *src, const int64_t *dst);

/* ---- graph construction (graph_base.h:335-436) --------------------------- */
/* Undirected CSR in the reference's insertion order: for each file edge
 * (s, d) in file order, append d to s's list, then s to d's list. */
int or_csr_build(int64_t n, int64_t m, const int64_t *src, const int64_t *dst,
                 int64_t *offsets, uint32_t *adj);
/* graph::check (graph_base.h:110-134): every file edge present both ways. */
int or_graph_check(int64_t n, int64_t m, const int64_t *src, const int64_t *dst,
                   const int64_t *offsets, const uint32_t *adj);

/* ---- root picker (hybrid_bfs_main.cc:136-144, lcg.h:4-32) ---------------- */
void or_pick_roots(int64_t n, const int64_t *offsets, uint64_t seed, int64_t k,
                   int64_t *roots);

/* ---- BFS oracles ---------------------------------------------------------- */
/* Serial queue BFS exactly as inside check() (hybrid_bfs.cc:285-307). */
void or_bfs_depth(int64_t n, const int64_t *offsets, const uint32_t *adj,
                  int64_t source, int32_t *depth);
/* check(source) (hybrid_bfs.cc:281-379).  Returns 1 = PASS.  `depth_scratch`
 * is int32[n]; on return it holds the serial BFS depths. */
int or_check(int64_t n, const int64_t *offsets, const uint32_t *adj,
             int64_t source, const int64_t *parent, int32_t *depth_scratch);
/* The same check; returns the vertex at which the reference's loop stops
 * (the one its LOG lines name), or -1 on PASS. */
int64_t or_check_first_bad(int64_t n, const int64_t *offsets, const uint32_t *adj,
                           int64_t source, const int64_t *parent, int32_t *depth_scratch);
/* Deterministic tree: parent(v) = min{u in N(v) : depth[u] == depth[v]-1},
 * parent(source) = source, unreached -> reference encoding. */
void or_min_parent(int64_t n, const int64_t *offsets, const uint32_t *adj,
                   int64_t source, const int32_t *depth, int64_t *parent);
/* components::run (components.cc:38-118), serial-elision order; returns
 * the reference's num_iters.  component and size are int64[n]. */
int64_t or_components(int64_t n, const int64_t *offsets, const uint32_t *adj,
                      int64_t *component, int64_t *size, int64_t *num_components);
/* components::check (components.cc:155-200).  Returns 1 = PASS. */
int or_components_check(int64_t n, const int64_t *offsets, const uint32_t *adj,
                        const int64_t *component);
/* count_num_traversed_edges (hybrid_bfs.cc:401-414). */
int64_t or_count_traversed(int64_t n, const int64_t *offsets, const int64_t *parent);

/* Direction sequence of run_beamer (hybrid_bfs.cc:152-191) derived from the
 * per-level profile of a depth array.  Writes one char per step ('T' / 'B')
 * into dirs (NUL terminated) and the number of vertices each step
 * discovered into found[].  Returns the number of steps, or -1 when
 * max_steps is too small. */
int or_beamer_sequence(int64_t n, int64_t m, const int64_t *offsets,
                       const int32_t *depth, int64_t source, int64_t alpha,
                       int64_t beta, char *dirs, int64_t *found, int max_steps);

/* Serial restatement of run_beamer with its top-down step
 * (hybrid_bfs.cc:71-100) and bottom-up step (hybrid_bfs.cc:111-143, using
 * the neighbour order of find.h:14-44).  mode: 0 beamer, 1 top-down only,
 * 2 bottom-up only.  Fills parent (reference encoding), depth, and the
 * direction string like or_beamer_sequence.  Returns the step count. */
int or_run_bfs(int64_t n, int64_t m, const int64_t *offsets, const uint32_t *adj,
               int64_t source, int64_t alpha, int64_t beta, int mode,
               int64_t *parent, int32_t *depth, char *dirs, int max_steps);

/* ---- the project's seeded RMAT generator, restated ----------------------- */
/* Philox4x32-10 (Salmon et al., SC'11): one block of four 32-bit words. */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Raw RMAT edges (rmat_generator.h:91-140 recursion, self loops re-rolled as
 * in :183-189) from a counter-based stream: edge i, attempt t, draw j. */
void or_rmat_edges(int scale, int64_t num_edges, double a, double b, double c,
                   double d, uint64_t seed, int64_t *src, int64_t *dst);
/* Post-processing of rmat_dataset_dump.cc:48-57 with seeded permutations:
 * flip to src<dst, sort, dedup, relabel vertices, shuffle edge order.  Works
 * in place on src/dst; returns the number of edges kept. */
int64_t or_rmat_finish(int scale, int64_t num_edges, uint64_t seed,
                       int64_t *src, int64_t *dst);

/* ---- the reference generator's own stream, restated ---------------------- */
/* Threefish-256 cut to 20 rounds, key (key0, 0, 0, 0), zero tweak, on the
 * counter (block, 0, 0, 0): the block function of sitmo::prng_engine
 * (generator/prng_engine.hpp). */
void or_threefish20(uint64_t key0, uint64_t block, uint64_t out[4]);
/* Output t (0-based) of sitmo::prng_engine(seed). */
uint32_t or_sitmo_output(uint32_t seed, uint64_t t);
/* rmat_edge_generator(2^scale, a, b, c, d, seed) + rmat_fill
 * (rmat_generator.h:70-193) run serially: edges in generation order after
 * the self-loop re-roll.  Returns 0, -1 if re-rolls never end. */
int or_rmat_stream_edges(int scale, int64_t num_edges, double a, double b, double c,
                         double d, uint32_t seed, int64_t *src, int64_t *dst);

/* The project's grid generator (vertex r*cols+c, 4-neighbour edges, each
 * deleted with probability delete_frac by a seeded Philox draw). */
int64_t or_grid_edges(int64_t rows, int64_t cols, double delete_frac, uint64_t seed,
                      int64_t *src, int64_t *dst);

#ifdef __cplusplus
}
#endif
#endif
