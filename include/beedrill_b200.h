/* beedrill_b200.h -- C ABI of the B200 direction-optimizing BFS.
 *
 * This is the drop-in boundary for Beedrill's `hybrid_bfs` class
 * (hybrid_bfs.h:11-47) and the graph/edge-list layer it sits on
 * (graph_base.h, dist_edge_list.h, edge_list.h).  Plain C types only: host
 * pointers and sizes in, status codes out.  Every entry point returns
 * BD_OK (0) or a negative bd_status; none of them calls exit() or traps.
 *
 * Ownership: handles are opaque.  Device memory allocated by the library is
 * released only by the matching *_destroy call.  A handle is not thread
 * safe; use one host thread per handle.  Each bd_bfs owns a CUDA stream.
 *
 * Reference interface -> entry point:
 *   dist_edge_list::load_binary (dist_edge_list.cc:50-143)
 *     + create_graph_from_edge_list (graph_base.h:335-436)  -> bd_graph_from_el64
 *   create_graph_from_edge_list on in-memory edges          -> bd_graph_from_edges
 *   graph::check (graph_base.h:110-134)                     -> bd_graph_check
 *   generator/rmat_dataset_dump.cc (seeded, on the device)  -> bd_graph_rmat
 *   rmat_edge_generator + rmat_fill (rmat_generator.h:70-193)
 *     + rmat_dataset_dump.cc:48-53, the reference's stream  -> bd_graph_rmat_stream
 *   pick_random_vertex + lcg (hybrid_bfs_main.cc:136-144)   -> bd_graph_pick_roots
 *   hybrid_bfs::hybrid_bfs(graph&) (hybrid_bfs.cc:10-18)    -> bd_bfs_create
 *   hybrid_bfs::clear (hybrid_bfs.cc:433-443)               -> bd_bfs_clear
 *   hybrid_bfs::run_beamer (hybrid_bfs.cc:152-191)          -> bd_bfs_run_beamer
 *   run_with_migrating_threads / run_with_remote_writes
 *     (hybrid_bfs.cc:196-235)                               -> bd_bfs_run_top_down
 *   run_with_remote_writes_hybrid (hybrid_bfs.cc:243-277)   -> bd_bfs_run_beamer
 *   hybrid_bfs::check (hybrid_bfs.cc:281-379)               -> bd_bfs_check,
 *                                                              bd_graph_check_parents
 *   hybrid_bfs::count_num_traversed_edges (:401-414)        -> bd_bfs_count_traversed_edges
 *   hybrid_bfs::print_tree (hybrid_bfs.cc:381-399)          -> bd_bfs_get_parents (+ host printing)
 *   components::components(graph&) (components.cc:13-22)   -> bd_components_create
 *   components::run (components.cc:38-118)                  -> bd_components_run
 *   components::component_, component_size_ (components.h:13-15)
 *                                                           -> bd_components_get_labels, _get_sizes
 *   components::check (components.cc:155-200)               -> bd_components_check,
 *                                                              bd_graph_check_components
 */
#ifndef BEEDRILL_B200_H
#define BEEDRILL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int bd_status;
#define BD_OK 0
#define BD_ERR_INVALID (-1)    /* bad argument (null pointer, bad size, bad enum)    */
#define BD_ERR_IO (-2)         /* file cannot be opened / read / written              */
#define BD_ERR_FORMAT (-3)     /* el64 header or body rejected (edge_list.cc rules)  */
#define BD_ERR_OOM (-4)        /* host or device allocation failed                    */
#define BD_ERR_CUDA (-5)       /* a CUDA runtime call failed                          */
#define BD_ERR_TIMEOUT (-6)    /* a bounded device-side wait ran out                  */
#define BD_ERR_RANGE (-7)      /* vertex id out of range (hybrid_bfs.cc:155 assert)   */
#define BD_ERR_STATE (-8)      /* call out of order (e.g. results before a run)       */
#define BD_ERR_NODEV (-9)      /* no usable CUDA device (sm_100 required)             */
#define BD_ERR_LIMIT (-10)     /* size beyond a documented limit                      */

typedef struct bd_graph bd_graph;
typedef struct bd_bfs bd_bfs;

/* Adjacency order inside each vertex's neighbour list. */
#define BD_ORDER_INSERTION 0 /* reference order: file order, (s->d) then (d->s) */
#define BD_ORDER_SORTED 1    /* ascending neighbour id                          */
#define BD_ORDER_DEGREE 2    /* highest-degree neighbour first (ties: insertion
                                order); bottom-up scans meet visited hubs first */
#define BD_ORDER_HUB 3       /* BD_ORDER_DEGREE, and the traversal kernels run on
                                a second CSR whose vertices are renumbered by
                                degree, highest first (ties: id): the state of
                                the hubs most arcs lead to is packed into a few
                                cache lines.  Every call still takes and returns
                                the caller's vertex ids; the CSR the graph calls
                                expose is the BD_ORDER_DEGREE one.  No
                                counterpart in the reference. */

/* Direction policies (the reference's --algorithm values map onto these). */
#define BD_ALG_BEAMER 0    /* beamer_hybrid, remote_writes_hybrid                */
#define BD_ALG_TOP_DOWN 1  /* migrating_threads, remote_writes, top_down         */
#define BD_ALG_BOTTOM_UP 2 /* bottom_up                                          */
#define BD_ALG_LEARNED 3   /* MLP direction policy, Beamer as the fallback       */

#define BD_DIR_TOP_DOWN 0
#define BD_DIR_BOTTOM_UP 1

typedef struct bd_bfs_opts {
    int32_t alg;          /* BD_ALG_*                                            */
    int32_t min_parent;   /* 1: parent(v) = smallest neighbour one level up      */
    int64_t alpha;        /* Beamer alpha (hybrid_bfs_main.cc:74), must be > 0   */
    int64_t beta;         /* Beamer beta (hybrid_bfs_main.cc:75), must be > 0    */
    int32_t block_size;   /* threads per CTA; 0 = tuned default                  */
    int32_t large_degree; /* top-down CTA-split threshold; 0 = tuned default     */
    int32_t chunk_edges;  /* edges per split work unit; 0 = tuned default        */
    int32_t bu_prefix;    /* bottom-up per-thread scan before warp scan; 0 = def */
    int64_t spin_limit;   /* grid-barrier wait bound in polls; 0 = default (~2 s) */
    int32_t test_extra_ctas; /* TEST ONLY: barrier expects this many extra CTAs,
                                so it can never complete and must time out      */
    int32_t bu_words;     /* bottom-up: bitmap words in flight per warp: 1, 2, 4
                             (the warp shares each word), 32 (each lane owns a
                             word); 0 = tuned default                             */
    int32_t bu_sparse_words; /* the same once fewer than half of the vertices
                                of nonzero degree are unvisited; 0 = default.
                                Pairs available: equal to bu_words, or
                                (2 or 4, 32)                                     */
    int32_t reserved;
} bd_bfs_opts;

/* One BFS step as recorded on the device. */
typedef struct bd_step {
    int32_t dir;          /* BD_DIR_*                                             */
    int32_t level;        /* depth of the frontier this step expanded             */
    int64_t frontier;     /* vertices in that frontier                            */
    int64_t frontier_edges; /* sum of their degrees (m_f)                         */
    int64_t unexplored_edges; /* 2m - degree sum of all visited vertices (m_u)    */
    int64_t found;        /* vertices discovered by the step                      */
    int64_t ns;           /* device time of the step (ns, %globaltimer)           */
} bd_step;

typedef struct bd_run_stats {
    double ms;            /* CUDA-event time of the traversal kernel(s)           */
    int64_t num_steps;    /* steps taken (the last one discovers nothing)         */
    int64_t reached;      /* vertices reached, source included (n_c)              */
    int64_t traversed_edges; /* count_num_traversed_edges(): m_c                  */
    int64_t top_down_steps;
    int64_t bottom_up_steps;
} bd_run_stats;

/* ---- library ------------------------------------------------------------- */
const char *bd_status_string(bd_status s);
const char *bd_version(void);
/* Select the CUDA device used by handles created afterwards (default 0). */
bd_status bd_set_device(int device);

/* ---- graphs --------------------------------------------------------------- */
bd_status bd_graph_from_el64(const char *path, int32_t adjacency_order, bd_graph **out);
bd_status bd_graph_from_edges(int64_t num_vertices, int64_t num_edges, const int64_t *src,
                              const int64_t *dst, int32_t adjacency_order, bd_graph **out);
bd_status bd_graph_from_csr(int64_t num_vertices, int64_t num_arcs, const int64_t *offsets,
                            const uint32_t *adjacency, bd_graph **out);
/* Seeded RMAT graph built on the device: edge_factor << scale generated
 * edges, self loops re-rolled, flipped, sorted, deduplicated, vertex ids
 * permuted and edge order shuffled by `seed`. */
bd_status bd_graph_rmat(int32_t scale, int64_t edge_factor, double a, double b, double c,
                        double d, uint64_t seed, int32_t adjacency_order, bd_graph **out);
/* RMAT edges drawn exactly as the reference's generator draws them
 * (generator/rmat_generator.h:70-193 with rmat_edge_generator(.., seed =
 * stream_seed)): the sitmo::prng_engine stream (generator/prng_engine.hpp)
 * through libstdc++'s uniform_real_distribution<double>, edge i from stream
 * position i x 2 x (5 (scale-1) + 1), self loops re-rolled serially from the
 * stream's tail in edge order, as rmat_fill does; then flipped, sorted and
 * deduplicated (rmat_dataset_dump.cc:48-53).  edge_factor << scale edges.
 * permute = 0: the graph keeps the generator's vertex ids and the sorted
 * edge order -- the reference's edge list before its thread-count-dependent
 * relabel and shuffle (rmat_dataset_dump.cc:55-57); permute = 1: the seeded
 * relabel and shuffle of bd_graph_rmat (keyed by permute_seed) follow. */
bd_status bd_graph_rmat_stream(int32_t scale, int64_t edge_factor, double a, double b, double c,
                               double d, uint32_t stream_seed, int32_t permute,
                               uint64_t permute_seed, int32_t adjacency_order, bd_graph **out);
/* rows x cols grid, vertex r*cols+c, 4-neighbour edges (horizontal edges
 * first, row by row, then vertical), each deleted independently with
 * probability delete_frac by a seeded Philox draw.  The high-diameter
 * contrast graph of the evaluation (no counterpart in the reference). */
bd_status bd_graph_grid(int64_t rows, int64_t cols, double delete_frac, uint64_t seed,
                        int32_t adjacency_order, bd_graph **out);
/* Disjoint union of graphs: vertex ids of graph i are shifted by the vertex
 * count of graphs 0..i-1.  vertex_base (host, count+1 entries) receives the
 * shifts; may be NULL. */
bd_status bd_graph_concat(bd_graph *const *graphs, int64_t count, bd_graph **out,
                          int64_t *vertex_base);
bd_status bd_graph_info(const bd_graph *g, int64_t *num_vertices, int64_t *num_edges);
/* Copy the CSR to host buffers of n+1 and 2m entries. */
bd_status bd_graph_copy_csr(const bd_graph *g, int64_t *offsets, uint32_t *adjacency);
/* Edge list (generated / loaded order); only for graphs built from edges. */
bd_status bd_graph_copy_edges(const bd_graph *g, int64_t *src, int64_t *dst);
bd_status bd_graph_write_el64(const bd_graph *g, const char *path);
/* graph::check: every edge present in both lists, no adjacent duplicates.
 * ok receives 1 (pass) or 0. */
bd_status bd_graph_check(const bd_graph *g, int32_t *ok);
/* hybrid_bfs::check (hybrid_bfs.cc:281-379) of a caller's parent array
 * (host, n entries, the reference's encoding: the source is its own parent,
 * unreached vertices negative), run on the device against depths from an
 * independent device BFS from source.  ok receives 1 (pass) or 0;
 * bad_vertex (may be NULL) receives the lowest failing vertex -- the one
 * the reference's loop stops at -- or -1. */
bd_status bd_graph_check_parents(const bd_graph *g, int64_t source, const int64_t *parent,
                                 int32_t *ok, int64_t *bad_vertex);
/* Roots as hybrid_bfs_main.cc:136-144 with lcg(seed). */
bd_status bd_graph_pick_roots(const bd_graph *g, uint64_t seed, int64_t k, int64_t *roots);
/* Device pointers of the CSR (borrowed, valid until bd_graph_destroy). */
bd_status bd_graph_device_csr(const bd_graph *g, const int64_t **offsets,
                              const uint32_t **adjacency);
bd_status bd_graph_destroy(bd_graph *g);

/* ---- BFS ------------------------------------------------------------------ */
void bd_bfs_default_opts(bd_bfs_opts *opts);
bd_status bd_bfs_create(bd_graph *g, const bd_bfs_opts *opts, bd_bfs **out);
bd_status bd_bfs_clear(bd_bfs *b);
/* Run with the handle's policy (opts.alg).  stats may be NULL. */
bd_status bd_bfs_run(bd_bfs *b, int64_t source, bd_run_stats *stats);
bd_status bd_bfs_run_beamer(bd_bfs *b, int64_t source, int64_t alpha, int64_t beta,
                            bd_run_stats *stats);
bd_status bd_bfs_run_top_down(bd_bfs *b, int64_t source, bd_run_stats *stats);
bd_status bd_bfs_run_bottom_up(bd_bfs *b, int64_t source, bd_run_stats *stats);
/* Several sources expanded as one BFS (level 0 = all sources).  On a graph
 * made by bd_graph_concat with one source per part, each part gets its own
 * BFS tree and depths. */
bd_status bd_bfs_run_multi(bd_bfs *b, const int64_t *sources, int64_t count,
                           bd_run_stats *stats);
/* k single-source BFSs, one after another, with clear() before each (the
 * trial loop of hybrid_bfs_main.cc:252-302).  ms_out[i], edges_out[i] and
 * reached_out[i] (each may be NULL) get root i's run time, m_c and n_c.
 * e2e_ms (may be NULL) gets the device time of the whole call, from the
 * copy of the roots to the device to the copy of the results back. */
bd_status bd_bfs_run_many(bd_bfs *b, const int64_t *sources, int64_t k, double *ms_out,
                          int64_t *edges_out, int64_t *reached_out, double *e2e_ms);
/* bd_bfs_run_many, and root i's results end in d_depth[i * n ...] (int32,
 * -1 unreached) and d_parent[i * n ...] (int64, caller ids, the reference's
 * encoding), device arrays of k x n entries, written inside each root's
 * timed region: the trial loop with every trial's parent_ kept
 * (hybrid_bfs_main.cc:252-302). */
bd_status bd_bfs_run_many_into(bd_bfs *b, const int64_t *sources, int64_t k, int32_t *d_depth,
                               int64_t *d_parent, double *ms_out, int64_t *edges_out,
                               int64_t *reached_out, double *e2e_ms);
bd_status bd_bfs_get_depths(bd_bfs *b, int32_t *depth);
bd_status bd_bfs_get_parents(bd_bfs *b, int64_t *parent);
bd_status bd_bfs_device_ptrs(bd_bfs *b, const int32_t **depth, const int64_t **parent);
bd_status bd_bfs_count_traversed_edges(bd_bfs *b, int64_t *out);
bd_status bd_bfs_check(bd_bfs *b, int64_t source, int32_t *ok);
/* Per-step records of the last run (count <= capacity copied). */
bd_status bd_bfs_get_steps(bd_bfs *b, bd_step *steps, int64_t capacity, int64_t *count);
bd_status bd_bfs_destroy(bd_bfs *b);

/* Allocation-free BFS.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory on this call path: a
 * process whose device memory is reserved up front by its own pool allocator
 * (a cudaMalloc there fails or fragments the pool), or code that cannot
 * afford the device-wide synchronisation cudaMalloc / cudaFree may cause.
 * One Beamer BFS (alpha, beta) from `source` over a CSR already in device
 * memory (d_offsets: num_vertices+1 int64, d_adjacency: num_arcs uint32);
 * writes d_depth (int32, -1 unreached) and d_parent (reference encoding)
 * in caller-owned device memory, on `stream` (a cudaStream_t, NULL for the
 * default stream), and returns after the stream has finished.
 * traversed_edges (host, may be NULL) gets count_num_traversed_edges().
 *
 * All temporaries live in one fixed device array inside the library (about
 * 7.2 MB on every GPU that loads it, held until the process exits), so:
 *   - num_vertices must not exceed BD_NOALLOC_MAX_VERTICES (else
 *     BD_ERR_LIMIT, nothing launched);
 *   - the first call on a device looks the array's device address up on
 *     that device (cudaGetSymbolAddress) and keeps it for the life of the
 *     process: after a cudaDeviceReset of that device the kept address is
 *     stale, so do not call this entry point again in that process;
 *   - every call waits for `stream` twice (it reads two counters back), so
 *     no call may be made while a stream capture is under way;
 *   - every call shares the array: calls that overlap on the GPU (other
 *     streams, other host threads) race and corrupt each other.  Serialise
 *     them.
 * Launch parameters are the regular handle's defaults (bd_bfs_create),
 * except that on graphs of more than 4,194,304 arcs the large-degree
 * threshold rises above 32 (to num_arcs / 131072 + 1) so that its queue fits
 * the array.  Nothing is allocated or freed; the call uses the device
 * current on the calling thread. */
#define BD_NOALLOC_MAX_VERTICES 524288
bd_status bd_bfs_run_noalloc(const int64_t *d_offsets, const uint32_t *d_adjacency,
                             int64_t num_vertices, int64_t num_arcs, int64_t source,
                             int64_t alpha, int64_t beta, int32_t *d_depth, int64_t *d_parent,
                             void *stream, int64_t *traversed_edges);

/* ---- batched traversal ---------------------------------------------------- */
/* Many BFSs share each pass over the graph: roots are processed in groups of
 * up to 64, one bit lane of a uint64 per root (multi-source BFS), one
 * persistent launch per group; all groups of a call are replayed as one
 * captured CUDA graph.  Per root the results equal a single-source BFS from
 * that root (depths bit-exact, parents one level up, m_c).  No counterpart
 * class in the reference, whose driver loops over roots one at a time
 * (hybrid_bfs_main.cc:252-302); per-root results are read with the same
 * encodings as bd_bfs_get_depths / bd_bfs_get_parents. */
typedef struct bd_msbfs bd_msbfs;
typedef struct bd_msbfs_opts {
    int64_t alpha;         /* pull when frontier edges * alpha > edges left; > 0 */
    int32_t force_dir;     /* -1: rule; 0: push only; 1: pull only              */
    int32_t block_size;    /* 0 = default (512)                                 */
    int32_t large_degree;  /* push: degree at which a vertex is split; 0 = def  */
    int32_t chunk_edges;   /* push: edges per split work unit; 0 = default      */
    int32_t pull_prefix;   /* pull: arcs a lane scans alone; 0 = default        */
    int32_t use_graph;     /* 1 (default via bd_msbfs_default_opts): replay the
                              groups of a call as one captured CUDA graph       */
    int64_t spin_limit;    /* grid-barrier poll bound; 0 = default (~2 s)       */
    int32_t heavy_degree;  /* pull: lists longer than this are cut into chunks
                              shared by all warps; 0 = default (4096)           */
    int32_t heavy_chunk;   /* arcs per such chunk; 0 = default (2048)           */
    int32_t materialize;   /* 1: every run ends with each root's int32 depths
                              and int64 parents (caller ids, the reference's
                              encoding) in device memory owned by the handle,
                              as run_beamer leaves parent_ complete
                              (hybrid_bfs.cc:152-191); the run's time covers
                              it.  Costs 12 bytes x n x max_roots of device
                              memory.  0: results are extracted when read   */
    int32_t min_parent;    /* 1 (implies materialize): each root's parent(v) is
                              the smallest neighbour one level up, as
                              bd_bfs_opts.min_parent -- bit-exact trees        */
} bd_msbfs_opts;
void bd_msbfs_default_opts(bd_msbfs_opts *opts);
/* max_roots: capacity of one call (results of all roots stay readable). */
bd_status bd_msbfs_create(bd_graph *g, int32_t max_roots, const bd_msbfs_opts *opts,
                          bd_msbfs **out);
/* BFS from each of sources[0..count); stats (may be NULL): ms = device time
 * of all groups, traversed_edges = sum of m_c, reached = sum of n_c. */
bd_status bd_msbfs_run(bd_msbfs *b, const int64_t *sources, int32_t count, bd_run_stats *stats);
bd_status bd_msbfs_get_depths(bd_msbfs *b, int32_t root_index, int32_t *depth);
bd_status bd_msbfs_get_parents(bd_msbfs *b, int32_t root_index, int64_t *parent);
/* count_num_traversed_edges() (m_c) and reached vertices (n_c) of one root. */
bd_status bd_msbfs_count_traversed_edges(bd_msbfs *b, int32_t root_index, int64_t *edges,
                                         int64_t *reached);
/* hybrid_bfs::check (hybrid_bfs.cc:281-379) of one root's parents. */
bd_status bd_msbfs_check(bd_msbfs *b, int32_t root_index, int32_t *ok);
/* Borrowed device pointers (n entries each, valid until the next run or
 * destroy) to one root's materialized depths and parents; BD_ERR_STATE
 * unless the handle was made with opts.materialize.  Counterpart of
 * bd_bfs_device_ptrs: the reference's parent_ (hybrid_bfs.h:43) per root. */
bd_status bd_msbfs_device_results(bd_msbfs *b, int32_t root_index, const int32_t **depth,
                                  const int64_t **parent);
/* Step records of the last group of the last call (found = new lanes). */
bd_status bd_msbfs_get_steps(bd_msbfs *b, bd_step *steps, int64_t capacity, int64_t *count);
/* Installs (params != NULL) or removes the learned push/pull policy of the
 * batched traversal (same network layout and features as bd_bfs_set_policy;
 * unexplored degree sum = degree sum of vertices some lane has not reached). */
bd_status bd_msbfs_set_policy(bd_msbfs *b, const float *params, const float *mean,
                              const float *inv_std, const float *lo, const float *hi,
                              float margin);
bd_status bd_msbfs_destroy(bd_msbfs *b);

/* ---- connected components ------------------------------------------------- */
/* Labels every vertex with the smallest vertex id of its component -- the
 * labelling the reference's label propagation converges to, so labels,
 * sizes and the component count equal the reference's exactly.  One pass
 * over the arcs builds a union-find forest on the device (num_iters = 1;
 * the reference counts its label-propagation passes).  On a CSR that does
 * not hold every edge in both directions the components are those of the
 * undirected graph its arcs form; check() follows arcs as stored, like the
 * reference's, so it is meaningful for symmetric graphs only. */
typedef struct bd_components bd_components;
typedef struct bd_components_stats {
    int64_t num_components; /* isolated vertices count as one component each */
    int64_t num_iters;      /* passes over the arcs */
    double ms;              /* device time of run() */
} bd_components_stats;
bd_status bd_components_create(bd_graph *g, bd_components **out);
/* components::clear is empty in the reference; run() starts over. */
bd_status bd_components_clear(bd_components *cc);
bd_status bd_components_run(bd_components *cc, bd_components_stats *stats);
/* component_ / component_size_ (host int64[n]; size is indexed by label,
 * 0 for ids that label nothing). */
bd_status bd_components_get_labels(bd_components *cc, int64_t *component);
bd_status bd_components_get_sizes(bd_components *cc, int64_t *component_size);
/* Labels in device memory (borrowed, valid until the next run or destroy). */
bd_status bd_components_device_labels(bd_components *cc, const int64_t **component);
/* components::check of the last run's labels, on the device. */
bd_status bd_components_check(bd_components *cc, int32_t *ok);
bd_status bd_components_destroy(bd_components *cc);
/* components::check (components.cc:155-200) of any labelling (host int64[n]):
 * passes when every edge joins two vertices of one label and no label spans
 * two components.  bad_vertex (may be NULL) receives the lowest vertex that
 * breaks the rule (an edge to another label, or not reached from its
 * label's representative), or -1. */
bd_status bd_graph_check_components(const bd_graph *g, const int64_t *component, int32_t *ok,
                                    int64_t *bad_vertex);

/* ---- learned direction policy -------------------------------------------- */
/* An fp32 MLP 8 -> 32 (ReLU) -> 32 (ReLU) -> 2 that picks the direction of
 * every step in place of the alpha/beta rule (hybrid_bfs.cc:166-188).
 * Parameter vector, BD_POLICY_PARAMS floats:
 *   w1[32][8], b1[32], w2[32][32], b2[32], w3[2][32], b3[2].
 * Features per step (raw, before standardisation with mean / inv_std), with
 * L(x) = log2(1 + x), all free of the graph's size:
 *   L(m_f) - L(m_u)            frontier degree sum vs unexplored degree sum
 *   L(frontier) - L(n)         frontier vertices vs vertices
 *   L(m_u) - L(2m)             unexplored degree sum vs arcs
 *   L(level)
 *   L(m) - L(n)                average degree
 *   previous direction (0 top-down, 1 bottom-up)
 *   L(previous step us) - L(m / 2^20)
 *   L(m_f) - L(frontier)       frontier average degree
 * Output: logits (top-down, bottom-up).  The Beamer rule decides whenever
 * |logit gap| < margin, whenever a feature lies outside [lo, hi] -- the
 * kernels test feature 0 first and run the network only inside its range
 * (the band where the policy may overrule the rule) -- and always when no
 * policy is installed. */
#define BD_POLICY_PARAMS 1410
#define BD_POLICY_FEATURES 8
/* Installs (or, with params == NULL or margin == +inf, removes) the policy
 * used by BD_ALG_LEARNED.  lo / hi (8 floats each, may be NULL for no limit)
 * bound the raw features the policy is trusted on; outside them the Beamer
 * rule decides.  Host pointers; copied. */
bd_status bd_bfs_set_policy(bd_bfs *b, const float *params, const float *mean,
                            const float *inv_std, const float *lo, const float *hi,
                            float margin);
/* Device forward pass over n standardised feature rows (host buffers). */
bd_status bd_policy_forward(const float *params, const float *x, int64_t n, float *logits);
/* Weighted cross-entropy sum_i w_i CE(x_i, label_i) / sum_i w_i and its
 * gradient (BD_POLICY_PARAMS floats), computed by the device kernels. */
bd_status bd_policy_loss_grad(const float *params, const float *x, const int32_t *label,
                              const float *weight, int64_t n, float *loss, float *grad);
/* Full-batch Adam (beta1 0.9, beta2 0.999, eps 1e-8, L2 weight_decay) for
 * `epochs` steps on the device; params is updated in place; loss_history
 * (may be NULL) gets the loss before each step. */
bd_status bd_policy_train(float *params, const float *x, const int32_t *label,
                          const float *weight, int64_t n, int32_t epochs, float lr,
                          float weight_decay, float *loss_history);

#ifdef __cplusplus
}
#endif
#endif
