// bd_internal.h -- shared definitions of the B200 BFS library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "beedrill_b200.h"

namespace bd {

// Records the failing CUDA call for bd_status_string-style diagnostics and
// returns BD_ERR_CUDA.
bd_status cuda_fail(cudaError_t err, const char *what, const char *file, int line);
// Library-wide device selection (bd_set_device).
int current_device();
// Checks that the selected device is usable (sm_100) and makes it current.
bd_status ensure_device();

}  // namespace bd

#define BD_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t bd_e_ = (call);                                          \
        if (bd_e_ != cudaSuccess) {                                          \
            return bd::cuda_fail(bd_e_, #call, __FILE__, __LINE__);          \
        }                                                                    \
    } while (0)

#define BD_TRY(expr)                                                         \
    do {                                                                     \
        bd_status bd_s_ = (expr);                                            \
        if (bd_s_ != BD_OK) { return bd_s_; }                                \
    } while (0)

// A graph resident in HBM: CSR with int64 offsets and uint32 neighbour ids,
// plus a bitmap with one bit per vertex of degree zero (padding bits past n
// are set too, so bit scans can treat them as already finished).
struct bd_graph {
    int device = 0;
    int64_t n = 0;          // vertices
    int64_t m = 0;          // undirected edges (arcs / 2)
    int64_t arcs = 0;       // entries of the adjacency array
    int64_t n_live = 0;     // vertices of nonzero degree
    int32_t order = BD_ORDER_INSERTION;
    // Every arc u->v has its reverse v->u (graphs built from edge lists, and
    // unions of them); not assumed for a caller's CSR.
    bool symmetric = false;
    int64_t *d_off = nullptr;     // [n + 1]
    uint32_t *d_adj = nullptr;    // [arcs]
    uint32_t *d_isolated = nullptr;  // [words(n)]
    // Edge list in file / generation order, kept for el64 export and check.
    int64_t *d_src = nullptr;     // [m] or null
    int64_t *d_dst = nullptr;     // [m] or null
    // BD_ORDER_HUB: the traversal CSR, vertices renumbered by degree
    // (highest first), its isolated bitmap, and the two numberings.
    // Null for the other orders: the traversal kernels use d_off / d_adj.
    int64_t *d_toff = nullptr;      // [n + 1]
    uint32_t *d_tadj = nullptr;     // [arcs]
    uint32_t *d_tisolated = nullptr;  // [words(n)]
    uint32_t *d_perm = nullptr;     // [n] caller id -> traversal id
    uint32_t *d_iperm = nullptr;    // [n] traversal id -> caller id
};

namespace bd {

inline int64_t bitmap_words(int64_t n) { return (n + 31) / 32; }

// The CSR the traversal kernels run on.
inline const int64_t *traversal_off(const bd_graph *g) { return g->d_toff ? g->d_toff : g->d_off; }
inline const uint32_t *traversal_adj(const bd_graph *g) { return g->d_tadj ? g->d_tadj : g->d_adj; }
inline const uint32_t *traversal_isolated(const bd_graph *g)
{
    return g->d_tisolated ? g->d_tisolated : g->d_isolated;
}

// Builds the CSR of an edge list that is already on the device (src/dst
// int64[m]); takes ownership of d_src/d_dst.
bd_status graph_from_device_edges(int64_t n, int64_t m, int64_t *d_src, int64_t *d_dst,
                                  int32_t order, bd_graph **out);
struct PolicyBlob;
// Host-side PolicyBlob from the ABI's arrays (bd_policy.cu).
bd_status policy_blob(const float *params, const float *mean, const float *inv_std,
                      const float *lo, const float *hi, float margin, PolicyBlob *blob);
// hybrid_bfs::check on the device (bd_check.cu) for a parent array in
// device memory, in the reference's encoding and the caller's vertex ids;
// *ok = 1 when it passes, *bad_vertex (may be null) gets the lowest failing
// vertex or -1.
bd_status check_parents_device(const bd_graph *g, int64_t source, const int64_t *d_parent,
                               int32_t *ok, int64_t *bad_vertex);
// components::check on the device (bd_check.cu) for labels in device
// memory (int64[n]); *ok = 1 when it passes, *bad_vertex (may be null) gets
// the lowest vertex that is unreached from its label's representative or
// has an arc to another label, or -1.
bd_status check_components_device(const bd_graph *g, const int64_t *d_label, int32_t *ok,
                                  int64_t *bad_vertex);
// The deterministic parent tree (bd_bfs.cu): for every vertex of depth
// d > 0, the smallest neighbour of depth d - 1 in the CSR (off, adj), written
// to parent; other entries are left as they are.  Queued on s.
cudaError_t launch_min_parent(const int64_t *off, const uint32_t *adj, int64_t n,
                              const int32_t *depth, int64_t *parent, cudaStream_t s);
// BD_ORDER_HUB: builds the renumbered traversal CSR of a finished graph.
bd_status graph_build_hub(bd_graph *g, cudaStream_t s);
// Fills d_isolated from d_off.
bd_status graph_finish(bd_graph *g, cudaStream_t s);
void graph_free(bd_graph *g);

}  // namespace bd
