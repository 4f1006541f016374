// bd_check.cu -- hybrid_bfs::check (hybrid_bfs.cc:281-379) on the device.
//
// The reference validates a parent array against the depths of its own
// serial queue BFS: a vertex that both reached must have its parent among
// its neighbours exactly one level up (the source is its own parent at
// depth 0), and the two must agree on which vertices were reached.  The
// verdict depends only on the BFS depths, which do not depend on the order
// of the search, so a parallel search gives the same verdict:
//
//   check_level_kernel   one launch per level: a vertex queue, one warp per
//                        queued vertex, depth claims by atomicCAS.  It shares
//                        no code with the traversal kernels, so it is an
//                        independent witness of the depths they claim.
//   check_verify_kernel  one warp per vertex, all vertices at once: the
//                        reference's per-vertex test.  A failing vertex
//                        lowers a shared minimum, so the lowest failing
//                        vertex -- the one the reference's ascending loop
//                        stops at and logs -- is reported.
//
// Device memory: 12 bytes per vertex (depths and two queues) for the call.
//
// components::check (components.cc:155-200) runs a serial BFS from one
// vertex of each distinct label, requires every neighbour it meets to carry
// that label, and requires every vertex to be visited.  That verdict is:
// every arc joins two vertices of the same label, and each component holds
// the representative of its label (so no label spans two components).
// Here the representatives come from a radix sort of (label, vertex); a
// multi-source run of check_level_kernel from all of them marks what they
// reach; check_components_kernel tests both conditions for every vertex.
// Device memory: 36 bytes per vertex plus the sort's scratch.
#include <cub/cub.cuh>

#include <climits>

#include "bd_internal.h"

namespace bd {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

int grid_for_warps(int64_t warps)
{
    int64_t b = (warps + kWarps - 1) / kWarps;
    if (b < 1) { b = 1; }
    if (b > 148 * 64) { b = 148 * 64; }  // warp-stride beyond this
    return (int)b;
}

__global__ void __launch_bounds__(kThreads) check_level_kernel(
    const int64_t *off, const uint32_t *adj, const uint32_t *q, int64_t len, int32_t next_depth,
    int32_t *depth, uint32_t *q_next, unsigned long long *next_len)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * kWarps;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; i < len; i += warps) {
        const uint32_t u = q[i];
        const int64_t e = off[u + 1];
        for (int64_t k = off[u] + lane; k < e; k += 32) {
            const uint32_t v = adj[k];
            // Each vertex is claimed once over the whole search, so the
            // queues never hold more than n entries.
            if (__ldcg(&depth[v]) == -1 && atomicCAS(&depth[v], -1, next_depth) == -1) {
                q_next[atomicAdd(next_len, 1ull)] = v;
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) check_verify_kernel(
    const int64_t *off, const uint32_t *adj, int64_t n, int64_t source, const int32_t *depth,
    const int64_t *parent, unsigned long long *first_bad)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * kWarps;
    // Every branch below is uniform across the warp: all lanes test vertex u.
    for (int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; u < n; u += warps) {
        const int32_t d = depth[u];
        const int64_t p = parent[u];
        bool bad;
        if (d >= 0 && p >= 0) {
            if (u == source) {
                bad = !(p == u && d == 0);
            } else {
                // The first occurrence of p in u's list decides
                // (hybrid_bfs.cc:343-355); p < n there, since it equals an
                // adjacency entry.
                const int64_t e = off[u + 1];
                bool found = false, good = false;
                for (int64_t k0 = off[u]; k0 < e && !found; k0 += 32) {
                    const int64_t k = k0 + lane;
                    const unsigned hit = __ballot_sync(0xffffffffu, k < e && (int64_t)adj[k] == p);
                    if (hit) {
                        found = true;
                        good = depth[adj[k0 + __ffs(hit) - 1]] == d - 1;
                    }
                }
                bad = !good;
            }
        } else {
            bad = (d < 0) != (p < 0);
        }
        if (bad && lane == 0) { atomicMin(first_bad, (unsigned long long)u); }
    }
}

__global__ void iota_kernel(uint32_t *v, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        v[i] = (uint32_t)i;
    }
}

// The first vertex of each run of equal labels in sorted order becomes a
// source: depth 0, queued.
__global__ void label_sources_kernel(const int64_t *sorted_label, const uint32_t *sorted_vertex,
                                     int64_t n, int32_t *depth, uint32_t *q,
                                     unsigned long long *len)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i == 0 || sorted_label[i] != sorted_label[i - 1]) {
            const uint32_t v = sorted_vertex[i];
            depth[v] = 0;
            q[atomicAdd(len, 1ull)] = v;
        }
    }
}

__global__ void __launch_bounds__(kThreads) check_components_kernel(
    const int64_t *off, const uint32_t *adj, int64_t n, const int32_t *depth,
    const int64_t *label, unsigned long long *first_bad)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * kWarps;
    for (int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; u < n; u += warps) {
        bool bad = depth[u] < 0;
        const int64_t mine = label[u], e = off[u + 1];
        for (int64_t k0 = off[u]; k0 < e && !bad; k0 += 32) {
            const int64_t k = k0 + lane;
            bad = __any_sync(0xffffffffu, k < e && label[adj[k]] != mine);
        }
        if (bad && lane == 0) { atomicMin(first_bad, (unsigned long long)u); }
    }
}

int grid_for(int64_t items)
{
    int64_t b = (items + kThreads - 1) / kThreads;
    if (b < 1) { b = 1; }
    if (b > 148 * 64) { b = 148 * 64; }
    return (int)b;
}

// Depths by level-synchronous search from the len sources already queued
// in q[0] (depth 0 there, -1 elsewhere).
cudaError_t search_levels(const bd_graph *g, int32_t *depth, uint32_t *q[2],
                          unsigned long long *cnt, unsigned long long len)
{
    int cur = 0;
    for (int32_t level = 0; len > 0; ++level, cur ^= 1) {
        cudaError_t e = cudaMemset(cnt, 0, sizeof(unsigned long long));
        if (e != cudaSuccess) { return e; }
        check_level_kernel<<<grid_for_warps((int64_t)len), kThreads>>>(
            g->d_off, g->d_adj, q[cur], (int64_t)len, level + 1, depth, q[cur ^ 1], cnt);
        e = cudaGetLastError();
        if (e == cudaSuccess) { e = cudaMemcpy(&len, cnt, sizeof(len), cudaMemcpyDeviceToHost); }
        if (e != cudaSuccess) { return e; }
    }
    return cudaSuccess;
}

}  // namespace

bd_status check_parents_device(const bd_graph *g, int64_t source, const int64_t *d_parent,
                               int32_t *ok, int64_t *bad_vertex)
{
    const int64_t n = g->n;
    if (source < 0 || source >= n) { return BD_ERR_RANGE; }
    BD_CUDA(cudaSetDevice(g->device));
    int32_t *depth = nullptr;
    uint32_t *q[2] = {nullptr, nullptr};
    unsigned long long *cnt = nullptr;  // [0] next queue length, [1] lowest failing vertex
    auto release = [&]() {
        cudaFree(depth);
        cudaFree(q[0]);
        cudaFree(q[1]);
        cudaFree(cnt);
    };
    if (cudaMalloc(&depth, sizeof(int32_t) * n) != cudaSuccess ||
        cudaMalloc(&q[0], sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&q[1], sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&cnt, sizeof(unsigned long long) * 2) != cudaSuccess) {
        release();
        return BD_ERR_OOM;
    }
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t r) {
        if (e == cudaSuccess) { e = r; }
        return e == cudaSuccess;
    };
    const uint32_t src32 = (uint32_t)source;
    step(cudaMemset(depth, 0xff, sizeof(int32_t) * n));
    step(cudaMemset(depth + source, 0, sizeof(int32_t)));
    step(cudaMemcpy(q[0], &src32, sizeof(uint32_t), cudaMemcpyHostToDevice));
    if (e == cudaSuccess) { step(search_levels(g, depth, q, cnt, 1)); }
    unsigned long long first_bad = ULLONG_MAX;
    if (step(cudaMemset(cnt + 1, 0xff, sizeof(unsigned long long)))) {
        check_verify_kernel<<<grid_for_warps(n), kThreads>>>(g->d_off, g->d_adj, n, source, depth,
                                                             d_parent, cnt + 1);
        if (step(cudaGetLastError())) {
            step(cudaMemcpy(&first_bad, cnt + 1, sizeof(first_bad), cudaMemcpyDeviceToHost));
        }
    }
    release();
    if (e != cudaSuccess) { return cuda_fail(e, "device check", __FILE__, __LINE__); }
    *ok = first_bad == ULLONG_MAX ? 1 : 0;
    if (bad_vertex) { *bad_vertex = first_bad == ULLONG_MAX ? -1 : (int64_t)first_bad; }
    return BD_OK;
}

bd_status check_components_device(const bd_graph *g, const int64_t *d_label, int32_t *ok,
                                  int64_t *bad_vertex)
{
    const int64_t n = g->n;
    if (n <= 0) { return BD_ERR_INVALID; }
    BD_CUDA(cudaSetDevice(g->device));
    int64_t *sorted_label = nullptr;
    uint32_t *vertex = nullptr, *sorted_vertex = nullptr;
    int32_t *depth = nullptr;
    uint32_t *q[2] = {nullptr, nullptr};
    unsigned long long *cnt = nullptr;  // [0] queue length, [1] lowest failing vertex
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    auto release = [&]() {
        cudaFree(sorted_label);
        cudaFree(vertex);
        cudaFree(sorted_vertex);
        cudaFree(depth);
        cudaFree(q[0]);
        cudaFree(q[1]);
        cudaFree(cnt);
        cudaFree(scratch);
    };
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, scratch_bytes, d_label, sorted_label,
                                                    vertex, sorted_vertex, n);
    if (e != cudaSuccess) { return cuda_fail(e, "components check", __FILE__, __LINE__); }
    if (cudaMalloc(&sorted_label, sizeof(int64_t) * n) != cudaSuccess ||
        cudaMalloc(&vertex, sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&sorted_vertex, sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&depth, sizeof(int32_t) * n) != cudaSuccess ||
        cudaMalloc(&q[0], sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&q[1], sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&cnt, sizeof(unsigned long long) * 2) != cudaSuccess ||
        cudaMalloc(&scratch, scratch_bytes ? scratch_bytes : 1) != cudaSuccess) {
        release();
        return BD_ERR_OOM;
    }
    auto step = [&](cudaError_t r) {
        if (e == cudaSuccess) { e = r; }
        return e == cudaSuccess;
    };
    iota_kernel<<<grid_for(n), kThreads>>>(vertex, n);
    step(cudaGetLastError());
    step(cub::DeviceRadixSort::SortPairs(scratch, scratch_bytes, d_label, sorted_label, vertex,
                                         sorted_vertex, n));
    step(cudaMemset(depth, 0xff, sizeof(int32_t) * n));
    step(cudaMemset(cnt, 0, sizeof(unsigned long long)));
    unsigned long long sources = 0;
    if (e == cudaSuccess) {
        label_sources_kernel<<<grid_for(n), kThreads>>>(sorted_label, sorted_vertex, n, depth, q[0],
                                                        cnt);
        if (step(cudaGetLastError())) {
            step(cudaMemcpy(&sources, cnt, sizeof(sources), cudaMemcpyDeviceToHost));
        }
    }
    if (e == cudaSuccess) { step(search_levels(g, depth, q, cnt, sources)); }
    unsigned long long first_bad = ULLONG_MAX;
    if (step(cudaMemset(cnt + 1, 0xff, sizeof(unsigned long long)))) {
        check_components_kernel<<<grid_for_warps(n), kThreads>>>(g->d_off, g->d_adj, n, depth,
                                                                 d_label, cnt + 1);
        if (step(cudaGetLastError())) {
            step(cudaMemcpy(&first_bad, cnt + 1, sizeof(first_bad), cudaMemcpyDeviceToHost));
        }
    }
    release();
    if (e != cudaSuccess) { return cuda_fail(e, "components check", __FILE__, __LINE__); }
    *ok = first_bad == ULLONG_MAX ? 1 : 0;
    if (bad_vertex) { *bad_vertex = first_bad == ULLONG_MAX ? -1 : (int64_t)first_bad; }
    return BD_OK;
}

}  // namespace bd

extern "C" {

bd_status bd_graph_check_parents(const bd_graph *g, int64_t source, const int64_t *parent,
                                 int32_t *ok, int64_t *bad_vertex)
{
    if (!g || !parent || !ok) { return BD_ERR_INVALID; }
    if (source < 0 || source >= g->n) { return BD_ERR_RANGE; }
    BD_TRY(bd::ensure_device());
    BD_CUDA(cudaSetDevice(g->device));
    int64_t *d_parent = nullptr;
    if (cudaMalloc(&d_parent, sizeof(int64_t) * g->n) != cudaSuccess) { return BD_ERR_OOM; }
    const cudaError_t e =
        cudaMemcpy(d_parent, parent, sizeof(int64_t) * g->n, cudaMemcpyHostToDevice);
    const bd_status st = e == cudaSuccess
                             ? bd::check_parents_device(g, source, d_parent, ok, bad_vertex)
                             : bd::cuda_fail(e, "copy parents", __FILE__, __LINE__);
    cudaFree(d_parent);
    return st;
}


bd_status bd_graph_check_components(const bd_graph *g, const int64_t *component, int32_t *ok,
                                    int64_t *bad_vertex)
{
    if (!g || !component || !ok) { return BD_ERR_INVALID; }
    if (g->n <= 0) { return BD_ERR_INVALID; }
    BD_TRY(bd::ensure_device());
    BD_CUDA(cudaSetDevice(g->device));
    int64_t *d_label = nullptr;
    if (cudaMalloc(&d_label, sizeof(int64_t) * g->n) != cudaSuccess) { return BD_ERR_OOM; }
    const cudaError_t e =
        cudaMemcpy(d_label, component, sizeof(int64_t) * g->n, cudaMemcpyHostToDevice);
    const bd_status st = e == cudaSuccess
                             ? bd::check_components_device(g, d_label, ok, bad_vertex)
                             : bd::cuda_fail(e, "copy labels", __FILE__, __LINE__);
    cudaFree(d_label);
    return st;
}

}  // extern "C"
