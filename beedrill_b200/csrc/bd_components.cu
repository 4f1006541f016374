// bd_components.cu -- connected components (components.cc:38-118) on the
// device.
//
// The reference labels every vertex with the smallest vertex id of its
// component by label propagation: passes over all arcs lower a vertex's
// label to a neighbour's smaller one, pointer jumping shortens label
// chains, and passes repeat until nothing changes (num_iters of them).
// The labelling it converges to is unique -- each vertex gets the minimum
// id of its component -- so any algorithm that finds the components and
// names each by its minimum id gives the reference's labels exactly.
//
// Here one pass over the arcs builds a union-find forest in HBM (one
// uint32 parent per vertex; at scale 24 the 64 MB array stays in L2):
//
//   cc_hook_kernel        one warp per vertex, lanes over its arcs; each
//                         arc (u, v) with v < u joins the trees of u and v
//                         (a symmetric CSR holds every edge twice, once in
//                         each direction; any other CSR joins every arc).
//                         Vertices of more than kHeavy arcs are listed
//                         for the next kernel instead.
//   cc_hook_heavy_kernel  the listed vertices, each one's arcs spread over
//                         every thread of the grid.
//   cc_compress_kernel    each vertex's label becomes its tree's root;
//                         sizes per label and the count of roots.
//
// Joining links the larger root under the smaller one with one atomicCAS
// on the larger root's parent word, so every parent id is smaller than its
// child's and every root is the minimum id of its tree: the final roots
// are exactly the reference's labels.  Finds shorten paths as they walk
// (path splitting: each visited vertex is pointed at its grandparent, an
// ancestor, so the forest stays valid under concurrent finds and links).
// Every loop ends: a find walks strictly decreasing ids, and a join retries
// only after another thread's link took its root, which happens at most
// n - 1 times in all.
#include <cstring>

#include "bd_internal.h"

namespace bd {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int64_t kHeavy = 4096;  // arcs above which a vertex is split over the grid

int grid_for_warps(int64_t warps)
{
    int64_t b = (warps + kWarps - 1) / kWarps;
    if (b < 1) { b = 1; }
    if (b > 148 * 64) { b = 148 * 64; }
    return (int)b;
}

// Root of x's tree, pointing each vertex on the way at its grandparent.
__device__ __forceinline__ uint32_t cc_find(uint32_t *parent, uint32_t x)
{
    uint32_t p = __ldcg(&parent[x]);
    while (p != x) {
        const uint32_t gp = __ldcg(&parent[p]);
        if (gp != p) { __stcg(&parent[x], gp); }
        x = p;
        p = gp;
    }
    return x;
}

// Joins the trees of a and b: the larger root goes under the smaller.
__device__ __forceinline__ void cc_join(uint32_t *parent, uint32_t a, uint32_t b)
{
    uint32_t ra = cc_find(parent, a), rb = cc_find(parent, b);
    while (ra != rb) {
        if (ra < rb) {
            const uint32_t t = ra;
            ra = rb;
            rb = t;
        }
        const uint32_t old = atomicCAS(&parent[ra], ra, rb);
        if (old == ra) { return; }
        // ra was linked under `old` meanwhile; both roots may have moved.
        ra = cc_find(parent, old);
        rb = cc_find(parent, rb);
    }
}

__global__ void cc_init_kernel(uint32_t *parent, int64_t n, int64_t *size)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        parent[v] = (uint32_t)v;
        size[v] = 0;
    }
}

__global__ void __launch_bounds__(kThreads) cc_hook_kernel(
    const int64_t *off, const uint32_t *adj, int64_t n, int symmetric, uint32_t *parent,
    uint32_t *heavy, unsigned long long *heavy_count)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * kWarps;
    for (int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; u < n; u += warps) {
        const int64_t b = off[u], e = off[u + 1];
        if (e - b > kHeavy) {
            if (lane == 0) { heavy[atomicAdd(heavy_count, 1ull)] = (uint32_t)u; }
            continue;
        }
        for (int64_t k = b + lane; k < e; k += 32) {
            const uint32_t v = adj[k];
            if (!symmetric || v < (uint32_t)u) { cc_join(parent, (uint32_t)u, v); }
        }
    }
}

__global__ void __launch_bounds__(kThreads) cc_hook_heavy_kernel(
    const int64_t *off, const uint32_t *adj, int symmetric, uint32_t *parent,
    const uint32_t *heavy, const unsigned long long *heavy_count)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t count = (int64_t)*heavy_count;
    for (int64_t i = 0; i < count; ++i) {
        const uint32_t u = heavy[i];
        const int64_t e = off[u + 1];
        for (int64_t k = off[u] + t; k < e; k += stride) {
            const uint32_t v = adj[k];
            if (!symmetric || v < u) { cc_join(parent, u, v); }
        }
    }
}

__global__ void cc_compress_kernel(uint32_t *parent, int64_t n, int64_t *label, int64_t *size,
                                   unsigned long long *roots)
{
    const int lane = threadIdx.x & 31;
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane; base < n;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = base + lane;
        bool root = false;
        if (v < n) {
            const uint32_t r = cc_find(parent, (uint32_t)v);
            __stcg(&parent[v], r);
            label[v] = r;
            atomicAdd(reinterpret_cast<unsigned long long *>(&size[r]), 1ull);
            root = r == (uint32_t)v;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, root);
        if (lane == 0 && mask) { atomicAdd(roots, (unsigned long long)__popc(mask)); }
    }
}

int grid_for(int64_t items)
{
    int64_t b = (items + kThreads - 1) / kThreads;
    if (b < 1) { b = 1; }
    if (b > 148 * 64) { b = 148 * 64; }
    return (int)b;
}

}  // namespace
}  // namespace bd

// Handle: the graph it borrows, its stream and the device arrays.
struct bd_components {
    int device = 0;
    bd_graph *g = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t *parent = nullptr;            // [n] union-find forest
    uint32_t *heavy = nullptr;             // [arcs / kHeavy + 1] vertices split over the grid
    unsigned long long *counters = nullptr;  // [0] heavy vertices, [1] roots
    int64_t *label = nullptr;              // [n] component_ (components.h:13)
    int64_t *size = nullptr;               // [n] component_size_ (components.h:15)
    bool ran = false;
    bd_components_stats last{};
};

namespace {

void components_free(bd_components *c)
{
    if (!c) { return; }
    cudaSetDevice(c->device);
    if (c->stream) { cudaStreamSynchronize(c->stream); }
    cudaFree(c->parent);
    cudaFree(c->heavy);
    cudaFree(c->counters);
    cudaFree(c->label);
    cudaFree(c->size);
    if (c->ev0) { cudaEventDestroy(c->ev0); }
    if (c->ev1) { cudaEventDestroy(c->ev1); }
    if (c->stream) { cudaStreamDestroy(c->stream); }
    delete c;
}

}  // namespace

extern "C" {

bd_status bd_components_create(bd_graph *g, bd_components **out)
{
    if (!g || !out) { return BD_ERR_INVALID; }
    BD_TRY(bd::ensure_device());
    BD_CUDA(cudaSetDevice(g->device));
    auto *c = new bd_components();
    c->device = g->device;
    c->g = g;
    const int64_t n = g->n;
    const int64_t heavy_cap = g->arcs / bd::kHeavy + 1;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaMalloc(&c->parent, sizeof(uint32_t) * (n ? n : 1)) != cudaSuccess ||
        cudaMalloc(&c->heavy, sizeof(uint32_t) * heavy_cap) != cudaSuccess ||
        cudaMalloc(&c->counters, sizeof(unsigned long long) * 2) != cudaSuccess ||
        cudaMalloc(&c->label, sizeof(int64_t) * (n ? n : 1)) != cudaSuccess ||
        cudaMalloc(&c->size, sizeof(int64_t) * (n ? n : 1)) != cudaSuccess) {
        components_free(c);
        return BD_ERR_OOM;
    }
    *out = c;
    return BD_OK;
}

// components::clear (components.cc:33-36) does nothing; run() starts over.
bd_status bd_components_clear(bd_components *c)
{
    if (!c) { return BD_ERR_INVALID; }
    return BD_OK;
}

bd_status bd_components_run(bd_components *c, bd_components_stats *stats)
{
    if (!c) { return BD_ERR_INVALID; }
    BD_CUDA(cudaSetDevice(c->device));
    const bd_graph *g = c->g;
    const int64_t n = g->n;
    cudaStream_t s = c->stream;
    BD_CUDA(cudaEventRecord(c->ev0, s));
    BD_CUDA(cudaMemsetAsync(c->counters, 0, sizeof(unsigned long long) * 2, s));
    bd::cc_init_kernel<<<bd::grid_for(n), bd::kThreads, 0, s>>>(c->parent, n, c->size);
    bd::cc_hook_kernel<<<bd::grid_for_warps(n), bd::kThreads, 0, s>>>(
        g->d_off, g->d_adj, n, g->symmetric ? 1 : 0, c->parent, c->heavy, c->counters);
    bd::cc_hook_heavy_kernel<<<148 * 8, bd::kThreads, 0, s>>>(
        g->d_off, g->d_adj, g->symmetric ? 1 : 0, c->parent, c->heavy, c->counters);
    bd::cc_compress_kernel<<<bd::grid_for(n), bd::kThreads, 0, s>>>(c->parent, n, c->label,
                                                                    c->size, c->counters + 1);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaEventRecord(c->ev1, s));
    unsigned long long roots = 0;
    BD_CUDA(cudaMemcpyAsync(&roots, c->counters + 1, sizeof(roots), cudaMemcpyDeviceToHost, s));
    BD_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    BD_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last.num_components = (int64_t)roots;
    c->last.num_iters = 1;
    c->last.ms = ms;
    c->ran = true;
    if (stats) { *stats = c->last; }
    return BD_OK;
}

bd_status bd_components_get_labels(bd_components *c, int64_t *component)
{
    if (!c || !component) { return BD_ERR_INVALID; }
    if (!c->ran) { return BD_ERR_STATE; }
    BD_CUDA(cudaSetDevice(c->device));
    BD_CUDA(cudaMemcpy(component, c->label, sizeof(int64_t) * c->g->n, cudaMemcpyDeviceToHost));
    return BD_OK;
}

bd_status bd_components_get_sizes(bd_components *c, int64_t *component_size)
{
    if (!c || !component_size) { return BD_ERR_INVALID; }
    if (!c->ran) { return BD_ERR_STATE; }
    BD_CUDA(cudaSetDevice(c->device));
    BD_CUDA(cudaMemcpy(component_size, c->size, sizeof(int64_t) * c->g->n, cudaMemcpyDeviceToHost));
    return BD_OK;
}

bd_status bd_components_device_labels(bd_components *c, const int64_t **component)
{
    if (!c || !component) { return BD_ERR_INVALID; }
    if (!c->ran) { return BD_ERR_STATE; }
    *component = c->label;
    return BD_OK;
}

bd_status bd_components_check(bd_components *c, int32_t *ok)
{
    if (!c || !ok) { return BD_ERR_INVALID; }
    if (!c->ran) { return BD_ERR_STATE; }
    return bd::check_components_device(c->g, c->label, ok, nullptr);
}

bd_status bd_components_destroy(bd_components *c)
{
    if (!c) { return BD_ERR_INVALID; }
    components_free(c);
    return BD_OK;
}

}  // extern "C"
