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
// Here a union-find forest in HBM (one uint32 parent per vertex; at scale
// 24 the 64 MB array stays in L2) is built by joins of arcs; joining links
// the larger root under the smaller one with one atomicCAS on the larger
// root's parent word, so every parent id is smaller than its child's and
// every root is the minimum id of its tree: the final roots are exactly the
// reference's labels.  Finds shorten paths as they walk (path splitting:
// each visited vertex is pointed at its grandparent, an ancestor, so the
// forest stays valid under concurrent finds and links).  Every loop ends: a
// find walks strictly decreasing ids, and a join retries only after another
// thread's link took its root, which happens at most n - 1 times in all.
//
// Which arcs are joined (symmetric CSR, every edge stored both ways), after
// Sutton, Ben-Nun and Barak, "Optimizing Parallel Graph Connectivity
// Computation via Subgraph Sampling" (IPDPS 2018, "Afforest"):
//   cc_sample_first_kernel, cc_sample_second_kernel
//                         every vertex joins its first arc, then its
//                         second, each round followed by pointing every
//                         vertex at its root (cc_flatten_kernel);
//   the largest tree      found by sampling kProbe vertices' roots;
//   cc_walk_kernel        every vertex OUTSIDE that tree (its parent word
//                         is not the tree's root) joins the rest of its
//                         arcs.  An edge between the largest tree and
//                         another vertex is stored at that other vertex
//                         too, and is joined from there, so skipping the
//                         largest tree's own arcs loses no edge.  A warp
//                         loads 32 vertices' parent words at once and walks
//                         only the lists of those with work; lists of more
//                         than kHeavy arcs go to cc_heavy_kernel, which
//                         deals every listed vertex's arcs over the grid in
//                         one flat range (a binary search per chunk, the
//                         chunk prefix from cc_heavy_chunks_kernel).
//   cc_compress_kernel    labels (each vertex's root), sizes per label
//                         (one atomic per distinct label of a warp) and the
//                         count of roots.
// A CSR that does not hold every edge both ways takes every arc of every
// vertex instead (the same cc_walk_kernel / cc_heavy_kernel pair).
#include <algorithm>
#include <cstring>
#include <vector>

#include "bd_internal.h"

namespace bd {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int64_t kHeavy = 4096;    // arcs above which a vertex is split over the grid
constexpr int kSampleArcs = 2;      // arc positions joined before the rest of the lists
constexpr int kProbe = 1024;        // vertices whose roots vote for the largest tree
constexpr int64_t kHeavyChunk = 1024;  // arcs per unit of the heavy pass

int grid_for_warps(int64_t warps)
{
    int64_t b = (warps + kWarps - 1) / kWarps;
    if (b < 1) { b = 1; }
    if (b > 148 * 64) { b = 148 * 64; }
    return (int)b;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x)
{
    for (int d = 16; d > 0; d >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, d); }
    return x;
}

// Root of x's tree, pointing each vertex on the way at its grandparent.
//
// The loads go through L1 (ld.ca), which is not coherent between SMs, so a
// load may return an older value of a parent word.  That is safe: every
// value a parent word ever holds is an ancestor of its vertex with a
// smaller id (links and path splitting only write ancestors, and a tree
// only grows), so a stale walk still descends strictly and ends at a
// vertex that is, or was, a root of x's tree.  A join acts on such a root
// only through atomicCAS, which sees the current word.  What L1 buys: after
// a sampling round nearly every vertex points at the largest tree's root,
// and checking that root's own word from every thread put millions of
// loads on one L2 slice (a second sampling round ran 3x slower than the
// first); from L1 each SM loads it once.
__device__ __forceinline__ uint32_t cc_find(uint32_t *parent, uint32_t x)
{
    uint32_t p = __ldca(&parent[x]);
    while (p != x) {
        const uint32_t gp = __ldca(&parent[p]);
        if (gp != p) { __stcg(&parent[x], gp); }
        x = p;
        p = gp;
    }
    return x;
}

// Root of x's tree without writes, for passes in which no join runs (the
// roots stay fixed, so the walk ends at x's current root).
__device__ __forceinline__ uint32_t cc_root(const uint32_t *parent, uint32_t x)
{
    uint32_t p = __ldca(&parent[x]);
    while (p != x) {
        x = p;
        p = __ldca(&parent[x]);
    }
    return x;
}

// Joins the trees of a and b: the larger root goes under the smaller.
__device__ __forceinline__ void cc_join(uint32_t *parent, uint32_t a, uint32_t b)
{
    // one parent word each: vertices pointing at the same vertex share a
    // tree (after a flatten, the common case)
    if (__ldca(&parent[a]) == __ldca(&parent[b])) { return; }
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

// First sampling round: every vertex joins its first arc.  Its second arc
// (in the same 32-byte sector of the adjacency) is kept in `second` for the
// next round, which then reads 4 coalesced bytes per vertex instead of two
// offsets and a random adjacency sector again; a vertex with fewer than two
// arcs keeps its own id (joining itself does nothing).
__global__ void cc_sample_first_kernel(const int64_t *off, const uint32_t *adj, int64_t n,
                                       uint32_t *parent, uint32_t *second)
{
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = off[u], e = off[u + 1];
        uint32_t nxt = (uint32_t)u;
        if (e > b) {
            const uint32_t a0 = __ldg(&adj[b]);
            if (e - b > 1) { nxt = __ldg(&adj[b + 1]); }
            cc_join(parent, (uint32_t)u, a0);
        }
        __stcs(&second[u], nxt);
    }
}

// Second sampling round: every vertex joins its second arc.
__global__ void cc_sample_second_kernel(const uint32_t *second, int64_t n, uint32_t *parent)
{
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n;
         u += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = __ldcs(&second[u]);
        if (v != (uint32_t)u) { cc_join(parent, (uint32_t)u, v); }
    }
}

// Every vertex pointed at its root (a vertex already there is not
// written).  No join runs meanwhile, so the roots are fixed; the walks do
// not split paths, so no thread moves a word another thread has already
// pointed at its root.
__global__ void cc_flatten_kernel(uint32_t *parent, int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = __ldcg(&parent[v]);
        const uint32_t r = cc_root(parent, p);
        if (r != p) { __stcg(&parent[v], r); }
    }
}

// Roots of kProbe vertices spread evenly over the ids.
__global__ void cc_probe_kernel(uint32_t *parent, int64_t n, uint32_t *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kProbe) {
        const uint32_t v = (uint32_t)(((uint64_t)i * (uint64_t)n) / kProbe);
        out[i] = cc_find(parent, v);
    }
}

// Arcs [first, e) of the vertices of a warp's 32-vertex group that have
// work: each such vertex's list is walked by the whole warp, 32 arcs a
// round; lists longer than kHeavy are appended to `heavy` instead.
// skip_root: vertices whose root is this id have no work (the largest
// tree), or ~0u for none; first: arc position to start at; all_arcs: join
// every arc (else only arcs to smaller ids: each edge once, from its larger
// endpoint).
__global__ void __launch_bounds__(kThreads) cc_walk_kernel(
    const int64_t *off, const uint32_t *adj, int64_t n, uint32_t *parent, uint32_t skip_root,
    int first, int all_arcs, uint32_t *heavy, unsigned long long *heavy_count)
{
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = gw * 32; base < n; base += nw * 32) {
        const int64_t u = base + lane;
        int64_t b = 0, e = 0;
        bool work = false;
        if (u < n) {
            b = off[u] + first;
            e = off[u + 1];
            work = b < e && (skip_root == ~0u || __ldcg(&parent[u]) != skip_root);
            if (work && e - b > kHeavy) {
                heavy[atomicAdd(heavy_count, 1ull)] = (uint32_t)u;
                work = false;
            }
        }
        unsigned todo = __ballot_sync(0xffffffffu, work);
        while (todo) {
            const int owner = __ffs(todo) - 1;
            todo &= todo - 1;
            const int64_t bb = __shfl_sync(0xffffffffu, b, owner);
            const int64_t ee = __shfl_sync(0xffffffffu, e, owner);
            const uint32_t uu = (uint32_t)(base + owner);
            for (int64_t k = bb + lane; k < ee; k += 32) {
                const uint32_t v = __ldg(&adj[k]);
                if (all_arcs || v < uu) { cc_join(parent, uu, v); }
            }
        }
    }
}

// Chunk prefix of the heavy list: cbase[i] = chunks of heavy vertices < i.
// One block of 1024 threads scans 1024 entries per round.
__global__ void __launch_bounds__(1024) cc_heavy_chunks_kernel(
    const int64_t *off, const uint32_t *heavy, const unsigned long long *heavy_count, int first,
    unsigned long long *cbase)
{
    __shared__ unsigned long long warp_tot[32];
    __shared__ unsigned long long carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t count = (int64_t)*heavy_count;
    if (threadIdx.x == 0) { carry = 0; }
    __syncthreads();
    for (int64_t base = 0; base < count; base += 1024) {
        const int64_t i = base + threadIdx.x;
        unsigned long long c = 0;
        if (i < count) {
            const uint32_t u = heavy[i];
            const int64_t len = off[u + 1] - (off[u] + first);
            c = (unsigned long long)((len + kHeavyChunk - 1) / kHeavyChunk);
        }
        unsigned long long incl = c;
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) { incl += y; }
        }
        if (lane == 31) { warp_tot[warp] = incl; }
        __syncthreads();
        if (warp == 0) {
            unsigned long long t = warp_tot[lane];
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) { t += y; }
            }
            warp_tot[lane] = t;  // inclusive prefix over warps
        }
        __syncthreads();
        const unsigned long long before = carry + (warp ? warp_tot[warp - 1] : 0ull);
        if (i < count) { cbase[i] = before + incl - c; }
        __syncthreads();
        if (threadIdx.x == 1023) { carry = before + incl; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { cbase[count] = carry; }
}

// The heavy vertices' arcs as one flat range of kHeavyChunk-arc chunks dealt
// to the warps of the grid (a warp per chunk, a binary search for its
// vertex), so no thread walks one vertex's chunks after another.
__global__ void __launch_bounds__(kThreads) cc_heavy_kernel(
    const int64_t *off, const uint32_t *adj, uint32_t *parent, const uint32_t *heavy,
    const unsigned long long *heavy_count, const unsigned long long *cbase, int first,
    int all_arcs)
{
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t count = (int64_t)*heavy_count;
    if (count == 0) { return; }
    const int64_t total = (int64_t)cbase[count];
    for (int64_t c = gw; c < total; c += nw) {
        int64_t lo = 0, hi = count - 1;  // last i with cbase[i] <= c
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) >> 1;
            if ((int64_t)cbase[mid] <= c) { lo = mid; } else { hi = mid - 1; }
        }
        const uint32_t u = heavy[lo];
        const int64_t b = off[u] + first + (c - (int64_t)cbase[lo]) * kHeavyChunk;
        const int64_t e = min(off[u + 1], b + kHeavyChunk);
        for (int64_t k = b + lane; k < e; k += 32) {
            const uint32_t v = __ldg(&adj[k]);
            if (all_arcs || v < u) { cc_join(parent, u, v); }
        }
    }
}

// Labels, sizes and roots.  `hint` is a vertex of the largest tree (or
// ~0u): the lanes whose label is that tree's root count it in a block-wide
// total added once per block, as do the roots; the lanes of a warp that
// share any other label add it once (__match_any_sync).  (One atomic per
// warp on the largest component's size and on the root count put a few
// hundred thousand atomics on two addresses, which serialise at their L2
// slices.)
__global__ void cc_compress_kernel(uint32_t *parent, int64_t n, uint32_t hint, int64_t *label,
                                   int64_t *size, unsigned long long *roots)
{
    __shared__ uint32_t giant;
    __shared__ unsigned long long blk_giant, blk_roots;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        giant = hint < n ? cc_root(parent, hint) : 0xFFFFFFFFu;
        blk_giant = blk_roots = 0;
    }
    __syncthreads();
    const uint32_t g = giant;
    unsigned long long my_giant = 0, my_roots = 0;
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane; base < n;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = base + lane;
        const bool valid = v < n;
        uint32_t r = 0xFFFFFFFFu;
        if (valid) {
            // a vertex pointing at the largest tree's root needs no walk
            const uint32_t p = __ldcs(&parent[v]);
            r = p == g ? g : cc_root(parent, p);
            __stcs(&label[v], (int64_t)r);
        }
        const bool other = valid && r != g;
        const unsigned same = __match_any_sync(0xffffffffu, other ? r : 0xFFFFFFFFu);
        if (other && lane == __ffs(same) - 1) {
            atomicAdd(reinterpret_cast<unsigned long long *>(&size[r]),
                      (unsigned long long)__popc(same));
        }
        my_giant += (valid && r == g) ? 1ull : 0ull;
        my_roots += (valid && r == (uint32_t)v) ? 1ull : 0ull;
    }
    my_giant = warp_sum_u64(my_giant);
    my_roots = warp_sum_u64(my_roots);
    if (lane == 0) {
        if (my_giant) { atomicAdd(&blk_giant, my_giant); }
        if (my_roots) { atomicAdd(&blk_roots, my_roots); }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (blk_giant) {
            atomicAdd(reinterpret_cast<unsigned long long *>(&size[g]), blk_giant);
        }
        if (blk_roots) { atomicAdd(roots, blk_roots); }
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
    unsigned long long *cbase = nullptr;   // [arcs / kHeavy + 2] their chunk prefix
    uint32_t *probe = nullptr;             // [kProbe] sampled roots
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
    cudaFree(c->cbase);
    cudaFree(c->probe);
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
        cudaMalloc(&c->cbase, sizeof(unsigned long long) * (heavy_cap + 1)) != cudaSuccess ||
        cudaMalloc(&c->probe, sizeof(uint32_t) * bd::kProbe) != cudaSuccess ||
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
    uint32_t skip = ~0u;
    int first = 0;
    if (g->symmetric) {
        // the first and the second arc of every vertex, each round followed
        // by pointing every vertex at its root (the next round's finds are
        // short, and after the last one the largest tree's vertices are
        // recognised by one parent word)
        // (the label array, written only by the final pass, holds the
        // second arcs meanwhile)
        uint32_t *second = reinterpret_cast<uint32_t *>(c->label);
        bd::cc_sample_first_kernel<<<bd::grid_for(n), bd::kThreads, 0, s>>>(
            g->d_off, g->d_adj, n, c->parent, second);
        bd::cc_flatten_kernel<<<bd::grid_for(n), bd::kThreads, 0, s>>>(c->parent, n);
        bd::cc_sample_second_kernel<<<bd::grid_for(n), bd::kThreads, 0, s>>>(second, n, c->parent);
        bd::cc_flatten_kernel<<<bd::grid_for(n), bd::kThreads, 0, s>>>(c->parent, n);
        bd::cc_probe_kernel<<<(bd::kProbe + 255) / 256, 256, 0, s>>>(c->parent, n, c->probe);
        BD_CUDA(cudaGetLastError());
        std::vector<uint32_t> probe(bd::kProbe);
        BD_CUDA(cudaMemcpyAsync(probe.data(), c->probe, sizeof(uint32_t) * bd::kProbe,
                                cudaMemcpyDeviceToHost, s));
        BD_CUDA(cudaStreamSynchronize(s));
        // the most frequent root among the probes: the largest tree
        std::sort(probe.begin(), probe.end());
        size_t best = 0;
        for (size_t i = 0, j = 0; i < probe.size(); i = j) {
            for (j = i; j < probe.size() && probe[j] == probe[i]; ++j) {}
            if (j - i > best) {
                best = j - i;
                skip = probe[i];
            }
        }
        first = bd::kSampleArcs;
    }
    // symmetric: the rest of the arcs of vertices outside the largest tree;
    // otherwise every arc of every vertex
    bd::cc_walk_kernel<<<bd::grid_for_warps(n), bd::kThreads, 0, s>>>(
        g->d_off, g->d_adj, n, c->parent, skip, first, 1, c->heavy, c->counters);
    bd::cc_heavy_chunks_kernel<<<1, 1024, 0, s>>>(g->d_off, c->heavy, c->counters, first,
                                                  c->cbase);
    bd::cc_heavy_kernel<<<148 * 8, bd::kThreads, 0, s>>>(g->d_off, g->d_adj, c->parent, c->heavy,
                                                        c->counters, c->cbase, first, 1);
    bd::cc_compress_kernel<<<bd::grid_for(n), bd::kThreads, 0, s>>>(c->parent, n, skip, c->label,
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
