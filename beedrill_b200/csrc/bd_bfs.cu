// bd_bfs.cu -- the B200 direction-optimizing BFS (hybrid_bfs) and its C ABI.
//
// Data layout in HBM for one handle (n vertices, arcs = 2m):
//   depth   int32[n]      -1 = unvisited; claimed by atomicCAS in top-down
//   parent  int64[n]      written once per reached vertex; the reference's
//                         -deg / -1 encoding of unreached vertices is filled
//                         in lazily (finalize_parents_kernel) when read
//   vis[2]  uint32[n/32]  visited bitmaps; a bottom-up step reads vis[cur]
//                         (frozen) and writes whole words of vis[cur^1]
//   qs[2]   uint32[n]     frontier queue of vertices with degree < large_deg
//   ql[2], qlb[2]         frontier vertices with degree >= large_deg, with the
//                         prefix sum of their chunk counts (work units of
//                         `chunk` edges spread over all warps)
//   ctrl                  Ctrl block: barrier, Beamer state, step counters
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "bd_bfs_device.cuh"
#include "bd_device_util.cuh"
#include "bd_internal.h"

namespace bd {

namespace {

constexpr int64_t kRecCap = 1 << 15;
constexpr long long kDefaultSpin = 4000000;  // ~2 s of polling

using namespace dev;

// Per-thread accumulators of one step, reduced once per CTA at its end.
struct Local {
    unsigned long long found;
    unsigned long long degsum;
};

// What a step needs of the traversal state, in registers.
struct StepView {
    int dir;
    int level;
    int vis_cur;
    int q_cur;
    int step;
    int bu_sparse;
    long long f_small;
    long long f_large;
    long long f_chunks;
};

__device__ __forceinline__ StepView view_of(const LevelState &s)
{
    StepView v;
    v.dir = s.dir;
    v.bu_sparse = s.bu_sparse;
    v.level = s.level;
    v.vis_cur = s.vis_cur;
    v.q_cur = s.q_cur;
    v.step = s.step;
    v.f_small = s.f_small;
    v.f_large = s.f_large;
    v.f_chunks = s.f_chunks;
    return v;
}

// Visited-bit lookups.  A plain (L1-cacheable) load is correct here: the
// bitmap a bottom-up step reads is not written during that step, and every
// CTA passes the grid barrier's acquire before the step, after which weak
// loads observe all writes made before the barrier (PTX memory model).
__device__ __forceinline__ uint32_t ld_bits(const uint32_t *p) { return *p; }

// Warp-collective: reserves `count` large-queue slots and `chunks` chunk ids
// for this lane with one atomic for the whole warp.  Slots and chunk ids are
// handed out in the same lane order, so chunk bases stay sorted by slot.
__device__ __forceinline__ void warp_reserve_large(Acc *acc, unsigned count,
                                                   unsigned long long chunks,
                                                   unsigned long long &pos,
                                                   unsigned long long &cbase)
{
    const unsigned ci = warp_incl_scan(count);
    const unsigned long long hi = warp_incl_scan(chunks);
    const unsigned ct = __shfl_sync(kFull, ci, 31);
    const unsigned long long ht = __shfl_sync(kFull, hi, 31);
    unsigned long long old = 0;
    if (lane_id() == 0 && ct) {
        old = atomicAdd(&acc->large_packed, ((unsigned long long)ct << kLargeShift) | ht);
    }
    old = __shfl_sync(kFull, old, 0);
    pos = (old >> kLargeShift) + (ci - count);
    cbase = (old & kChunkMask) + (hi - chunks);
}

// Warp-collective append of up to K discoveries per lane with one atomic
// for all the small-degree ones.
template <int K>
__device__ __forceinline__ void warp_append_k(const BfsParams &p, Acc *acc, int qout,
                                              const bool (&has)[K], const uint32_t (&v)[K],
                                              const int64_t (&deg)[K], Local &loc)
{
    const int lane = lane_id();
    unsigned sm[K];
    bool large[K];
    unsigned total = 0, any_large = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (has[k]) {
            loc.found += 1;
            loc.degsum += (unsigned long long)deg[k];
        }
        large[k] = has[k] && deg[k] >= (int64_t)p.large_deg;
        sm[k] = __ballot_sync(kFull, has[k] && !large[k]);
        total += __popc(sm[k]);
        any_large |= __ballot_sync(kFull, large[k]);
    }
    if (total) {
        unsigned long long base = 0;
        if (lane == 0) { base = atomicAdd(&acc->small_cnt, (unsigned long long)total); }
        base = __shfl_sync(kFull, base, 0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (has[k] && !large[k]) { p.qs[qout][base + __popc(sm[k] & lanemask_lt())] = v[k]; }
            base += __popc(sm[k]);
        }
    }
    if (any_large) {
        unsigned count = 0;
        unsigned long long chunks = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (large[k]) {
                count += 1;
                chunks += (unsigned long long)((deg[k] + p.chunk - 1) / p.chunk);
            }
        }
        unsigned long long pos, cbase;
        warp_reserve_large(acc, count, chunks, pos, cbase);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (large[k]) {
                p.ql[qout][pos] = v[k];
                p.qlb[qout][pos] = cbase;
                pos += 1;
                cbase += (unsigned long long)((deg[k] + p.chunk - 1) / p.chunk);
            }
        }
    }
}

__device__ __forceinline__ int64_t degree_of(const BfsParams &p, uint32_t v)
{
    return __ldg(&p.off[v + 1]) - __ldg(&p.off[v]);
}

constexpr int kILP = 4;

// Top-down claims of a batch of kILP neighbours per lane (hybrid_bfs.cc:83-96):
// visited-bit filter, then atomicCAS on the depth word decides the single
// winner, which writes the parent, sets the visited bit and joins the next
// frontier.  Every stage issues its kILP memory operations back to back.
__device__ __forceinline__ void td_claim_batch(const BfsParams &p, Acc *acc, uint32_t *vis,
                                               int qout, int new_level, const bool (&ok)[kILP],
                                               const uint32_t (&v)[kILP],
                                               const uint32_t (&src)[kILP], Local &loc)
{
    uint32_t w[kILP];
#pragma unroll
    for (int i = 0; i < kILP; ++i) { w[i] = ok[i] ? __ldcg(&vis[v[i] >> 5]) : 0xFFFFFFFFu; }
    int old[kILP];
#pragma unroll
    for (int i = 0; i < kILP; ++i) {
        const bool cand = ok[i] && !((w[i] >> (v[i] & 31)) & 1u);
        old[i] = cand ? atomicCAS(&p.depth[v[i]], -1, new_level) : 0;
    }
    bool won[kILP];
    int64_t deg[kILP];
#pragma unroll
    for (int i = 0; i < kILP; ++i) {
        won[i] = ok[i] && !((w[i] >> (v[i] & 31)) & 1u) && old[i] == -1;
        deg[i] = 0;
        if (won[i]) {
            p.parent[v[i]] = (int64_t)src[i];
            atomicOr(&vis[v[i] >> 5], 1u << (v[i] & 31));
            deg[i] = degree_of(p, v[i]);
        }
    }
    warp_append_k<kILP>(p, acc, qout, won, v, deg, loc);
}

// Processes arcs [b, e) of vertex u with all 32 lanes (coalesced reads).
__device__ __forceinline__ void td_edges_warp(const BfsParams &p, Acc *acc, uint32_t *vis,
                                              int qout, int new_level, uint32_t u, int64_t b,
                                              int64_t e, Local &loc)
{
    const int lane = lane_id();
    for (int64_t base = b; base < e; base += 32 * kILP) {
        uint32_t v[kILP], src[kILP];
        bool ok[kILP];
#pragma unroll
        for (int i = 0; i < kILP; ++i) {
            const int64_t k = base + i * 32 + lane;
            ok[i] = k < e;
            v[i] = ok[i] ? __ldg(&p.adj[k]) : 0u;
            src[i] = u;
        }
        td_claim_batch(p, acc, vis, qout, new_level, ok, v, src, loc);
    }
}

struct WarpScratch {
    int32_t incl[32];
    uint32_t u[32];
    int64_t beg[32];
};

template <int BLOCK>
struct SharedState {
    WarpScratch warp[BLOCK / 32];
    unsigned long long red_found[BLOCK / 32];
    unsigned long long red_deg[BLOCK / 32];
    LevelState st;       // this CTA's copy of the traversal state
    PolicyBlob pol;      // the learned policy's weights, staged once
    int rule_dir;
};

template <int BLOCK>
__device__ void td_step(const BfsParams &p, const StepView &sv, SharedState<BLOCK> &sh,
                        Local &loc)
{
    const int lane = lane_id();
    const int warp = threadIdx.x >> 5;
    const long long gw = (long long)blockIdx.x * (BLOCK / 32) + warp;
    const long long nw = (long long)gridDim.x * (BLOCK / 32);
    const int qin = sv.q_cur, qout = sv.q_cur ^ 1;
    uint32_t *vis = p.vis[sv.vis_cur];
    Acc *acc = &p.ctrl->acc[sv.step % 3];
    const int new_level = sv.level + 1;

    // Phase A: chunks of large-degree frontier vertices.  Warp gw takes a
    // contiguous range of chunk ids, so every warp gets the same number of
    // edges (within one chunk); one binary search finds the range's first
    // vertex, then the walk moves forward.
    const long long nl = sv.f_large;
    const long long nch = sv.f_chunks;
    if (nch > 0) {
        const long long per = (nch + nw - 1) / nw;
        const long long c0 = gw * per;
        const long long c1 = min(nch, c0 + per);
        if (c0 < c1) {
            long long lo = 0, hi = nl - 1;  // last i with qlb[i] <= c0
            while (lo < hi) {
                long long mid = (lo + hi + 1) >> 1;
                if ((long long)__ldcg(&p.qlb[qin][mid]) <= c0) { lo = mid; } else { hi = mid - 1; }
            }
            long long i = lo;
            long long ibase = (long long)__ldcg(&p.qlb[qin][i]);
            long long inext = i + 1 < nl ? (long long)__ldcg(&p.qlb[qin][i + 1]) : nch;
            for (long long c = c0; c < c1; ++c) {
                while (c >= inext) {
                    ++i;
                    ibase = inext;
                    inext = i + 1 < nl ? (long long)__ldcg(&p.qlb[qin][i + 1]) : nch;
                }
                const uint32_t u = __ldcg(&p.ql[qin][i]);
                const int64_t ub = __ldg(&p.off[u]), ue = __ldg(&p.off[u + 1]);
                const int64_t b = ub + (c - ibase) * (int64_t)p.chunk;
                const int64_t e = min(ue, b + (int64_t)p.chunk);
                td_edges_warp(p, acc, vis, qout, new_level, u, b, e, loc);
            }
        }
    }

    // Phase B: small-degree frontier vertices, 32 per warp; their arcs are
    // laid end to end and dealt to the lanes 32 at a time.
    WarpScratch &ws = sh.warp[warp];
    for (long long g = gw; g * 32 < sv.f_small; g += nw) {
        const long long idx = g * 32 + lane;
        uint32_t u = 0;
        int64_t beg = 0;
        int32_t deg = 0;
        if (idx < sv.f_small) {
            u = __ldcg(&p.qs[qin][idx]);
            beg = __ldg(&p.off[u]);
            deg = (int32_t)(__ldg(&p.off[u + 1]) - beg);
        }
        const int32_t incl = warp_incl_scan(deg);
        const int32_t total = __shfl_sync(kFull, incl, 31);
        ws.incl[lane] = incl;
        ws.u[lane] = u;
        ws.beg[lane] = beg;
        __syncwarp();
        for (int32_t base = 0; base < total; base += 32 * kILP) {
            uint32_t v[kILP], src[kILP];
            bool ok[kILP];
#pragma unroll
            for (int i = 0; i < kILP; ++i) {
                const int32_t e = base + i * 32 + lane;
                ok[i] = e < total;
                v[i] = 0;
                src[i] = 0;
                if (ok[i]) {
                    int lo = 0, hi = 31;  // first owner with incl > e
                    while (lo < hi) {
                        int mid = (lo + hi) >> 1;
                        if (ws.incl[mid] > e) { hi = mid; } else { lo = mid + 1; }
                    }
                    const int32_t excl = lo ? ws.incl[lo - 1] : 0;
                    src[i] = ws.u[lo];
                    v[i] = __ldg(&p.adj[ws.beg[lo] + (e - excl)]);
                }
            }
            td_claim_batch(p, acc, vis, qout, new_level, ok, v, src, loc);
        }
        __syncwarp();
    }
}

// Bottom-up step (hybrid_bfs.cc:111-143).  A warp works on K consecutive
// bitmap words (32 K vertices) at a time, so K independent load chains are
// in flight per lane.  Unvisited lanes scan their own neighbour lists (the
// first bu_prefix arcs, P arcs per word per round), stopping at the first
// visited neighbour; lists longer than that are finished by the whole warp,
// 32 arcs per ballot (warp-ballot early exit).  Reads only the frozen bitmap
// vis[cur]; writes whole words of vis[cur^1].
template <int BLOCK, int K>
__device__ void bu_step(const BfsParams &p, const StepView &sv, Local &loc)
{
    constexpr int P = K >= 4 ? 2 : 4;
    const int lane = lane_id();
    const int warp = threadIdx.x >> 5;
    const long long gw = (long long)blockIdx.x * (BLOCK / 32) + warp;
    const long long nw = (long long)gridDim.x * (BLOCK / 32);
    const uint32_t *vin = p.vis[sv.vis_cur];
    uint32_t *vout = p.vis[sv.vis_cur ^ 1];
    const int qout = sv.q_cur ^ 1;
    Acc *acc = &p.ctrl->acc[sv.step % 3];
    const int new_level = sv.level + 1;

    // Warp gw owns groups gw, gw + nw, gw + 2 nw, ... of K words.  It loads
    // 32 / K of its groups at once (one word per lane), passes full groups
    // through, and works only on the groups with unvisited vertices: late
    // levels, where most words are full, cost a bitmap sweep.
    constexpr int GPB = 32 / K;
    constexpr unsigned kGroupMask = (1u << K) - 1u;
    for (long long t0 = 0; (gw + t0 * nw) * K < p.words; t0 += GPB) {
        const int j = lane / K;
        const long long wl = (gw + (t0 + j) * nw) * K + lane % K;
        const uint32_t mw = wl < p.words ? __ldcg(&vin[wl]) : kFull;
        const unsigned openm = __ballot_sync(kFull, mw != kFull);
        if (!((openm >> (j * K)) & kGroupMask) && wl < p.words) { vout[wl] = kFull; }
        unsigned groups = 0;
#pragma unroll
        for (int g = 0; g < GPB; ++g) {
            if ((openm >> (g * K)) & kGroupMask) { groups |= 1u << g; }
        }
        while (groups) {
            const int g = __ffs(groups) - 1;
            groups &= groups - 1;
            const long long w0 = (gw + (t0 + g) * nw) * K;
            uint32_t word[K];
#pragma unroll
            for (int k = 0; k < K; ++k) { word[k] = __shfl_sync(kFull, mw, g * K + k); }
            uint32_t v[K], par[K];
            bool found[K], unv[K];
            int64_t beg[K], end[K], next[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                v[k] = (uint32_t)((w0 + k) * 32 + lane);
                unv[k] = !((word[k] >> lane) & 1u);
                found[k] = false;
                par[k] = 0;
                beg[k] = end[k] = next[k] = 0;
                if (unv[k]) {
                    beg[k] = __ldg(&p.off[v[k]]);
                    end[k] = __ldg(&p.off[v[k] + 1]);
                }
            }
            // per-lane scan of the first bu_prefix arcs, P arcs per word per round
            for (int r = 0; r < p.bu_prefix; r += P) {
                uint32_t x[K][P];
                bool in[K][P];
#pragma unroll
                for (int k = 0; k < K; ++k) {
#pragma unroll
                    for (int j = 0; j < P; ++j) {
                        const int64_t e = beg[k] + r + j;
                        in[k][j] = unv[k] && !found[k] && e < end[k];
                        x[k][j] = in[k][j] ? __ldg(&p.adj[e]) : 0u;
                    }
                }
                uint32_t bits[K][P];
#pragma unroll
                for (int k = 0; k < K; ++k) {
#pragma unroll
                    for (int j = 0; j < P; ++j) { bits[k][j] = in[k][j] ? ld_bits(&vin[x[k][j] >> 5]) : 0u; }
                }
                bool more = false;
#pragma unroll
                for (int k = 0; k < K; ++k) {
#pragma unroll
                    for (int j = 0; j < P; ++j) {
                        if (in[k][j] && !found[k] && ((bits[k][j] >> (x[k][j] & 31)) & 1u)) {
                            found[k] = true;
                            par[k] = x[k][j];
                        }
                    }
                    more |= unv[k] && !found[k] && beg[k] + r + P < end[k];
                }
                if (!__any_sync(kFull, more)) { break; }
            }
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int64_t lim = min(end[k], beg[k] + (int64_t)((p.bu_prefix + P - 1) / P * P));
                next[k] = found[k] ? end[k] : lim;
                unsigned pending = __ballot_sync(kFull, unv[k] && !found[k] && next[k] < end[k]);
                while (pending) {
                    const int owner = __ffs(pending) - 1;
                    pending &= pending - 1;
                    const int64_t b = __shfl_sync(kFull, next[k], owner);
                    const int64_t e = __shfl_sync(kFull, end[k], owner);
                    for (int64_t base = b; base < e; base += 32) {
                        const int64_t kk = base + lane;
                        bool hit = false;
                        uint32_t xx = 0;
                        if (kk < e) {
                            xx = __ldg(&p.adj[kk]);
                            hit = (ld_bits(&vin[xx >> 5]) >> (xx & 31)) & 1u;
                        }
                        const unsigned hm = __ballot_sync(kFull, hit);
                        if (hm) {
                            const uint32_t hx = __shfl_sync(kFull, xx, __ffs(hm) - 1);
                            if (lane == owner) {
                                found[k] = true;
                                par[k] = hx;
                            }
                            break;
                        }
                    }
                }
                const unsigned fm = __ballot_sync(kFull, found[k]);
                if (lane == 0 && w0 + k < p.words) { vout[w0 + k] = word[k] | fm; }
                if (found[k]) {
                    p.depth[v[k]] = new_level;
                    p.parent[v[k]] = (int64_t)par[k];
                }
            }
            int64_t deg[K];
#pragma unroll
            for (int k = 0; k < K; ++k) { deg[k] = end[k] - beg[k]; }
            warp_append_k<K>(p, acc, qout, found, v, deg, loc);
        }
    }
}

// Bottom-up step, lane-owned words (hybrid_bfs.cc:111-143).  Each lane owns
// one bitmap word (32 vertices) and walks its unvisited vertices on its own:
// a lane that finds a parent moves straight to its next vertex instead of
// waiting for the warp's slowest list.  P arcs are probed per iteration.
// Lists longer than kLongList are left to the whole warp (ballot scan) after
// the per-lane walk.  Reads only the frozen bitmap vis[cur]; writes whole
// words of vis[cur^1].
constexpr int64_t kLongList = 256;

template <int BLOCK>
__device__ void bu_step_lanes(const BfsParams &p, const StepView &sv, Local &loc)
{
    constexpr int P = 4;
    const int lane = lane_id();
    const int warp = threadIdx.x >> 5;
    const long long gw = (long long)blockIdx.x * (BLOCK / 32) + warp;
    const long long nw = (long long)gridDim.x * (BLOCK / 32);
    const uint32_t *vin = p.vis[sv.vis_cur];
    uint32_t *vout = p.vis[sv.vis_cur ^ 1];
    const int qout = sv.q_cur ^ 1;
    Acc *acc = &p.ctrl->acc[sv.step % 3];
    const int new_level = sv.level + 1;

    for (long long base = gw * 32; base < p.words; base += nw * 32) {
        const long long w = base + lane;
        const bool mine = w < p.words;
        const uint32_t word = mine ? __ldcg(&vin[w]) : kFull;
        uint32_t todo = ~word;     // unvisited vertices of this lane's word
        uint32_t found = 0;        // ... that found a parent
        uint32_t longs = 0;        // ... with lists left to the warp
        int64_t e = 0, end = 0;
        int cur = -1;
        unsigned long long degsum = 0;
        while (__any_sync(kFull, todo != 0 || cur >= 0)) {
            if (cur < 0 && todo) {
                cur = __ffs(todo) - 1;
                todo &= todo - 1;
                const uint32_t v = (uint32_t)(w * 32 + cur);
                e = __ldg(&p.off[v]);
                end = __ldg(&p.off[v + 1]);
                if (end - e > kLongList) {
                    longs |= 1u << cur;
                    cur = -1;
                }
            }
            if (cur >= 0) {
                uint32_t x[P], bits[P];
#pragma unroll
                for (int j = 0; j < P; ++j) { x[j] = (e + j < end) ? __ldg(&p.adj[e + j]) : 0u; }
#pragma unroll
                for (int j = 0; j < P; ++j) { bits[j] = (e + j < end) ? ld_bits(&vin[x[j] >> 5]) : 0u; }
                int hit = -1;
#pragma unroll
                for (int j = P - 1; j >= 0; --j) {
                    if ((e + j < end) && ((bits[j] >> (x[j] & 31)) & 1u)) { hit = j; }
                }
                if (hit >= 0) {
                    const uint32_t v = (uint32_t)(w * 32 + cur);
                    found |= 1u << cur;
                    p.depth[v] = new_level;
                    p.parent[v] = (int64_t)x[hit];
                    degsum += (unsigned long long)(end - __ldg(&p.off[v]));
                    cur = -1;
                } else {
                    e += P;
                    if (e >= end) { cur = -1; }
                }
            }
        }
        // long lists: the whole warp, one vertex at a time, 32 arcs a ballot
        unsigned owners = __ballot_sync(kFull, longs != 0);
        while (owners) {
            const int owner = __ffs(owners) - 1;
            uint32_t ol = __shfl_sync(kFull, longs, owner);
            const long long ow = __shfl_sync(kFull, w, owner);
            while (ol) {
                const int bit = __ffs(ol) - 1;
                ol &= ol - 1;
                const uint32_t v = (uint32_t)(ow * 32 + bit);
                const int64_t b = __ldg(&p.off[v]), en = __ldg(&p.off[v + 1]);
                for (int64_t kb = b; kb < en; kb += 32) {
                    const int64_t k = kb + lane;
                    bool hit = false;
                    uint32_t xx = 0;
                    if (k < en) {
                        xx = __ldg(&p.adj[k]);
                        hit = (ld_bits(&vin[xx >> 5]) >> (xx & 31)) & 1u;
                    }
                    const unsigned hm = __ballot_sync(kFull, hit);
                    if (hm) {
                        const uint32_t hx = __shfl_sync(kFull, xx, __ffs(hm) - 1);
                        if (lane == owner) {
                            found |= 1u << bit;
                            p.depth[v] = new_level;
                            p.parent[v] = (int64_t)hx;
                            degsum += (unsigned long long)(en - b);
                        }
                        break;
                    }
                }
            }
            owners &= owners - 1;
        }
        if (mine) { vout[w] = word | found; }
        // append this lane's discoveries: one atomic per warp for the small
        // ones, one per large vertex (rare)
        uint32_t small = 0, large = 0;
        for (uint32_t f = found; f; f &= f - 1) {
            const int bit = __ffs(f) - 1;
            const uint32_t v = (uint32_t)(w * 32 + bit);
            if (__ldg(&p.off[v + 1]) - __ldg(&p.off[v]) >= (int64_t)p.large_deg) {
                large |= 1u << bit;
            } else {
                small |= 1u << bit;
            }
        }
        const unsigned cnt = __popc(small);
        const unsigned incl = warp_incl_scan(cnt);
        const unsigned total = __shfl_sync(kFull, incl, 31);
        if (total) {
            unsigned long long start = 0;
            if (lane == 0) { start = atomicAdd(&acc->small_cnt, (unsigned long long)total); }
            start = __shfl_sync(kFull, start, 0) + (incl - cnt);
            for (uint32_t f = small; f; f &= f - 1) {
                p.qs[qout][start++] = (uint32_t)(w * 32 + (__ffs(f) - 1));
            }
        }
        if (__any_sync(kFull, large != 0)) {
            unsigned long long chunks = 0;
            for (uint32_t f = large; f; f &= f - 1) {
                const uint32_t v = (uint32_t)(w * 32 + (__ffs(f) - 1));
                const int64_t d = __ldg(&p.off[v + 1]) - __ldg(&p.off[v]);
                chunks += (unsigned long long)((d + p.chunk - 1) / p.chunk);
            }
            unsigned long long pos, cbase;
            warp_reserve_large(acc, __popc(large), chunks, pos, cbase);
            for (uint32_t f = large; f; f &= f - 1) {
                const uint32_t v = (uint32_t)(w * 32 + (__ffs(f) - 1));
                const int64_t d = __ldg(&p.off[v + 1]) - __ldg(&p.off[v]);
                p.ql[qout][pos] = v;
                p.qlb[qout][pos] = cbase;
                pos += 1;
                cbase += (unsigned long long)((d + p.chunk - 1) / p.chunk);
            }
        }
        loc.found += __popc(found);
        loc.degsum += degsum;
    }
}

// Beamer's rule (hybrid_bfs.cc:152-191) for the step about to run, given the
// frontier in the state.  Updates the Beamer state like the reference loop
// does when it commits to that direction.
__device__ int beamer_choose(LevelState &c, const BfsParams &p, bool commit)
{
    if (c.in_bu) { return kDirBU; }
    if (c.scout > c.etc / p.alpha) {
        if (commit) {
            c.in_bu = 1;
            c.awake = c.f_count;  // queue_.combined_size()
        }
        return kDirBU;
    }
    if (commit) { c.etc -= c.scout; }
    return kDirTD;
}

// After a step of direction `dir` found `found` vertices of degree sum
// `degsum`: the reference's bookkeeping (scout after top-down, the awake
// test of the bottom-up do-while, scout = 1 on leaving it).
__device__ void beamer_after_step(LevelState &c, const BfsParams &p, int dir, long long found,
                                  long long degsum)
{
    if (dir == kDirTD) {
        c.scout = degsum;
    } else if (c.in_bu) {
        c.old_awake = c.awake;
        c.awake = found;
        if (!(c.awake >= c.old_awake || c.awake > p.n / p.beta)) {
            c.in_bu = 0;
            c.scout = 1;
        }
    }
}

// Whether the learned policy is consulted for the step after state c: it is
// installed, the BFS goes on, and the frontier's degree sum over the
// unexplored one lies in the band the policy was trained to decide in
// (outside it the rule decides and the network is not run).
__device__ __forceinline__ bool policy_applies(const LevelState &c, const BfsParams &p)
{
    return p.alg == BD_ALG_LEARNED && p.policy != nullptr && c.f_count != 0 &&
           policy_in_band(p.policy, c.f_degsum, 2 * p.m - c.visited_degsum);
}

// The rule's direction for the next step (committed into the Beamer state
// unless the learned policy will decide).  One thread.
__device__ int rule_direction(LevelState &c, const BfsParams &p)
{
    if (c.f_count == 0) { return kDirDone; }
    if (p.alg == BD_ALG_TOP_DOWN) { return kDirTD; }
    if (p.alg == BD_ALG_BOTTOM_UP) { return kDirBU; }
    return beamer_choose(c, p, !policy_applies(c, p));
}

// The learned policy's pick over the rule's (NaN gap: a feature outside the
// trusted range, the rule decides); keeps the rule's state consistent with
// the step actually taken.  One thread.
__device__ int apply_policy(LevelState &c, const PolicyBlob *w, int rule, float gap)
{
    int d = rule;
    if (isfinite(gap) && fabsf(gap) >= w->margin) { d = gap > 0.f ? kDirBU : kDirTD; }
    if (d != rule) { c.policy_overrides += 1; }
    if (d == kDirTD) {
        c.in_bu = 0;
        c.etc -= c.scout;
    } else if (!c.in_bu) {
        c.in_bu = 1;
        c.awake = c.f_count;
    }
    return d;
}

// Picks c.dir for the next step: thread 0 applies the rule, warp 0 runs the
// policy network from w (shared or global memory) where it applies.  Called
// by every thread of the block.
template <typename Shared>
__device__ void decide_next(LevelState &c, const BfsParams &p, const PolicyBlob *w, Shared &sh)
{
    if (threadIdx.x == 0) { sh.rule_dir = rule_direction(c, p); }
    __syncthreads();
    if (!policy_applies(c, p)) {
        if (threadIdx.x == 0) { c.dir = sh.rule_dir; }
        return;
    }
    if (threadIdx.x < 32) {
        const float gap = policy_gap_warp(w, c.f_count, c.f_degsum, 2 * p.m - c.visited_degsum,
                                          c.level, p.n, p.m, c.prev_dir, c.prev_ns);
        if (threadIdx.x == 0) { c.dir = apply_policy(c, w, sh.rule_dir, gap); }
    }
}

// Advances the state over the step that just ended, from that step's
// counters a and its end time.  One thread per CTA; every CTA computes the
// same result.
__device__ void advance(LevelState &c, const BfsParams &p, const Acc &a, long long t_end)
{
    const long long found = (long long)a.found;
    const long long degsum = (long long)a.degsum;
    const unsigned long long lp = a.large_packed;
    const long long ns = t_end - c.t_last;
    const int dir = c.dir;
    c.visited_degsum += degsum;
    c.reached += found;
    // once fewer than half of the live vertices are unvisited, bottom-up
    // work per bitmap word is sparse: switch to the lane-owned layout
    c.bu_sparse = 2 * (p.n_live - c.reached) < p.n_live;
    c.f_count = found;
    c.f_degsum = degsum;
    c.f_small = (long long)a.small_cnt;
    c.f_large = (long long)(lp >> kLargeShift);
    c.f_chunks = (long long)(lp & kChunkMask);
    c.prev_dir = dir;
    c.prev_ns = ns;
    c.t_last = t_end;
    if (dir == kDirTD) { c.td_steps += 1; } else { c.bu_steps += 1; }
    c.level += 1;
    c.q_cur ^= 1;
    if (dir == kDirBU) { c.vis_cur ^= 1; }
    beamer_after_step(c, p, dir, found, degsum);
    c.step += 1;
}

// The end of a step: block reduction of the counters, arrival at the grid
// barrier (one release-add per CTA), acquire polling until every CTA has
// arrived, then every CTA advances its copy of the state from the step's
// counters and decides the next direction.  Every wait is bounded by
// p.spin_limit polls; running out sets ctrl->error = BD_ERR_TIMEOUT and ends
// this CTA's loop.
template <int BLOCK>
__device__ void end_step(const BfsParams &p, const StepView &sv, SharedState<BLOCK> &sh,
                         Local &loc)
{
    Ctrl *c = p.ctrl;
    const int lane = lane_id();
    const int warp = threadIdx.x >> 5;
    const unsigned long long f = warp_sum(loc.found);
    const unsigned long long d = warp_sum(loc.degsum);
    if (lane == 0) {
        sh.red_found[warp] = f;
        sh.red_deg[warp] = d;
    }
    loc.found = 0;
    loc.degsum = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long tf = 0, td = 0;
        for (int i = 0; i < BLOCK / 32; ++i) {
            tf += sh.red_found[i];
            td += sh.red_deg[i];
        }
        const int s = sv.step;
        Acc *acc = &c->acc[s % 3];
        if (tf) { atomicAdd(&acc->found, tf); }
        if (td) { atomicAdd(&acc->degsum, td); }
        if (blockIdx.x == 0) {
            Acc *z = &c->acc[(s + 1) % 3];
            z->found = z->degsum = z->small_cnt = z->large_packed = z->t_end = 0;
        }
        atomicMax(&acc->t_end, (unsigned long long)globaltimer());
        red_release_add64(&c->bar, 1ull);
        const unsigned long long target = (unsigned long long)(s + 1) * p.expected_ctas;
        long long it = 0;
        bool ok = true;
        while (ld_acquire64(&c->bar) < target) {
            if (++it > p.spin_limit) {
                atomicExch(&c->error, (int)BD_ERR_TIMEOUT);
                ok = false;
                break;
            }
            __nanosleep(32);
        }
        if (ok && __ldcg(&c->error) == 0) {
            Acc a;
            a.found = __ldcg(&acc->found);
            a.degsum = __ldcg(&acc->degsum);
            a.small_cnt = __ldcg(&acc->small_cnt);
            a.large_packed = __ldcg(&acc->large_packed);
            const long long t_end = (long long)__ldcg(&acc->t_end);
            LevelState &st = sh.st;
            if (s == 0) { st.t_last = (long long)__ldcg(&c->t_start); }
            if (blockIdx.x == 0 && s < p.rec_cap) {
                bd_step r;
                r.dir = st.dir;
                r.level = st.level;
                r.frontier = st.f_count;
                r.frontier_edges = st.f_degsum;
                r.unexplored_edges = 2 * p.m - st.visited_degsum;
                r.found = (long long)a.found;
                r.ns = t_end - st.t_last;
                p.rec[s] = r;
            }
            advance(st, p, a, t_end);
        } else {
            sh.st.f_count = 0;  // leave the loop
        }
    }
    __syncthreads();
    decide_next(sh.st, p, &sh.pol, sh);
    __syncthreads();
}

// K bitmap words per warp step: 1, 2, 4 (warp-shared words) or 32 (one word
// per lane).
template <int BLOCK, int K>
__device__ __forceinline__ void bu_layout(const BfsParams &p, const StepView &sv, Local &loc)
{
    if constexpr (K == 32) {
        bu_step_lanes<BLOCK>(p, sv, loc);
    } else {
        bu_step<BLOCK, K>(p, sv, loc);
    }
}

// KD: bottom-up layout while most live vertices are unvisited; KS: after.
template <int BLOCK, int MINB, int KD, int KS>
__global__ void __launch_bounds__(BLOCK, MINB) bfs_persistent_kernel(BfsParams p)
{
    __shared__ SharedState<BLOCK> sh;
    Ctrl *c = p.ctrl;
    if (threadIdx.x == 0) {
        sh.st = c->st;  // written by the init kernel before this launch
        atomicMin(&c->t_start, (unsigned long long)globaltimer());
    }
    if (p.policy) {
        const float *src = reinterpret_cast<const float *>(p.policy);
        float *dst = reinterpret_cast<float *>(&sh.pol);
        for (int i = threadIdx.x; i < (int)(sizeof(PolicyBlob) / sizeof(float)); i += BLOCK) {
            dst[i] = src[i];
        }
    }
    __syncthreads();
    Local loc{0, 0};
    while (sh.st.dir != kDirDone) {
        const StepView sv = view_of(sh.st);
        if (sv.dir == kDirTD) {
            td_step<BLOCK>(p, sv, sh, loc);
        } else {
            if (sv.bu_sparse) {
                bu_layout<BLOCK, KS>(p, sv, loc);
            } else {
                bu_layout<BLOCK, KD>(p, sv, loc);
            }
        }
        end_step<BLOCK>(p, sv, sh, loc);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { c->st = sh.st; }
}

struct InitShared {
    int rule_dir;
    LevelState st;
};

// clear() + the source frontier (hybrid_bfs.cc:152-160 for one source; any
// number of sources start as one frontier), and the first decision.  One
// CTA of 32 threads.
__global__ void init_sources_kernel(BfsParams p, const int64_t *sources, int64_t count,
                                    int64_t source_index)
{
    __shared__ InitShared sh;
    Ctrl *c = p.ctrl;
    if (threadIdx.x == 0) {
        memset(c, 0, sizeof(Ctrl));
        c->t_start = ~0ull;
        LevelState &st = sh.st;
        memset(&st, 0, sizeof(LevelState));
        long long degsum = 0, nf = 0, nsmall = 0;
        unsigned long long lp = 0;
        const int64_t first = source_index >= 0 ? source_index : 0;
        const int64_t last = source_index >= 0 ? source_index + 1 : count;
        for (int64_t i = first; i < last; ++i) {
            const uint32_t s = p.perm ? p.perm[sources[i]] : (uint32_t)sources[i];
            if (p.depth[s] == 0) { continue; }  // repeated source
            p.depth[s] = 0;
            p.parent[s] = (int64_t)s;
            p.vis[0][s >> 5] |= 1u << (s & 31);
            const int64_t deg = p.off[s + 1] - p.off[s];
            degsum += deg;
            nf += 1;
            if (deg >= (int64_t)p.large_deg) {
                const unsigned long long pos = lp >> kLargeShift;
                p.ql[0][pos] = s;
                p.qlb[0][pos] = lp & kChunkMask;
                lp += (1ull << kLargeShift) | (unsigned long long)((deg + p.chunk - 1) / p.chunk);
            } else {
                p.qs[0][nsmall++] = s;
            }
        }
        st.f_count = nf;
        st.f_degsum = degsum;
        st.f_small = nsmall;
        st.f_large = (long long)(lp >> kLargeShift);
        st.f_chunks = (long long)(lp & kChunkMask);
        st.visited_degsum = degsum;
        st.reached = nf;
        st.etc = 2 * p.m;       // edges_to_check = num_edges * 2
        st.scout = degsum;      // scout_count = out_degree(source)
        st.prev_dir = kDirTD;
    }
    __syncthreads();
    decide_next(sh.st, p, p.policy, sh);
    __syncthreads();
    if (threadIdx.x == 0) { c->st = sh.st; }
}

// Deterministic tree: parent(v) = min{u in N(v) : depth[u] == depth[v]-1}.
// Warp per 32 vertices; short lists per lane, long lists by the whole warp.
__global__ void min_parent_kernel(const int64_t *off, const uint32_t *adj, int64_t n,
                                  const int32_t *depth, int64_t *parent)
{
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long words = (n + 31) / 32;
    for (long long w = gw; w < words; w += nw) {
        const int64_t v = w * 32 + lane;
        int32_t dv = v < n ? depth[v] : -1;
        int64_t b = 0, e = 0;
        uint32_t best = 0xFFFFFFFFu;
        const bool want = dv > 0;
        if (want) {
            b = off[v];
            e = off[v + 1];
            if (e - b <= 32) {
                for (int64_t k = b; k < e; ++k) {
                    uint32_t u = adj[k];
                    if (u < best && depth[u] == dv - 1) { best = u; }
                }
            }
        }
        unsigned big = __ballot_sync(kFull, want && e - b > 32);
        while (big) {
            const int owner = __ffs(big) - 1;
            big &= big - 1;
            const int64_t bb = __shfl_sync(kFull, b, owner);
            const int64_t ee = __shfl_sync(kFull, e, owner);
            const int32_t d = __shfl_sync(kFull, dv, owner);
            uint32_t mine = 0xFFFFFFFFu;
            for (int64_t k = bb + lane; k < ee; k += 32) {
                uint32_t u = adj[k];
                if (u < mine && depth[u] == d - 1) { mine = u; }
            }
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) { mine = min(mine, __shfl_xor_sync(kFull, mine, s)); }
            if (lane == owner) { best = mine; }
        }
        if (want) { parent[v] = (int64_t)best; }
    }
}

// The reference's encoding of unreached vertices (hybrid_bfs.cc:433-443).
__global__ void finalize_parents_kernel(const int64_t *off, int64_t n, const int32_t *depth,
                                        int64_t *parent)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (depth[v] < 0) {
            const int64_t d = off[v + 1] - off[v];
            parent[v] = d != 0 ? -d : -1;
        }
    }
}

// BD_ORDER_HUB: depths and parents in the caller's numbering (traversal
// arrays are indexed, and parents named, by traversal id), with the
// reference's encoding of unreached vertices.
__global__ void hub_outputs_kernel(const uint32_t *perm, const uint32_t *iperm, const int64_t *off,
                                   int64_t n, const int32_t *depth, const int64_t *parent,
                                   int32_t *out_depth, int64_t *out_parent)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t t = perm[v];
        const int32_t d = depth[t];
        out_depth[v] = d;
        if (d >= 0) {
            out_parent[v] = (int64_t)iperm[parent[t]];
        } else {
            const int64_t deg = off[v + 1] - off[v];
            out_parent[v] = deg != 0 ? -deg : -1;
        }
    }
}

__global__ void save_result_kernel(const Ctrl *c, int64_t *out, int64_t i)
{
    out[2 * i] = c->st.visited_degsum / 2;
    out[2 * i + 1] = c->st.reached;
}

int grid_for(int64_t items, int threads = 256)
{
    int64_t b = (items + threads - 1) / threads;
    if (b < 1) { b = 1; }
    if (b > 148 * 32) { b = 148 * 32; }
    return (int)b;
}

using KernelFn = void (*)(BfsParams);

struct KernelChoice {
    KernelFn fn;
    int block;
};

KernelChoice pick_kernel(int block, int kd = 4, int ks = 4)
{
#define BD_KC(B, M, D, S) \
    if (block == B && kd == D && ks == S) { return {bfs_persistent_kernel<B, M, D, S>, B}; }
#define BD_KC_B(B, M)                                                                  \
    BD_KC(B, M, 1, 1) BD_KC(B, M, 2, 2) BD_KC(B, M, 4, 4) BD_KC(B, M, 32, 32)          \
    BD_KC(B, M, 2, 32) BD_KC(B, M, 4, 32)
    BD_KC_B(256, 4) BD_KC_B(512, 2) BD_KC_B(1024, 1)
#undef BD_KC_B
#undef BD_KC
    return {nullptr, 0};
}

}  // namespace

}  // namespace bd

using namespace bd;

struct bd_bfs {
    bd_graph *g = nullptr;
    bd_bfs_opts opts{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int32_t *depth = nullptr;
    int64_t *parent = nullptr;
    uint32_t *vis[2] = {nullptr, nullptr};
    uint32_t *qs[2] = {nullptr, nullptr};
    uint32_t *ql[2] = {nullptr, nullptr};
    unsigned long long *qlb[2] = {nullptr, nullptr};
    Ctrl *ctrl = nullptr;
    bd_step *rec = nullptr;
    int64_t *d_sources = nullptr;
    int64_t sources_cap = 0;
    PolicyBlob *policy = nullptr;  // device copy, or null
    KernelFn kernel = nullptr;
    int block = 512;
    int grid = 0;
    int64_t cap_large = 0;
    // BD_ORDER_HUB graphs: depths and parents in the caller's numbering,
    // filled from the traversal arrays when first read after a run
    int32_t *out_depth = nullptr;
    int64_t *out_parent = nullptr;
    bool cleared = false;
    bool ran = false;
    bool parents_final = false;  // caller-visible depths and parents are up to date
    int64_t last_source = -1;
    Ctrl last{};
};

namespace bd {

bd_status bfs_install_policy(bd_bfs *b, const PolicyBlob *blob)
{
    BD_CUDA(cudaSetDevice(b->device));
    if (!blob) {
        cudaFree(b->policy);
        b->policy = nullptr;
        return BD_OK;
    }
    if (!b->policy) { BD_CUDA(cudaMalloc(&b->policy, sizeof(PolicyBlob))); }
    BD_CUDA(cudaMemcpy(b->policy, blob, sizeof(PolicyBlob), cudaMemcpyHostToDevice));
    return BD_OK;
}

namespace {

BfsParams make_params(bd_bfs *b)
{
    BfsParams p{};
    p.off = traversal_off(b->g);
    p.adj = traversal_adj(b->g);
    p.n = b->g->n;
    p.m = b->g->m;
    p.depth = b->depth;
    p.parent = b->parent;
    p.vis[0] = b->vis[0];
    p.vis[1] = b->vis[1];
    p.words = bitmap_words(b->g->n);
    p.n_live = b->g->n_live;
    for (int i = 0; i < 2; ++i) {
        p.qs[i] = b->qs[i];
        p.ql[i] = b->ql[i];
        p.qlb[i] = b->qlb[i];
    }
    p.ctrl = b->ctrl;
    p.rec = b->rec;
    p.rec_cap = kRecCap;
    p.alg = b->opts.alg;
    p.alpha = b->opts.alpha;
    p.beta = b->opts.beta;
    p.large_deg = (uint32_t)b->opts.large_degree;
    p.chunk = (uint32_t)b->opts.chunk_edges;
    p.bu_prefix = b->opts.bu_prefix;
    p.spin_limit = b->opts.spin_limit;
    p.expected_ctas = (unsigned)(b->grid + b->opts.test_extra_ctas);
    p.policy = b->policy;
    p.perm = b->g->d_perm;
    return p;
}

bd_status enqueue_clear(bd_bfs *b)
{
    const int64_t n = b->g->n;
    BD_CUDA(cudaMemsetAsync(b->depth, 0xFF, sizeof(int32_t) * n, b->stream));
    BD_CUDA(cudaMemcpyAsync(b->vis[0], traversal_isolated(b->g),
                            sizeof(uint32_t) * bitmap_words(n), cudaMemcpyDeviceToDevice,
                            b->stream));
    return BD_OK;
}

bd_status ensure_sources(bd_bfs *b, int64_t count)
{
    if (count <= b->sources_cap) { return BD_OK; }
    cudaFree(b->d_sources);
    b->d_sources = nullptr;
    b->sources_cap = 0;
    BD_CUDA(cudaMalloc(&b->d_sources, sizeof(int64_t) * count));
    b->sources_cap = count;
    return BD_OK;
}

// Depths and parents in the caller's arrays with the reference's encoding
// of unreached vertices (graphs without a hub numbering: the same ids).
__global__ void copy_outputs_kernel(const int64_t *off, int64_t n, const int32_t *depth,
                                    const int64_t *parent, int32_t *out_depth, int64_t *out_parent)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = depth[v];
        out_depth[v] = d;
        if (d >= 0) {
            out_parent[v] = parent[v];
        } else {
            const int64_t deg = off[v + 1] - off[v];
            out_parent[v] = deg != 0 ? -deg : -1;
        }
    }
}

// Enqueues init + the persistent kernel (+ min-parent pass) for either a
// set of sources (index < 0) or source d_sources[index].  With out_depth /
// out_parent (device, n entries each) the results are also written there
// in the caller's ids and the reference's encoding, inside the timed region.
bd_status enqueue_bfs(bd_bfs *b, int64_t count, int64_t index, cudaEvent_t start,
                      cudaEvent_t stop, int32_t *out_depth = nullptr,
                      int64_t *out_parent = nullptr)
{
    BfsParams p = make_params(b);
    // The timed region starts with the source setup, as run_beamer's does
    // (hybrid_bfs.cc:158-160); clear() stays outside it.
    if (start) { BD_CUDA(cudaEventRecord(start, b->stream)); }
    init_sources_kernel<<<1, 32, 0, b->stream>>>(p, b->d_sources, count, index);
    BD_CUDA(cudaGetLastError());
    void *args[] = {&p};
    BD_CUDA(cudaLaunchCooperativeKernel((const void *)b->kernel, dim3(b->grid), dim3(b->block),
                                        args, 0, b->stream));
    if (out_depth) {
        const int64_t n = b->g->n;
        if (b->g->d_perm) {
            hub_outputs_kernel<<<grid_for(n), 256, 0, b->stream>>>(
                b->g->d_perm, b->g->d_iperm, b->g->d_off, n, b->depth, b->parent, out_depth,
                out_parent);
        } else {
            copy_outputs_kernel<<<grid_for(n), 256, 0, b->stream>>>(b->g->d_off, n, b->depth,
                                                                   b->parent, out_depth, out_parent);
        }
        BD_CUDA(cudaGetLastError());
        if (b->opts.min_parent) {
            min_parent_kernel<<<grid_for(bitmap_words(n) * 32), 256, 0, b->stream>>>(
                b->g->d_off, b->g->d_adj, n, out_depth, out_parent);
            BD_CUDA(cudaGetLastError());
        }
    } else if (b->opts.min_parent) {
        // the smallest parent in the caller's numbering: on a hub graph, map
        // the outputs back first, then pick parents on the caller's CSR
        const int64_t n = b->g->n;
        int32_t *depth = b->depth;
        int64_t *parent = b->parent;
        if (b->out_depth) {
            hub_outputs_kernel<<<grid_for(n), 256, 0, b->stream>>>(
                b->g->d_perm, b->g->d_iperm, b->g->d_off, n, b->depth, b->parent, b->out_depth,
                b->out_parent);
            BD_CUDA(cudaGetLastError());
            depth = b->out_depth;
            parent = b->out_parent;
        }
        min_parent_kernel<<<grid_for(bitmap_words(n) * 32), 256, 0, b->stream>>>(
            b->g->d_off, b->g->d_adj, n, depth, parent);
        BD_CUDA(cudaGetLastError());
    }
    if (stop) { BD_CUDA(cudaEventRecord(stop, b->stream)); }
    return BD_OK;
}

bd_status collect(bd_bfs *b, bd_run_stats *stats, double ms)
{
    BD_CUDA(cudaMemcpyAsync(&b->last, b->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, b->stream));
    BD_CUDA(cudaStreamSynchronize(b->stream));
    b->ran = true;
    b->cleared = false;
    // a min-parent run on a hub graph wrote the caller-order outputs itself
    b->parents_final = b->out_depth != nullptr && b->opts.min_parent;
    if (b->last.error) { return (bd_status)b->last.error; }
    if (stats) {
        stats->ms = ms;
        stats->num_steps = b->last.st.step;
        stats->reached = b->last.st.reached;
        stats->traversed_edges = b->last.st.visited_degsum / 2;
        stats->top_down_steps = b->last.st.td_steps;
        stats->bottom_up_steps = b->last.st.bu_steps;
    }
    return BD_OK;
}

bd_status run_sources(bd_bfs *b, const int64_t *sources, int64_t count, bd_run_stats *stats)
{
    if (!b || !sources || count <= 0) { return BD_ERR_INVALID; }
    for (int64_t i = 0; i < count; ++i) {
        if (sources[i] < 0 || sources[i] >= b->g->n) { return BD_ERR_RANGE; }
    }
    BD_CUDA(cudaSetDevice(b->device));
    BD_TRY(ensure_sources(b, count));
    if (!b->cleared) { BD_TRY(enqueue_clear(b)); }
    BD_CUDA(cudaMemcpyAsync(b->d_sources, sources, sizeof(int64_t) * count,
                            cudaMemcpyHostToDevice, b->stream));
    BD_TRY(enqueue_bfs(b, count, -1, b->ev0, b->ev1));
    BD_CUDA(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    BD_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_source = count == 1 ? sources[0] : -1;
    return collect(b, stats, (double)ms);
}

// Makes the caller-visible depths and parents current: the reference's
// -deg / -1 encoding of unreached vertices, and on a hub graph the mapping
// back to the caller's numbering.
bd_status finalize_parents(bd_bfs *b)
{
    if (!b->ran) { return BD_ERR_STATE; }
    if (b->parents_final) { return BD_OK; }
    const int64_t n = b->g->n;
    if (b->out_depth) {
        hub_outputs_kernel<<<grid_for(n), 256, 0, b->stream>>>(
            b->g->d_perm, b->g->d_iperm, b->g->d_off, n, b->depth, b->parent, b->out_depth,
            b->out_parent);
    } else {
        finalize_parents_kernel<<<grid_for(n), 256, 0, b->stream>>>(b->g->d_off, n, b->depth,
                                                                  b->parent);
    }
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaStreamSynchronize(b->stream));
    b->parents_final = true;
    return BD_OK;
}

void bfs_free(bd_bfs *b)
{
    if (!b) { return; }
    cudaSetDevice(b->device);
    if (b->stream) { cudaStreamSynchronize(b->stream); }
    cudaFree(b->depth);
    cudaFree(b->parent);
    cudaFree(b->out_depth);
    cudaFree(b->out_parent);
    for (int i = 0; i < 2; ++i) {
        cudaFree(b->vis[i]);
        cudaFree(b->qs[i]);
        cudaFree(b->ql[i]);
        cudaFree(b->qlb[i]);
    }
    cudaFree(b->ctrl);
    cudaFree(b->rec);
    cudaFree(b->d_sources);
    cudaFree(b->policy);
    if (b->ev0) { cudaEventDestroy(b->ev0); }
    if (b->ev1) { cudaEventDestroy(b->ev1); }
    if (b->stream) { cudaStreamDestroy(b->stream); }
    delete b;
}

}  // namespace

cudaError_t launch_min_parent(const int64_t *off, const uint32_t *adj, int64_t n,
                              const int32_t *depth, int64_t *parent, cudaStream_t s)
{
    min_parent_kernel<<<grid_for(bitmap_words(n) * 32), 256, 0, s>>>(off, adj, n, depth, parent);
    return cudaGetLastError();
}

}  // namespace bd

extern "C" {

void bd_bfs_default_opts(bd_bfs_opts *o)
{
    if (!o) { return; }
    memset(o, 0, sizeof(*o));
    o->alg = BD_ALG_BEAMER;
    o->alpha = 15;
    o->beta = 18;
}

bd_status bd_bfs_create(bd_graph *g, const bd_bfs_opts *opts, bd_bfs **out)
{
    if (!g || !out) { return BD_ERR_INVALID; }
    bd_bfs_opts o;
    bd_bfs_default_opts(&o);
    if (opts) { o = *opts; }
    if (o.alg < BD_ALG_BEAMER || o.alg > BD_ALG_LEARNED || o.alpha <= 0 || o.beta <= 0) {
        return BD_ERR_INVALID;
    }
    if (o.block_size == 0) { o.block_size = 512; }
    if (o.block_size != 256 && o.block_size != 512 && o.block_size != 1024) { return BD_ERR_INVALID; }
    if (o.bu_words == 0) { o.bu_words = 4; }
    if (o.bu_sparse_words == 0) { o.bu_sparse_words = o.bu_words == 1 ? 1 : 32; }
    if (o.large_degree <= 0) { o.large_degree = 32; }
    if (o.large_degree > (1 << 20)) { return BD_ERR_INVALID; }
    if (o.chunk_edges <= 0) { o.chunk_edges = 256; }
    if (o.bu_prefix <= 0) { o.bu_prefix = 32; }
    if (o.spin_limit <= 0) { o.spin_limit = kDefaultSpin; }
    if (o.test_extra_ctas < 0) { return BD_ERR_INVALID; }
    BD_TRY(ensure_device());
    auto *b = new bd_bfs();
    b->g = g;
    b->opts = o;
    b->device = current_device();
    const int64_t n = g->n;
    const int64_t words = bitmap_words(n);
    b->cap_large = std::min<int64_t>(n, g->arcs / o.large_degree + 1);
    auto fail = [&](bd_status st) { bfs_free(b); return st; };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
        return fail(BD_ERR_CUDA);
    }
    bool ok = cudaMalloc(&b->depth, sizeof(int32_t) * n) == cudaSuccess &&
              cudaMalloc(&b->parent, sizeof(int64_t) * n) == cudaSuccess &&
              (!g->d_perm || (cudaMalloc(&b->out_depth, sizeof(int32_t) * n) == cudaSuccess &&
                              cudaMalloc(&b->out_parent, sizeof(int64_t) * n) == cudaSuccess)) &&
              cudaMalloc(&b->ctrl, sizeof(Ctrl)) == cudaSuccess &&
              cudaMalloc(&b->rec, sizeof(bd_step) * kRecCap) == cudaSuccess;
    for (int i = 0; i < 2 && ok; ++i) {
        ok = cudaMalloc(&b->vis[i], sizeof(uint32_t) * words) == cudaSuccess &&
             cudaMalloc(&b->qs[i], sizeof(uint32_t) * n) == cudaSuccess &&
             cudaMalloc(&b->ql[i], sizeof(uint32_t) * b->cap_large) == cudaSuccess &&
             cudaMalloc(&b->qlb[i], sizeof(unsigned long long) * b->cap_large) == cudaSuccess;
    }
    if (!ok) { return fail(BD_ERR_OOM); }
    KernelChoice kc = pick_kernel(o.block_size, o.bu_words, o.bu_sparse_words);
    if (!kc.fn) { return fail(BD_ERR_INVALID); }
    b->kernel = kc.fn;
    b->block = kc.block;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)b->kernel, b->block, 0) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ||
        per_sm < 1) {
        return fail(BD_ERR_CUDA);
    }
    b->grid = per_sm * sms;
    *out = b;
    return BD_OK;
}

bd_status bd_bfs_clear(bd_bfs *b)
{
    if (!b) { return BD_ERR_INVALID; }
    BD_CUDA(cudaSetDevice(b->device));
    BD_TRY(enqueue_clear(b));
    BD_CUDA(cudaStreamSynchronize(b->stream));
    b->cleared = true;
    b->ran = false;
    return BD_OK;
}

bd_status bd_bfs_run(bd_bfs *b, int64_t source, bd_run_stats *stats)
{
    return run_sources(b, &source, 1, stats);
}

bd_status bd_bfs_run_multi(bd_bfs *b, const int64_t *sources, int64_t count, bd_run_stats *stats)
{
    return run_sources(b, sources, count, stats);
}

static bd_status run_with_alg(bd_bfs *b, int alg, int64_t alpha, int64_t beta, int64_t source,
                              bd_run_stats *stats)
{
    if (!b) { return BD_ERR_INVALID; }
    if (alpha <= 0 || beta <= 0) { return BD_ERR_INVALID; }
    bd_bfs_opts saved = b->opts;
    b->opts.alg = alg;
    b->opts.alpha = alpha;
    b->opts.beta = beta;
    bd_status st = run_sources(b, &source, 1, stats);
    b->opts = saved;
    return st;
}

bd_status bd_bfs_run_beamer(bd_bfs *b, int64_t source, int64_t alpha, int64_t beta,
                            bd_run_stats *stats)
{
    return run_with_alg(b, BD_ALG_BEAMER, alpha, beta, source, stats);
}

bd_status bd_bfs_run_top_down(bd_bfs *b, int64_t source, bd_run_stats *stats)
{
    if (!b) { return BD_ERR_INVALID; }
    return run_with_alg(b, BD_ALG_TOP_DOWN, b->opts.alpha, b->opts.beta, source, stats);
}

bd_status bd_bfs_run_bottom_up(bd_bfs *b, int64_t source, bd_run_stats *stats)
{
    if (!b) { return BD_ERR_INVALID; }
    return run_with_alg(b, BD_ALG_BOTTOM_UP, b->opts.alpha, b->opts.beta, source, stats);
}

}  // extern "C"

namespace bd {
namespace {

bd_status run_many(bd_bfs *b, const int64_t *sources, int64_t k, int32_t *d_depth,
                   int64_t *d_parent, double *ms_out, int64_t *edges_out, int64_t *reached_out,
                   double *e2e_ms)
{
    if (!b || !sources || k <= 0) { return BD_ERR_INVALID; }
    for (int64_t i = 0; i < k; ++i) {
        if (sources[i] < 0 || sources[i] >= b->g->n) { return BD_ERR_RANGE; }
    }
    BD_CUDA(cudaSetDevice(b->device));
    BD_TRY(ensure_sources(b, k));
    int64_t *d_edges = nullptr;
    std::vector<cudaEvent_t> ev(2 * k, nullptr);
    bd_status st = BD_OK;
    cudaEvent_t wall0 = nullptr, wall1 = nullptr;
    auto cleanup = [&]() {
        for (auto e : ev) { if (e) { cudaEventDestroy(e); } }
        if (wall0) { cudaEventDestroy(wall0); }
        if (wall1) { cudaEventDestroy(wall1); }
        cudaFree(d_edges);
    };
    if (cudaMalloc(&d_edges, sizeof(int64_t) * 2 * k) != cudaSuccess ||
        cudaEventCreate(&wall0) != cudaSuccess || cudaEventCreate(&wall1) != cudaSuccess) {
        cleanup();
        return BD_ERR_OOM;
    }
    for (auto &e : ev) {
        if (cudaEventCreate(&e) != cudaSuccess) { cleanup(); return BD_ERR_CUDA; }
    }
    std::vector<int64_t> host_edges(2 * k);
    cudaEventRecord(wall0, b->stream);
    if (cudaMemcpyAsync(b->d_sources, sources, sizeof(int64_t) * k, cudaMemcpyHostToDevice,
                        b->stream) != cudaSuccess) {
        cleanup();
        return BD_ERR_CUDA;
    }
    const int64_t n = b->g->n;
    for (int64_t i = 0; i < k && st == BD_OK; ++i) {
        st = enqueue_clear(b);
        if (st == BD_OK) {
            st = enqueue_bfs(b, k, i, ev[2 * i], ev[2 * i + 1], d_depth ? d_depth + i * n : nullptr,
                             d_depth ? d_parent + i * n : nullptr);
        }
        if (st == BD_OK) {
            save_result_kernel<<<1, 1, 0, b->stream>>>(b->ctrl, d_edges, i);
            if (cudaGetLastError() != cudaSuccess) { st = BD_ERR_CUDA; }
        }
    }
    if (st == BD_OK &&
        (cudaMemcpyAsync(host_edges.data(), d_edges, sizeof(int64_t) * 2 * k, cudaMemcpyDeviceToHost,
                         b->stream) != cudaSuccess ||
         cudaEventRecord(wall1, b->stream) != cudaSuccess ||
         cudaStreamSynchronize(b->stream) != cudaSuccess)) {
        st = BD_ERR_CUDA;
    }
    if (st == BD_OK) {
        float w = 0.f;
        cudaEventElapsedTime(&w, wall0, wall1);
        if (e2e_ms) { *e2e_ms = (double)w; }
        for (int64_t i = 0; i < k; ++i) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
            if (ms_out) { ms_out[i] = (double)ms; }
            if (edges_out) { edges_out[i] = host_edges[2 * i]; }
            if (reached_out) { reached_out[i] = host_edges[2 * i + 1]; }
        }
        b->last_source = sources[k - 1];
        st = collect(b, nullptr, 0.0);
    }
    cleanup();
    return st;
}

}  // namespace
}  // namespace bd

extern "C" {

bd_status bd_bfs_run_many(bd_bfs *b, const int64_t *sources, int64_t k, double *ms_out,
                          int64_t *edges_out, int64_t *reached_out, double *e2e_ms)
{
    return run_many(b, sources, k, nullptr, nullptr, ms_out, edges_out, reached_out, e2e_ms);
}

bd_status bd_bfs_run_many_into(bd_bfs *b, const int64_t *sources, int64_t k, int32_t *d_depth,
                               int64_t *d_parent, double *ms_out, int64_t *edges_out,
                               int64_t *reached_out, double *e2e_ms)
{
    if (!d_depth || !d_parent) { return BD_ERR_INVALID; }
    return run_many(b, sources, k, d_depth, d_parent, ms_out, edges_out, reached_out, e2e_ms);
}

bd_status bd_bfs_get_depths(bd_bfs *b, int32_t *depth)
{
    if (!b || !depth) { return BD_ERR_INVALID; }
    if (!b->ran) { return BD_ERR_STATE; }
    BD_CUDA(cudaSetDevice(b->device));
    BD_TRY(finalize_parents(b));
    BD_CUDA(cudaMemcpy(depth, b->out_depth ? b->out_depth : b->depth, sizeof(int32_t) * b->g->n,
                       cudaMemcpyDeviceToHost));
    return BD_OK;
}

bd_status bd_bfs_get_parents(bd_bfs *b, int64_t *parent)
{
    if (!b || !parent) { return BD_ERR_INVALID; }
    BD_CUDA(cudaSetDevice(b->device));
    BD_TRY(finalize_parents(b));
    BD_CUDA(cudaMemcpy(parent, b->out_parent ? b->out_parent : b->parent,
                       sizeof(int64_t) * b->g->n, cudaMemcpyDeviceToHost));
    return BD_OK;
}

bd_status bd_bfs_device_ptrs(bd_bfs *b, const int32_t **depth, const int64_t **parent)
{
    if (!b) { return BD_ERR_INVALID; }
    BD_CUDA(cudaSetDevice(b->device));
    BD_TRY(finalize_parents(b));
    if (depth) { *depth = b->out_depth ? b->out_depth : b->depth; }
    if (parent) { *parent = b->out_parent ? b->out_parent : b->parent; }
    return BD_OK;
}

bd_status bd_bfs_count_traversed_edges(bd_bfs *b, int64_t *out)
{
    if (!b || !out) { return BD_ERR_INVALID; }
    if (!b->ran) { return BD_ERR_STATE; }
    *out = b->last.st.visited_degsum / 2;
    return BD_OK;
}

// hybrid_bfs::check (hybrid_bfs.cc:281-379), on the device (bd_check.cu),
// of the parents the last run left in HBM.
bd_status bd_bfs_check(bd_bfs *b, int64_t source, int32_t *ok)
{
    if (!b || !ok) { return BD_ERR_INVALID; }
    if (source < 0 || source >= b->g->n) { return BD_ERR_RANGE; }
    const int64_t *parent = nullptr;
    BD_TRY(bd_bfs_device_ptrs(b, nullptr, &parent));
    return check_parents_device(b->g, source, parent, ok, nullptr);
}

bd_status bd_bfs_get_steps(bd_bfs *b, bd_step *steps, int64_t capacity, int64_t *count)
{
    if (!b || !count || capacity < 0 || (!steps && capacity)) { return BD_ERR_INVALID; }
    if (!b->ran) { return BD_ERR_STATE; }
    int64_t have = std::min<int64_t>(b->last.st.step, kRecCap);
    int64_t take = std::min(have, capacity);
    if (take) {
        BD_CUDA(cudaSetDevice(b->device));
        BD_CUDA(cudaMemcpy(steps, b->rec, sizeof(bd_step) * take, cudaMemcpyDeviceToHost));
    }
    *count = have;
    return BD_OK;
}

bd_status bd_bfs_destroy(bd_bfs *b)
{
    if (!b) { return BD_ERR_INVALID; }
    bfs_free(b);
    return BD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point (bd_bfs_run_noalloc).
//
// For callers that must not allocate device memory while they run a BFS:
// a service whose device memory is fully carved up in advance by its own
// pool allocator (a cudaMalloc there fails or fragments the pool), or code
// that cannot afford the device-wide synchronisation cudaMalloc / cudaFree
// may cause.  The caller passes the CSR and the output arrays; every
// temporary (control block, the two visited bitmaps, the frontier queues)
// lives in one file-scope device array of fixed size, so graphs are limited
// to BD_NOALLOC_MAX_VERTICES vertices.  Each GPU that loads this library
// holds that array (about 7.2 MB) until the process exits.
// ---------------------------------------------------------------------------
namespace bd {
namespace {

constexpr int64_t kNaMaxVertices = BD_NOALLOC_MAX_VERTICES;
constexpr int64_t kNaWords = kNaMaxVertices / 32;
constexpr int64_t kNaLarge = 1 << 17;  // slots for large-degree frontier vertices
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNaOffCtrl = 0;
constexpr size_t kNaOffSource = align256(kNaOffCtrl + sizeof(Ctrl));
constexpr size_t kNaOffLive = kNaOffSource + sizeof(int64_t);  // vertices of nonzero degree
constexpr size_t kNaOffVis = align256(kNaOffLive + sizeof(unsigned long long));
constexpr size_t kNaOffQs = align256(kNaOffVis + 2 * sizeof(uint32_t) * kNaWords);
constexpr size_t kNaOffQl = align256(kNaOffQs + 2 * sizeof(uint32_t) * kNaMaxVertices);
constexpr size_t kNaOffQlb = align256(kNaOffQl + 2 * sizeof(uint32_t) * kNaLarge);
constexpr size_t kNaBytes = align256(kNaOffQlb + 2 * sizeof(unsigned long long) * kNaLarge);

// The scratch array.  Host code must not use this name as an address: it
// gets the device address from cudaGetSymbolAddress (noalloc_scratch_base).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
unsigned char *g_na_base[kNaMaxDevices] = {};
int g_na_grid[kNaMaxDevices] = {};

// Once per device, with that device current: the device address of the
// scratch array and the co-resident grid size of the persistent kernel.
bd_status noalloc_setup(int dev, unsigned char **base, int *grid)
{
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_base[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) { return cuda_fail(e, "cudaGetSymbolAddress", __FILE__, __LINE__); }
        int per_sm = 0, sms = 0;
        KernelChoice kc = pick_kernel(512);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)kc.fn, kc.block, 0);
        if (e == cudaSuccess) { e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev); }
        if (e != cudaSuccess) { return cuda_fail(e, "occupancy", __FILE__, __LINE__); }
        if (per_sm < 1) { return BD_ERR_CUDA; }
        g_na_grid[dev] = per_sm * sms;
        g_na_base[dev] = static_cast<unsigned char *>(ptr);
    }
    *base = g_na_base[dev];
    *grid = g_na_grid[dev];
    return BD_OK;
}

// depth = -1; vis[0] = degree-zero and padding bits; the source id; the
// count of vertices of nonzero degree added into *live (zeroed before).
__global__ void noalloc_prepare_kernel(const int64_t *off, int64_t n, int32_t *depth,
                                       uint32_t *vis0, int64_t source, int64_t *source_slot,
                                       unsigned long long *live)
{
    const int64_t words = (n + 31) / 32;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t v = t; v < n; v += stride) { depth[v] = -1; }
    unsigned long long nz = 0;
    for (int64_t w = t; w < words; w += stride) {
        uint32_t b = 0;
        for (int k = 0; k < 32; ++k) {
            const int64_t v = w * 32 + k;
            if (v >= n || off[v + 1] == off[v]) { b |= 1u << k; }
        }
        vis0[w] = b;
        nz += 32 - __popc(b);
    }
    nz = dev::warp_sum(nz);
    if (dev::lane_id() == 0 && nz) { atomicAdd(live, nz); }
    if (t == 0) { *source_slot = source; }
}

}  // namespace
}  // namespace bd

extern "C" bd_status bd_bfs_run_noalloc(const int64_t *d_offsets, const uint32_t *d_adjacency,
                                        int64_t num_vertices, int64_t num_arcs, int64_t source,
                                        int64_t alpha, int64_t beta, int32_t *d_depth,
                                        int64_t *d_parent, void *stream,
                                        int64_t *traversed_edges)
{
    using namespace bd;
    if (!d_offsets || (!d_adjacency && num_arcs) || !d_depth || !d_parent || num_vertices <= 0 ||
        num_arcs < 0 || alpha <= 0 || beta <= 0) {
        return BD_ERR_INVALID;
    }
    if (num_vertices > kNaMaxVertices || num_arcs > ((int64_t)1 << 34)) { return BD_ERR_LIMIT; }
    if (source < 0 || source >= num_vertices) { return BD_ERR_RANGE; }
    int dev = 0, major = 0;
    BD_CUDA(cudaGetDevice(&dev));
    BD_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10 || dev >= kNaMaxDevices) { return BD_ERR_NODEV; }
    unsigned char *base = nullptr;
    int grid = 0;
    BD_TRY(noalloc_setup(dev, &base, &grid));
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    BfsParams p{};
    p.off = d_offsets;
    p.adj = d_adjacency;
    p.n = num_vertices;
    p.m = num_arcs / 2;
    p.depth = d_depth;
    p.parent = d_parent;
    p.words = bitmap_words(num_vertices);
    Ctrl *ctrl = reinterpret_cast<Ctrl *>(base + kNaOffCtrl);
    int64_t *source_slot = reinterpret_cast<int64_t *>(base + kNaOffSource);
    unsigned long long *live = reinterpret_cast<unsigned long long *>(base + kNaOffLive);
    for (int i = 0; i < 2; ++i) {
        p.vis[i] = reinterpret_cast<uint32_t *>(base + kNaOffVis) + i * kNaWords;
        p.qs[i] = reinterpret_cast<uint32_t *>(base + kNaOffQs) + i * kNaMaxVertices;
        p.ql[i] = reinterpret_cast<uint32_t *>(base + kNaOffQl) + i * kNaLarge;
        p.qlb[i] = reinterpret_cast<unsigned long long *>(base + kNaOffQlb) + i * kNaLarge;
    }
    p.ctrl = ctrl;
    p.rec = nullptr;
    p.rec_cap = 0;
    p.alg = BD_ALG_BEAMER;
    p.alpha = alpha;
    p.beta = beta;
    // The regular handle's defaults (bd_bfs_create), except that the
    // large-degree threshold rises above them on graphs of more than
    // 32 x kNaLarge arcs: at most num_arcs / large_deg vertices qualify, and
    // the array holds kNaLarge of them.
    p.large_deg = (uint32_t)std::max<int64_t>(32, num_arcs / kNaLarge + 1);
    p.chunk = 256;
    p.bu_prefix = 32;
    p.spin_limit = kDefaultSpin;
    p.expected_ctas = (unsigned)grid;
    p.policy = nullptr;

    // The control block, source slot, live count and vis[0] are rewritten
    // here; the queues and vis[1] are written before they are read within a
    // run.  The live count (vertices of nonzero degree) decides the
    // bottom-up layout switch, so it is read back before the launch.
    BD_CUDA(cudaMemsetAsync(live, 0, sizeof(unsigned long long), s));
    noalloc_prepare_kernel<<<grid_for(std::max<int64_t>(num_vertices, 1)), 256, 0, s>>>(
        d_offsets, num_vertices, d_depth, p.vis[0], source, source_slot, live);
    BD_CUDA(cudaGetLastError());
    unsigned long long n_live = 0;
    BD_CUDA(cudaMemcpyAsync(&n_live, live, sizeof(n_live), cudaMemcpyDeviceToHost, s));
    BD_CUDA(cudaStreamSynchronize(s));
    p.n_live = (int64_t)n_live;
    init_sources_kernel<<<1, 32, 0, s>>>(p, source_slot, 1, 0);
    BD_CUDA(cudaGetLastError());
    KernelChoice kc = pick_kernel(512);
    void *args[] = {&p};
    BD_CUDA(cudaLaunchCooperativeKernel((const void *)kc.fn, dim3(grid), dim3(kc.block), args, 0, s));
    finalize_parents_kernel<<<grid_for(num_vertices), 256, 0, s>>>(d_offsets, num_vertices, d_depth,
                                                                   d_parent);
    BD_CUDA(cudaGetLastError());
    Ctrl host{};
    BD_CUDA(cudaMemcpyAsync(&host, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
    BD_CUDA(cudaStreamSynchronize(s));
    if (host.error) { return (bd_status)host.error; }
    if (traversed_edges) { *traversed_edges = host.st.visited_degsum / 2; }
    return BD_OK;
}
