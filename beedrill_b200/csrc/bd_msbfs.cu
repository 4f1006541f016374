// bd_msbfs.cu -- batched traversal: up to 64 BFSs at once, one bit lane of a
// uint64 per root ("multi-source BFS"), in one persistent cooperative launch.
//
// The reference runs its trials one root at a time (hybrid_bfs_main.cc:252-302);
// every root re-reads the whole graph.  Here R <= 64 roots share each pass
// over the adjacency: vertex v carries reach[v] (lanes delivered to it so
// far, this step's deliveries included) and F[v] (lanes whose frontier holds
// it), and a level updates all lanes with 64-bit ORs.  Results per lane are exactly
// those of a single-source BFS from that lane's root: depths equal, parents
// one level up (each (vertex, lane) gets the first neighbour that delivered
// the lane's bit).
//
// Steps, chosen per level on the device (Beamer-style rule over the batch):
//   push  frontier vertices OR their lanes into their neighbours' reach
//         word (atomicOr; the returned old word identifies the one writer
//         that delivered each new lane, which becomes that lane's parent),
//         then into the next frontier word;
//   pull  each vertex not yet reached by every lane ORs its neighbours'
//         frontier words until it has all the lanes it still needs that
//         some frontier holds (the lanes delivered by the step before).
//
// Layout in HBM (n vertices, R lanes):
//   reach   uint64[n]      lanes delivered to v so far: one load tells a
//                          push which lanes v still lacks; after the run,
//                          the lanes that reached v
//   F[3]    uint64[n]      frontier words, three buffers: step s reads
//                          F[s%3], writes F[(s+1)%3], clears F[(s+2)%3]
//   Q[3]                   the vertex lists of those frontiers (degree bins)
//   done    uint32[n/32]   vertices every lane has reached, and isolated ones:
//                          pull steps skip them by the word
//   drec    16 B [n][16]   delivery records: {lane mask lo, hi, provider,
//                          level}, one store for all the lanes one
//                          neighbour delivered at one level, push or pull
//                          (drec_cnt[n] counts them)
//   depth   int32[n][R]    per-lane rows, vertex-major (a vertex's lanes share
//   parent  uint32[n][R]   sectors): deliveries past a vertex's 16 records
// The kernel leaves F zero when it ends (it clears the last
// frontier's words), so a call needs no memsets of them.
#include <algorithm>
#include <cstring>
#include <vector>

#include "bd_device_util.cuh"
#include "bd_internal.h"
#include "bd_policy.cuh"

namespace bd {
namespace {

using namespace dev;
using ull = unsigned long long;

constexpr int kPush = 0, kPull = 1, kMsDone = 2;
constexpr int kLargeShift = 38;
constexpr ull kChunkMask = (1ull << kLargeShift) - 1;
constexpr int64_t kMsRecCap = 1 << 14;
constexpr long long kMsDefaultSpin = 4000000;
constexpr unsigned kRecSlots = 16;  // delivery records per vertex

// Counters of one step, in a ring of three slots (step s uses s % 3; CTA 0
// clears (s + 1) % 3 during step s, after every CTA has read it).
struct MsAcc {
    ull vertices;    // vertices entering the next frontier
    ull degsum;      // their degree sum
    ull lanes;       // new (vertex, lane) pairs
    ull small_cnt;
    ull large_packed;
    ull done_degsum; // degree sum of vertices that just got every lane
    ull t_end;       // max over CTAs of their arrival time
    ull work;        // pull steps: next bitmap word to hand out
    ull lanes_or;    // lanes delivered in the step (the next frontier's lanes)
};

// State between steps: written first by the init kernel, then kept by every
// CTA as an identical copy in shared memory (advanced by the same function
// of the same counters), written back by CTA 0 at the end.
struct MsState {
    int dir, level, step, prev_dir;
    long long f_count, f_degsum, f_small, f_large, f_chunks;
    long long p_small, p_large;  // lists of the frontier read by the previous step
    long long arcs_left;         // 2m - degree sum of vertices reached by all lanes
    long long lanes_total;
    long long t_last, push_steps, pull_steps;
    long long prev_ns, policy_overrides;
    ull active;                  // lanes the frontier about to be expanded holds
};

struct MsCtrl {
    ull bar;       // barrier arrivals; step s is complete at (s + 1) * CTAs
    int error, pad0;
    ull t_start;   // min over CTAs of their start time
    MsState st;
    MsAcc acc[3];
};

struct MsParams {
    const int64_t *off;
    const uint32_t *adj;
    uint32_t *done;   // bit v: every lane reached v, or v is isolated (no lane can)
    int64_t n, m;
    ull *reach;       // lanes delivered to v so far (the handle's seen array)
    ull *F[3];
    uint32_t *qs[3];
    uint32_t *ql[3];
    ull *qlb[3];
    int32_t *depth;     // per-lane rows, used when a vertex runs out of records
    uint32_t *parent;
    uint4 *drec;        // [n][kRecSlots] delivery records {mask lo, mask hi, provider, level}
    uint32_t *drec_cnt; // [n] records written (may exceed kRecSlots)
    int R;
    ull all;
    MsCtrl *ctrl;
    bd_step *rec;
    int64_t rec_cap;
    int64_t alpha;
    uint32_t large_deg, chunk;
    int prefix;
    long long spin_limit;
    unsigned expected_ctas;
    int force_dir;  // -1 rule, kPush, kPull
    const PolicyBlob *policy;  // null: the rule decides
    const uint32_t *perm;      // caller id -> traversal id (BD_ORDER_HUB), or null
    // vertices whose pull scan is split into chunks over all warps
    const uint32_t *heavy;           // [n_heavy]
    const ull *heavy_cbase;          // [n_heavy + 1] chunk prefix sums
    int64_t n_heavy;
    int64_t heavy_deg;               // degree above which a vertex is heavy
    uint32_t heavy_chunk;            // arcs per chunk
};

struct MsLocal {
    ull vertices, degsum, lanes, done_degsum, lanes_or;
};

// Frontier word of v (zero outside the frontier).  Read directly: most arcs
// a pull scans lead to frontier hubs, whose words the hub layout keeps in
// L2, so checking the frontier bitmap first would only add a dependent load
// to every arc (same-box A/B: the direct read is 12 % faster at RMAT scale
// 24, 16 % at scale 20).  Plain loads: the buffers read in a step are not
// written in it, and every CTA passed the grid barrier's acquire before the
// step.
__device__ __forceinline__ ull frontier_word(const MsParams &p, int buf, uint32_t v)
{
    return p.F[buf][v];
}

__device__ __forceinline__ int64_t ms_degree(const MsParams &p, uint32_t v)
{
    return __ldg(&p.off[v + 1]) - __ldg(&p.off[v]);
}

// Warp-collective append of new frontier vertices, binned by degree
// (same scheme as the single-source kernel).
__device__ __forceinline__ void ms_append(const MsParams &p, MsAcc *acc, int qn, bool has,
                                          uint32_t v, int64_t deg, MsLocal &loc)
{
    if (has) {
        loc.vertices += 1;
        loc.degsum += (ull)deg;
    }
    const int lane = lane_id();
    const bool large = has && deg >= (int64_t)p.large_deg;
    const unsigned sm = __ballot_sync(kFullMask, has && !large);
    if (sm) {
        const int leader = __ffs(sm) - 1;
        ull base = 0;
        if (lane == leader) { base = atomicAdd(&acc->small_cnt, (ull)__popc(sm)); }
        base = __shfl_sync(kFullMask, base, leader);
        if (has && !large) { p.qs[qn][base + __popc(sm & lanemask_lt())] = v; }
    }
    const unsigned lm = __ballot_sync(kFullMask, large);
    if (lm) {
        const ull nch = large ? (ull)((deg + p.chunk - 1) / p.chunk) : 0ull;
        const ull incl = warp_incl_scan(nch);
        const ull total = __shfl_sync(kFullMask, incl, 31);
        const int leader = __ffs(lm) - 1;
        ull old = 0;
        if (lane == leader) {
            old = atomicAdd(&acc->large_packed, ((ull)__popc(lm) << kLargeShift) | total);
        }
        old = __shfl_sync(kFullMask, old, leader);
        if (large) {
            const ull pos = (old >> kLargeShift) + __popc(lm & lanemask_lt());
            p.ql[qn][pos] = v;
            p.qlb[qn][pos] = (old & kChunkMask) + incl - nch;
        }
    }
}

// Warp-collective append of up to K new frontier vertices per lane: one
// atomic for all the small-degree ones of the warp, one for the large ones.
template <int K>
__device__ __forceinline__ void ms_append_k(const MsParams &p, MsAcc *acc, int qn,
                                            const bool (&has)[K], const uint32_t (&v)[K],
                                            const int64_t (&deg)[K], MsLocal &loc)
{
    const int lane = lane_id();
    unsigned sm[K];
    bool large[K];
    unsigned total = 0, any_large = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (has[k]) {
            loc.vertices += 1;
            loc.degsum += (ull)deg[k];
        }
        large[k] = has[k] && deg[k] >= (int64_t)p.large_deg;
        sm[k] = __ballot_sync(kFullMask, has[k] && !large[k]);
        total += __popc(sm[k]);
        any_large |= __ballot_sync(kFullMask, large[k]);
    }
    if (total) {
        ull base = 0;
        if (lane == 0) { base = atomicAdd(&acc->small_cnt, (ull)total); }
        base = __shfl_sync(kFullMask, base, 0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (has[k] && !large[k]) { p.qs[qn][base + __popc(sm[k] & lanemask_lt())] = v[k]; }
            base += __popc(sm[k]);
        }
    }
    if (any_large) {
        unsigned count = 0;
        ull chunks = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (large[k]) {
                count += 1;
                chunks += (ull)((deg[k] + p.chunk - 1) / p.chunk);
            }
        }
        const unsigned ci = warp_incl_scan(count);
        const ull hi = warp_incl_scan(chunks);
        const unsigned ct = __shfl_sync(kFullMask, ci, 31);
        const ull ht = __shfl_sync(kFullMask, hi, 31);
        ull old = 0;
        if (lane == 0) { old = atomicAdd(&acc->large_packed, ((ull)ct << kLargeShift) | ht); }
        old = __shfl_sync(kFullMask, old, 0);
        ull pos = (old >> kLargeShift) + (ci - count);
        ull cbase = (old & kChunkMask) + (hi - chunks);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (large[k]) {
                p.ql[qn][pos] = v[k];
                p.qlb[qn][pos] = cbase;
                pos += 1;
                cbase += (ull)((deg[k] + p.chunk - 1) / p.chunk);
            }
        }
    }
}

// Lanes whose vertex has run out of delivery records: one depth and one
// parent entry per lane in the vertex-major rows.
__device__ __forceinline__ void write_rows(const MsParams &p, uint32_t v, ull lanes, int level,
                                           uint32_t parent)
{
    while (lanes) {
        const int r = __ffsll((long long)lanes) - 1;
        lanes &= lanes - 1;
        p.depth[(int64_t)v * p.R + r] = level;
        p.parent[(int64_t)v * p.R + r] = parent;
    }
}

// Delivery record `slot` of v: the lanes that `parent` delivered at `level`
// (one 16-byte store for all of them).  Past kRecSlots, per-lane rows.
__device__ __forceinline__ void put_record(const MsParams &p, uint32_t v, unsigned slot,
                                           ull lanes, int level, uint32_t parent)
{
    if (slot < kRecSlots) {
        p.drec[(int64_t)v * kRecSlots + slot] =
            make_uint4((uint32_t)lanes, (uint32_t)(lanes >> 32), parent, (uint32_t)level);
    } else {
        write_rows(p, v, lanes, level, parent);
    }
}

// A record from one of several concurrent deliverers (push, chunked pull).
__device__ __forceinline__ void record_shared(const MsParams &p, uint32_t v, ull lanes, int level,
                                              uint32_t parent)
{
    put_record(p, v, atomicAdd(&p.drec_cnt[v], 1u), lanes, level, parent);
}

struct MsView {
    int dir, level, step;
    long long f_small, f_large, f_chunks, p_small, p_large;
    ull active;
};

__device__ __forceinline__ MsView ms_view(const MsState &c)
{
    MsView v;
    v.dir = c.dir;
    v.level = c.level;
    v.step = c.step;
    v.f_small = c.f_small;
    v.f_large = c.f_large;
    v.f_chunks = c.f_chunks;
    v.p_small = c.p_small;
    v.p_large = c.p_large;
    v.active = c.active;
    return v;
}

// Zeroes the frontier words of the frontier read by the previous step.
__device__ void ms_clear_old(const MsParams &p, const MsView &sv)
{
    const int old = (sv.step + 2) % 3;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    for (long long i = t; i < sv.p_small; i += nt) { p.F[old][p.qs[old][i]] = 0ull; }
    for (long long i = t; i < sv.p_large; i += nt) { p.F[old][p.ql[old][i]] = 0ull; }
}

// push: lanes of frontier vertex u flow into neighbours [b, e), four arcs
// per lane per round with each stage's loads and atomics issued back to
// back.  One plain read of the neighbour's reach word filters the arcs
// that deliver nothing (a vertex every lane has reached holds all lanes in
// it, so no done-bit read is needed); the atomicOr on the
// reach word tells each deliverer which lanes it delivered first -- it
// writes one delivery record for them (a slot from an atomicAdd on the
// vertex's record count; every (vertex, lane) pair is delivered exactly
// once, so no two records hold the same pair; one 16-byte store instead of
// two 4-byte row stores per lane: 5 % off the scale-24 traversal) -- and an
// atomicOr on the next frontier word, issued together with the reach
// update rather than after it, tells which deliverer puts the neighbour on
// the next frontier's list.
constexpr int kPushU = 4;

// One round of up to kPushU arcs per lane: arc i of this lane goes from
// src[i] (whose frontier lanes are bits[i]) to v[i].
__device__ __forceinline__ void push_arcs(const MsParams &p, MsAcc *acc, int cur, int nxt,
                                          int new_level, const bool (&in)[kPushU],
                                          const uint32_t (&v)[kPushU],
                                          const uint32_t (&src)[kPushU],
                                          const ull (&bits)[kPushU], MsLocal &loc)
{
    ull g[kPushU];  // lanes to give, then the lanes this writer delivered first
#pragma unroll
    for (int i = 0; i < kPushU; ++i) {
        // a stale read only costs an atomic that changes nothing (a vertex
        // every lane has reached holds them all in its reach word)
        const ull have = in[i] ? __ldcg(&p.reach[v[i]]) : ~0ull;
        g[i] = bits[i] & ~have;
    }
    // Both atomics at once.  The frontier word takes the lanes v lacked
    // when the step began (the reach read above sees every earlier step's
    // lanes), so it ends up holding exactly the lanes delivered to v in this
    // step whichever deliverer's reach update lands first; the one writer
    // that finds it empty lists v, even if others delivered its lanes first.
    ull old_r[kPushU], old_f[kPushU];
#pragma unroll
    for (int i = 0; i < kPushU; ++i) {
        old_r[i] = g[i] ? atomicOr(&p.reach[v[i]], g[i]) : ~0ull;
        old_f[i] = g[i] ? atomicOr(&p.F[nxt][v[i]], g[i]) : ~0ull;
    }
    bool completed[kPushU], first[kPushU];
#pragma unroll
    for (int i = 0; i < kPushU; ++i) {
        first[i] = g[i] && old_f[i] == 0ull;
        g[i] &= ~old_r[i];
        completed[i] = g[i] && ((old_r[i] | g[i]) & p.all) == p.all;
    }
    int64_t deg[kPushU];
#pragma unroll
    for (int i = 0; i < kPushU; ++i) {
        deg[i] = 0;
        if (g[i]) {
            record_shared(p, v[i], g[i], new_level, src[i]);
            loc.lanes += __popcll(g[i]);
            loc.lanes_or |= g[i];
        }
        if (first[i] || completed[i]) { deg[i] = ms_degree(p, v[i]); }
        if (completed[i]) {
            loc.done_degsum += (ull)deg[i];
            atomicOr(&p.done[v[i] >> 5], 1u << (v[i] & 31));
        }
        if (!first[i]) { deg[i] = 0; }
    }
    ms_append_k<kPushU>(p, acc, nxt, first, v, deg, loc);
}

// Arcs [b, e) of frontier vertex u (lanes `bits`), all 32 lanes, coalesced.
__device__ __forceinline__ void push_edges(const MsParams &p, MsAcc *acc, int cur, int nxt,
                                           int new_level, uint32_t u, ull bits, int64_t b,
                                           int64_t e, MsLocal &loc)
{
    const int lane = lane_id();
    for (int64_t base = b; base < e; base += 32 * kPushU) {
        uint32_t v[kPushU], src[kPushU];
        ull bt[kPushU];
        bool in[kPushU];
#pragma unroll
        for (int i = 0; i < kPushU; ++i) {
            const int64_t k = base + 32 * i + lane;
            in[i] = k < e;
            v[i] = in[i] ? __ldg(&p.adj[k]) : 0u;
            src[i] = u;
            bt[i] = bits;
        }
        push_arcs(p, acc, cur, nxt, new_level, in, v, src, bt, loc);
    }
}

// Per-warp scratch of the small-vertex push: 32 frontier vertices, their
// lanes, list starts and the inclusive prefix of their degrees.
struct MsWarpScratch {
    int32_t incl[32];
    uint32_t u[32];
    int64_t beg[32];
    ull bits[32];
};

template <int BLOCK>
__device__ void ms_push_step(const MsParams &p, const MsView &sv, MsWarpScratch &ws, MsLocal &loc)
{
    const int lane = lane_id();
    const int warp = threadIdx.x >> 5;
    const long long gw = (long long)blockIdx.x * (BLOCK / 32) + warp;
    const long long nw = (long long)gridDim.x * (BLOCK / 32);
    const int cur = sv.step % 3, nxt = (sv.step + 1) % 3;
    MsAcc *acc = &p.ctrl->acc[sv.step % 3];
    const int new_level = sv.level + 1;
    // large frontier vertices: chunk c of vertex ql[i]
    for (long long c = gw; c < sv.f_chunks; c += nw) {
        long long lo = 0, hi = sv.f_large - 1;
        while (lo < hi) {
            long long mid = (lo + hi + 1) >> 1;
            if ((long long)__ldcg(&p.qlb[cur][mid]) <= c) { lo = mid; } else { hi = mid - 1; }
        }
        const uint32_t u = __ldcg(&p.ql[cur][lo]);
        const long long j = c - (long long)__ldcg(&p.qlb[cur][lo]);
        const ull bits = __ldcg(&p.F[cur][u]);
        const int64_t ub = __ldg(&p.off[u]), ue = __ldg(&p.off[u + 1]);
        const int64_t b = ub + j * (int64_t)p.chunk;
        push_edges(p, acc, cur, nxt, new_level, u, bits, b, min(ue, b + (int64_t)p.chunk), loc);
    }
    // small frontier vertices, 32 per warp: their lists are laid end to end
    // and dealt to the lanes kPushU x 32 arcs at a time
    for (long long g = gw; g * 32 < sv.f_small; g += nw) {
        const long long idx = g * 32 + lane;
        uint32_t u = 0;
        ull bits = 0;
        int64_t beg = 0;
        int32_t deg = 0;
        if (idx < sv.f_small) {
            u = __ldcg(&p.qs[cur][idx]);
            bits = __ldcg(&p.F[cur][u]);
            beg = __ldg(&p.off[u]);
            deg = (int32_t)(__ldg(&p.off[u + 1]) - beg);
        }
        const int32_t incl = warp_incl_scan(deg);
        const int32_t total = __shfl_sync(kFullMask, incl, 31);
        ws.incl[lane] = incl;
        ws.u[lane] = u;
        ws.beg[lane] = beg;
        ws.bits[lane] = bits;
        __syncwarp();
        for (int32_t base = 0; base < total; base += 32 * kPushU) {
            uint32_t v[kPushU], src[kPushU];
            ull bt[kPushU];
            bool in[kPushU];
#pragma unroll
            for (int i = 0; i < kPushU; ++i) {
                const int32_t e = base + i * 32 + lane;
                in[i] = e < total;
                v[i] = 0;
                src[i] = 0;
                bt[i] = 0;
                if (in[i]) {
                    int lo = 0, hi = 31;  // first owner with incl > e
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (ws.incl[mid] > e) { hi = mid; } else { lo = mid + 1; }
                    }
                    const int32_t excl = lo ? ws.incl[lo - 1] : 0;
                    src[i] = ws.u[lo];
                    bt[i] = ws.bits[lo];
                    v[i] = __ldg(&p.adj[ws.beg[lo] + (e - excl)]);
                }
            }
            push_arcs(p, acc, cur, nxt, new_level, in, v, src, bt, loc);
        }
        __syncwarp();
    }
}

// pull: warp per 32 vertices; short lists per lane, long lists by the warp.
// pull for heavy vertices: their lists are cut into chunks dealt to all
// warps.  A chunk ORs the lanes it finds into the vertex's next frontier
// word; the bits the atomic returns as new are the ones this chunk
// delivered first, so their parents come from this chunk.
template <int BLOCK>
__device__ void ms_pull_heavy(const MsParams &p, const MsView &sv, MsLocal &loc)
{
    const int lane = lane_id();
    const int warp = threadIdx.x >> 5;
    const long long gw = (long long)blockIdx.x * (BLOCK / 32) + warp;
    const long long nw = (long long)gridDim.x * (BLOCK / 32);
    const int cur = sv.step % 3, nxt = (sv.step + 1) % 3;
    MsAcc *acc = &p.ctrl->acc[sv.step % 3];
    const int new_level = sv.level + 1;
    const long long total = p.n_heavy ? (long long)__ldg(&p.heavy_cbase[p.n_heavy]) : 0;
    // chunks dealt round robin: the chunks of one heavy vertex run on
    // different warps at once, and any of them may find the vertex's last
    // missing lanes
    for (long long c = gw; c < total; c += nw) {
        long long lo = 0, hi = p.n_heavy - 1;  // last i with heavy_cbase[i] <= c
        while (lo < hi) {
            const long long mid = (lo + hi + 1) >> 1;
            if ((long long)__ldg(&p.heavy_cbase[mid]) <= c) { lo = mid; } else { hi = mid - 1; }
        }
        const uint32_t v = __ldg(&p.heavy[lo]);
        // lanes v lacks that the frontier holds (other chunks of v may have
        // delivered some already this step)
        const ull need = p.all & ~__ldcg(&p.reach[v]) & sv.active;
        if (!need) { continue; }
        const int64_t vb = __ldg(&p.off[v]), ve = __ldg(&p.off[v + 1]);
        const int64_t b = vb + (c - (long long)__ldg(&p.heavy_cbase[lo])) * (int64_t)p.heavy_chunk;
        const int64_t e = min(ve, b + (int64_t)p.heavy_chunk);
        ull have = 0;  // lanes this chunk found or saw others deliver
        for (int64_t base = b; base < e && (have & need) != need; base += 128) {
            uint32_t u[4];
            ull fu[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t k = base + 32 * i + lane;
                u[i] = k < e ? __ldg(&p.adj[k]) : 0u;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t k = base + 32 * i + lane;
                fu[i] = k < e ? frontier_word(p, cur, u[i]) & need : 0ull;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const ull f = fu[i] & ~have;
                if (!__any_sync(kFullMask, f != 0)) { continue; }
                const ull mine = f & ~warp_excl_or(f);
                const ull round = warp_or(f);
                ull old = 0, before = 0;
                if (lane == 0) {
                    // both atomics at once: the reach update takes the whole
                    // round (lanes another chunk delivered first are already
                    // in it), and the one update that completes v marks it
                    old = atomicOr(&p.F[nxt][v], round);
                    before = atomicOr(&p.reach[v], round) & p.all;
                }
                old = __shfl_sync(kFullMask, old, 0);
                const ull fresh = round & ~old;
                if (mine & fresh) { record_shared(p, v, mine & fresh, new_level, u[i]); }
                const bool first = lane == 0 && old == 0ull;
                if (lane == 0) {
                    loc.lanes += __popcll(fresh);
                    loc.lanes_or |= fresh;
                    if (before != p.all && ((before | round) & p.all) == p.all) {
                        loc.done_degsum += (ull)(ve - vb);
                        atomicOr(&p.done[v >> 5], 1u << (v & 31));
                    }
                }
                ms_append(p, acc, nxt, first, v, ve - vb, loc);
                have |= round | old;
            }
        }
    }
}

// The next chunk of a step's work for the calling warp: its own first
// (index gw, no atomic), then, when there are more chunks than warps, from
// the step's counter as chunk nw + k.
__device__ __forceinline__ ull ms_next_chunk(ull *counter, long long nw, long long chunks)
{
    if (chunks <= nw) { return (ull)chunks; }
    ull x = 0;
    if (lane_id() == 0) { x = atomicAdd(counter, 1ull); }
    return (ull)nw + __shfl_sync(kFullMask, x, 0);
}

template <int BLOCK>
__device__ void ms_pull_step(const MsParams &p, const MsView &sv, MsLocal &loc)
{
    const int lane = lane_id();
    const int cur = sv.step % 3, nxt = (sv.step + 1) % 3;
    MsAcc *acc = &p.ctrl->acc[sv.step % 3];
    const int new_level = sv.level + 1;
    const long long words = (p.n + 31) / 32;
    // Which words a warp walks.  Large graphs (at least two 32-word chunks
    // per warp): chunks handed out dynamically -- the warp's own first, then
    // from a counter of the step -- because work per word varies widely and
    // dynamic hand-out keeps the warps of a CTA finishing together; chunk c
    // holds words c, c + C, c + 2C, ... (C chunks), so the heavy
    // low-numbered words of a hub layout are spread over all chunks.
    // Smaller graphs: warp gw owns words gw, gw + nw, gw + 2 nw, ... (a
    // chunk per warp would leave most warps idle).  Either way a warp loads
    // 32 skip masks at once (one per lane) and walks only the words with
    // work: done vertices have nothing to do.
    const long long gw = (long long)blockIdx.x * (BLOCK / 32) + (threadIdx.x >> 5);
    const long long nw = (long long)gridDim.x * (BLOCK / 32);
    const long long chunks = (words + 31) / 32;
    const bool dynamic = chunks >= 2 * nw;
    const long long stride = dynamic ? chunks : nw;
    const long long limit = dynamic ? chunks : words;
    for (long long base = gw; base < limit;
         base = dynamic ? (long long)ms_next_chunk(&acc->work, nw, chunks) : base + 32 * nw) {
        const long long wl = base + lane * stride;
        const uint32_t sk = wl < words ? __ldcg(&p.done[wl]) : kFullMask;
        unsigned todo = __ballot_sync(kFullMask, sk != kFullMask);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const long long w = base + src * stride;
            const uint32_t skip = __shfl_sync(kFullMask, sk, src);
            const uint32_t v = (uint32_t)(w * 32 + lane);
            const bool live = !((skip >> lane) & 1u);
            ull need = 0, got = 0, s = 0;
            int64_t beg = 0, end = 0, next = 0;
            unsigned cnt = 0, cnt0 = 0;  // this vertex's delivery records
            if (live) {
                // lanes v lacks that some frontier vertex holds: only lanes
                // delivered by the previous step can arrive in this one
                s = __ldcg(&p.reach[v]);
                need = p.all & ~s & sv.active;
                if (need) {
                    beg = __ldg(&p.off[v]);
                    end = __ldg(&p.off[v + 1]);
                    if (end - beg > p.heavy_deg) {
                        // scanned in chunks by ms_pull_heavy
                        need = 0;
                        beg = end = 0;
                    }
                }
                if (need) {
                    cnt = cnt0 = __ldcg(&p.drec_cnt[v]);
                    const int64_t lim = min(end, beg + (int64_t)p.prefix);
                    int64_t k = beg;
                    // four arcs in flight per round
                    for (; k < lim && got != need; k += 4) {
                        uint32_t u[4];
                        ull fu[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) { u[i] = (k + i < lim) ? __ldg(&p.adj[k + i]) : 0u; }
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            fu[i] = (k + i < lim) ? frontier_word(p, cur, u[i]) : 0ull;
                        }
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const ull f = fu[i] & need & ~got;
                            if (f) {
                                got |= f;
                                put_record(p, v, cnt++, f, new_level, u[i]);
                            }
                        }
                    }
                    next = (got == need) ? end : min(k, lim);
                }
            }
            unsigned pending = __ballot_sync(kFullMask, need != 0 && got != need && next < end);
            while (pending) {
                const int owner = __ffs(pending) - 1;
                pending &= pending - 1;
                const int64_t b = __shfl_sync(kFullMask, next, owner);
                const int64_t e = __shfl_sync(kFullMask, end, owner);
                const ull nd = __shfl_sync(kFullMask, need, owner);
                ull have = __shfl_sync(kFullMask, got, owner);
                const uint32_t vo = __shfl_sync(kFullMask, v, owner);
                unsigned c = __shfl_sync(kFullMask, cnt, owner);
                // 128 arcs per round: four independent gathers per lane
                for (int64_t base = b; base < e && have != nd; base += 128) {
                    uint32_t u[4];
                    ull fu[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int64_t k = base + 32 * i + lane;
                        u[i] = k < e ? __ldg(&p.adj[k]) : 0u;
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int64_t k = base + 32 * i + lane;
                        fu[i] = k < e ? frontier_word(p, cur, u[i]) & nd : 0ull;
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const ull f = fu[i] & ~have;
                        if (!__any_sync(kFullMask, f != 0)) { continue; }
                        // arcs earlier in the list win: each lane keeps the bits
                        // no lower lane of this batch already delivered
                        const ull mine = f & ~warp_excl_or(f);
                        const unsigned bm = __ballot_sync(kFullMask, mine != 0);
                        if (mine) {
                            put_record(p, vo, c + __popc(bm & lanemask_lt()), mine, new_level, u[i]);
                        }
                        c += __popc(bm);
                        have |= warp_or(f);
                    }
                }
                if (lane == owner) {
                    got = have;
                    cnt = c;
                }
            }
            if (cnt != cnt0) { p.drec_cnt[v] = cnt; }
            const bool gained = got != 0;
            const bool completed = gained && ((s | got) & p.all) == p.all;
            const unsigned cm = __ballot_sync(kFullMask, completed);
            if (lane == 0 && cm) { atomicOr(&p.done[w], cm); }
            if (gained) {
                // v is this lane's alone in a pull step (heavy vertices are
                // left to ms_pull_heavy), so plain stores
                p.F[nxt][v] = got;
                p.reach[v] = s | got;
                loc.lanes += __popcll(got);
                loc.lanes_or |= got;
                if (completed) { loc.done_degsum += (ull)(end - beg); }
            }
            ms_append(p, acc, nxt, gained, v, end - beg, loc);
        }
    }
}

template <int BLOCK>
struct MsShared {
    MsWarpScratch warp[BLOCK / 32];
    ull red[5][BLOCK / 32];
    MsState st;     // this CTA's copy of the state
    PolicyBlob pol; // the learned policy's weights, staged once
    int rule_dir;
};

// The rule: pull once the frontier's edges are a sizeable share of the edges
// still able to deliver a lane (Beamer's alpha test over the batch) ...
__device__ int ms_rule(const MsState &c, const MsParams &p)
{
    if (c.f_count == 0) { return kMsDone; }
    if (p.force_dir >= 0) { return p.force_dir; }
    // ... and only once the frontier holds at least n / 1024 vertices: a
    // pull step sweeps the done bitmap, which a handful of frontier
    // vertices pushing their arcs does not pay for
    return (c.f_degsum * p.alpha > c.arcs_left && c.f_count * 1024 >= p.n) ? kPull : kPush;
}

// Advances the state over the step that just ended.  One thread per CTA;
// every CTA computes the same result.
__device__ void ms_advance(MsState &c, const MsAcc &a, long long t_end)
{
    c.prev_dir = c.dir;
    c.prev_ns = t_end - c.t_last;
    c.t_last = t_end;
    c.lanes_total += (long long)a.lanes;
    c.active = a.lanes_or;
    c.arcs_left -= (long long)a.done_degsum;
    c.p_small = c.f_small;
    c.p_large = c.f_large;
    c.f_count = (long long)a.vertices;
    c.f_degsum = (long long)a.degsum;
    c.f_small = (long long)a.small_cnt;
    c.f_large = (long long)(a.large_packed >> kLargeShift);
    c.f_chunks = (long long)(a.large_packed & kChunkMask);
    if (c.dir == kPush) { c.push_steps += 1; } else { c.pull_steps += 1; }
    c.level += 1;
    c.step += 1;
}

// Next direction: the rule, or the learned policy (warp 0, weights from w)
// where it is installed, trusted and confident.  Every thread of the block.
template <typename Shared>
__device__ void ms_decide(MsState &c, const MsParams &p, const PolicyBlob *w, Shared &sh)
{
    const int tid = threadIdx.x;
    if (tid == 0) { sh.rule_dir = ms_rule(c, p); }
    __syncthreads();
    // the network runs only where the frontier's degree sum over the
    // unexplored one lies in the band the policy was trained to decide in
    const bool learned = p.policy && p.force_dir < 0 && sh.rule_dir != kMsDone &&
                         policy_in_band(w, c.f_degsum, c.arcs_left);
    if (!learned) {
        if (tid == 0) { c.dir = sh.rule_dir; }
        return;
    }
    if (tid < 32) {
        const float gap = policy_gap_warp(w, c.f_count, c.f_degsum, c.arcs_left, c.level, p.n,
                                          p.m, c.prev_dir, c.prev_ns);
        if (tid == 0) {
            int d = sh.rule_dir;
            if (isfinite(gap) && fabsf(gap) >= w->margin) {
                const int pick = gap > 0.f ? kPull : kPush;
                if (pick != d) { c.policy_overrides += 1; }
                d = pick;
            }
            c.dir = d;
        }
    }
}

// The end of a step: block reduction of the counters, arrival at the grid
// barrier (one release-add per CTA), acquire polling until all CTAs have
// arrived, then every CTA advances its copy of the state and decides the
// next direction.  Waits are bounded by p.spin_limit polls.
template <int BLOCK>
__device__ void ms_end_step(const MsParams &p, const MsView &sv, MsShared<BLOCK> &sh, MsLocal &loc)
{
    MsCtrl *c = p.ctrl;
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    const ull a0 = warp_sum(loc.vertices), a1 = warp_sum(loc.degsum), a2 = warp_sum(loc.lanes),
              a3 = warp_sum(loc.done_degsum), a4 = warp_or(loc.lanes_or);
    if (lane == 0) {
        sh.red[0][warp] = a0;
        sh.red[1][warp] = a1;
        sh.red[2][warp] = a2;
        sh.red[3][warp] = a3;
        sh.red[4][warp] = a4;
    }
    loc = MsLocal{0, 0, 0, 0, 0};
    __syncthreads();
    if (threadIdx.x == 0) {
        ull t[4] = {0, 0, 0, 0}, lanes_or = 0;
        for (int i = 0; i < BLOCK / 32; ++i) {
            for (int j = 0; j < 4; ++j) { t[j] += sh.red[j][i]; }
            lanes_or |= sh.red[4][i];
        }
        const int s = sv.step;
        MsAcc *acc = &c->acc[s % 3];
        if (t[0]) { atomicAdd(&acc->vertices, t[0]); }
        if (t[1]) { atomicAdd(&acc->degsum, t[1]); }
        if (t[2]) { atomicAdd(&acc->lanes, t[2]); }
        if (t[3]) { atomicAdd(&acc->done_degsum, t[3]); }
        if (lanes_or) { atomicOr(&acc->lanes_or, lanes_or); }
        if (blockIdx.x == 0) {
            MsAcc *z = &c->acc[(s + 1) % 3];
            z->vertices = z->degsum = z->lanes = z->small_cnt = z->large_packed = 0;
            z->done_degsum = z->t_end = z->work = z->lanes_or = 0;
        }
        atomicMax(&acc->t_end, (ull)globaltimer());
        red_release_add64(&c->bar, 1ull);
        const ull target = (ull)(s + 1) * p.expected_ctas;
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
        MsState &st = sh.st;
        if (ok && __ldcg(&c->error) == 0) {
            MsAcc a;
            a.vertices = __ldcg(&acc->vertices);
            a.degsum = __ldcg(&acc->degsum);
            a.lanes = __ldcg(&acc->lanes);
            a.small_cnt = __ldcg(&acc->small_cnt);
            a.large_packed = __ldcg(&acc->large_packed);
            a.done_degsum = __ldcg(&acc->done_degsum);
            a.lanes_or = __ldcg(&acc->lanes_or);
            const long long t_end = (long long)__ldcg(&acc->t_end);
            if (s == 0) { st.t_last = (long long)__ldcg(&c->t_start); }
            if (blockIdx.x == 0 && s < p.rec_cap) {
                bd_step r;
                r.dir = st.dir;
                r.level = st.level;
                r.frontier = st.f_count;
                r.frontier_edges = st.f_degsum;
                r.unexplored_edges = st.arcs_left;
                r.found = (long long)a.lanes;
                r.ns = t_end - st.t_last;
                p.rec[s] = r;
            }
            ms_advance(st, a, t_end);
        } else {
            st.f_count = 0;  // leave the loop
        }
    }
    __syncthreads();
    ms_decide(sh.st, p, &sh.pol, sh);
    __syncthreads();
}

template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) msbfs_kernel(MsParams p)
{
    __shared__ MsShared<BLOCK> sh;
    MsCtrl *c = p.ctrl;
    if (threadIdx.x == 0) {
        sh.st = c->st;  // written by the init kernel before this launch
        atomicMin(&c->t_start, (ull)globaltimer());
    }
    if (p.policy) {
        const float *src = reinterpret_cast<const float *>(p.policy);
        float *dst = reinterpret_cast<float *>(&sh.pol);
        for (int i = threadIdx.x; i < (int)(sizeof(PolicyBlob) / sizeof(float)); i += BLOCK) {
            dst[i] = src[i];
        }
    }
    __syncthreads();
    MsLocal loc{0, 0, 0, 0, 0};
    while (sh.st.dir != kMsDone) {
        const MsView sv = ms_view(sh.st);
        ms_clear_old(p, sv);
        if (sv.dir == kPush) {
            ms_push_step<BLOCK>(p, sv, sh.warp[threadIdx.x >> 5], loc);
        } else {
            ms_pull_heavy<BLOCK>(p, sv, loc);
            ms_pull_step<BLOCK>(p, sv, loc);
        }
        ms_end_step<BLOCK>(p, sv, sh, loc);
    }
    // Leave the frontier buffers zero for the next group or call: the only
    // words still set are those of the last frontier read (the queues of
    // step - 1); after an error the host clears them instead.
    if (__ldcg(&c->error) == 0) { ms_clear_old(p, ms_view(sh.st)); }
    if (blockIdx.x == 0 && threadIdx.x == 0) { c->st = sh.st; }
}

// Sources: lane r starts at sources[r].  One thread (sources are few).
__global__ void ms_init_kernel(MsParams p, const int64_t *sources, int count)
{
    MsCtrl *c = p.ctrl;
    const int error = c->error;  // an earlier group's, reported for the call
    memset(c, 0, sizeof(MsCtrl));
    c->error = error;
    long long nsmall = 0, nf = 0, degsum = 0, done = 0;
    ull lp = 0;
    for (int r = 0; r < count; ++r) {
        const uint32_t s = p.perm ? p.perm[sources[r]] : (uint32_t)sources[r];
        const ull bit = 1ull << r;
        const ull before = p.F[0][s];
        p.F[0][s] = before | bit;
        p.reach[s] |= bit;
        put_record(p, s, p.drec_cnt[s]++, bit, 0, s);
        const int64_t deg = p.off[s + 1] - p.off[s];
        if (p.reach[s] == p.all) {
            done += deg;
            p.done[s >> 5] |= 1u << (s & 31);
        }
        if (before) { continue; }
        nf += 1;
        degsum += deg;
        if (deg >= (int64_t)p.large_deg) {
            const ull pos = lp >> kLargeShift;
            p.ql[0][pos] = s;
            p.qlb[0][pos] = lp & kChunkMask;
            lp += (1ull << kLargeShift) | (ull)((deg + p.chunk - 1) / p.chunk);
        } else {
            p.qs[0][nsmall++] = s;
        }
    }
    c->t_start = ~0ull;
    MsState &st = c->st;
    st.f_count = nf;
    st.f_degsum = degsum;
    st.f_small = nsmall;
    st.f_large = (long long)(lp >> kLargeShift);
    st.f_chunks = (long long)(lp & kChunkMask);
    st.arcs_left = 2 * p.m - done;
    st.active = p.all;
    st.lanes_total = count;
    st.dir = ms_rule(st, p);
}

// Per-lane reached count and degree sum (count_num_traversed_edges per root).
__global__ void ms_count_kernel(const ull *seen, const int64_t *off, int64_t n, ull all, int R,
                                unsigned long long *out /* [2][64]: reached, degsum */)
{
    __shared__ unsigned long long s_cnt[64], s_deg[64];
    __shared__ unsigned long long s_full_cnt, s_full_deg;
    for (int i = threadIdx.x; i < 64; i += blockDim.x) { s_cnt[i] = s_deg[i] = 0; }
    if (threadIdx.x == 0) { s_full_cnt = s_full_deg = 0; }
    __syncthreads();
    ull full_cnt = 0, full_deg = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        ull s = seen[v] & all;
        if (!s) { continue; }
        const int64_t d = off[v + 1] - off[v];
        if (s == all) {
            full_cnt += 1;
            full_deg += (ull)d;
            continue;
        }
        while (s) {
            const int r = __ffsll((long long)s) - 1;
            s &= s - 1;
            atomicAdd(&s_cnt[r], 1ull);
            atomicAdd(&s_deg[r], (ull)d);
        }
    }
    full_cnt = warp_sum(full_cnt);
    full_deg = warp_sum(full_deg);
    if (lane_id() == 0) {
        atomicAdd(&s_full_cnt, full_cnt);
        atomicAdd(&s_full_deg, full_deg);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const ull c = s_cnt[r] + s_full_cnt, dg = s_deg[r] + s_full_deg;
        if (c) { atomicAdd(&out[r], c); }
        if (dg) { atomicAdd(&out[64 + r], dg); }
    }
}

// Lane r's depths and parents in the single-source output format.  Lane r
// reached v iff seen bit r is set; its depth and parent are in the record of
// v whose mask holds bit r, or, when v ran out of records, in the per-lane
// rows.  Nothing else is valid, so neither the rows nor the records need
// clearing between runs (only the record counts do).
__global__ void ms_extract_kernel(const int32_t *depth, const uint32_t *parent, const uint4 *rec,
                                  const uint32_t *rec_cnt, const ull *seen, const int64_t *off,
                                  int64_t n, int R, int r, const uint32_t *perm,
                                  const uint32_t *iperm, int32_t *depth_out, int64_t *parent_out)
{
    // v: the caller's vertex id (output index, off); t: its traversal id
    // (state index, parents named by traversal id) -- equal unless the
    // graph has a hub numbering
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = perm ? (int64_t)perm[v] : v;
        int32_t d = -1;
        uint32_t par = 0;
        if ((seen[t] >> r) & 1ull) {
            const unsigned cnt = min(rec_cnt[t], kRecSlots);
            bool found = false;
            for (unsigned i = 0; i < cnt && !found; ++i) {
                const uint4 x = rec[t * kRecSlots + i];
                const ull mask = ((ull)x.y << 32) | x.x;
                if ((mask >> r) & 1ull) {
                    d = (int32_t)x.w;
                    par = x.z;
                    found = true;
                }
            }
            if (!found) {
                d = depth[t * R + r];
                par = parent[t * R + r];
            }
        }
        if (depth_out) { depth_out[v] = d; }
        if (parent_out) {
            if (d >= 0) {
                parent_out[v] = (int64_t)(iperm && par < n ? iperm[par] : par);
            } else {
                const int64_t g = off[v + 1] - off[v];
                parent_out[v] = g != 0 ? -g : -1;
            }
        }
    }
}

// Every lane of one group in the single-source output format at once: root
// (root0 + r) gets depth_out[(root0 + r) * n + v] and parent_out[...] for
// every caller vertex v (caller ids, the reference's encoding: the source is
// its own parent, unreached vertices -deg or -1).  One pass over the group's
// state instead of one per lane: thread i of a CTA takes caller vertex
// v0 + i of a tile of kMatThreads consecutive vertices and
//   fill   reads the vertex's seen word, record count and records once (a
//          record covers every lane one provider delivered at one level, so
//          the provider is renamed once per record) and the per-lane rows of
//          lanes past its records.  Every distinct (depth, parent) pair gets
//          a slot of a 16-entry table in shared memory (a record's slot is
//          its own; lanes one push delivered share a pair), and the slot of
//          every lane is kept as four 64-bit planes (bit r of plane b = bit b
//          of lane r's slot): a record sets its lanes in four ORs, whatever
//          their number, so the threads of a warp do not wait for the one
//          whose records hold the most lanes;
//   write  walks the roots with the planes shifted one lane a step: the
//          lane's slot gives its depth and parent with no branch, and the
//          CTA's threads store each root's row entries for kMatThreads
//          consecutive vertices, streaming past L2.
// No thread reads another's table, so there is no barrier and a warp's
// writes overlap another's loads.  A lane whose pair finds the table full
// reads its row in the write loop (more than 16 distinct deliverers).
struct MsOutParams {
    const int32_t *depth;     // per-lane rows [n][R]
    const uint32_t *parent;
    const uint4 *rec;         // [n][kRecSlots]
    const uint32_t *rec_cnt;  // [n]
    const ull *seen;          // [n]
    const int64_t *off;       // the caller's CSR offsets (unreached encoding)
    const uint32_t *perm;     // caller id -> traversal id, or null
    const uint32_t *iperm;    // traversal id -> caller id, or null
    int64_t n;
    int R;                    // lane stride of the rows
    int lanes;                // roots in the group
    int32_t *depth_out;       // row of the group's first root
    int64_t *parent_out;
};

constexpr int kMatThreads = 256;
constexpr unsigned kMatSlots = 16;
// per thread: a (depth, parent) pair per slot, slot-major [kMatSlots][threads]
constexpr size_t kMatSmem = (size_t)kMatThreads * kMatSlots * sizeof(uint2);

// Adds `lanes` to the planes of slot k.
__device__ __forceinline__ void mat_set_slot(ull (&plane)[4], unsigned k, ull lanes)
{
#pragma unroll
    for (int b = 0; b < 4; ++b) { plane[b] |= ((k >> b) & 1u) ? lanes : 0ull; }
}

__global__ void __launch_bounds__(kMatThreads) ms_materialize_kernel(MsOutParams o)
{
    extern __shared__ __align__(16) unsigned char mat_raw[];
    const int tid = threadIdx.x;
    uint2 *tab = reinterpret_cast<uint2 *>(mat_raw);  // [kMatSlots][threads]: {depth, parent}
    const ull all = o.lanes >= 64 ? ~0ull : ((1ull << o.lanes) - 1);
    const long long tiles = (o.n + kMatThreads - 1) / kMatThreads;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t v = tile * kMatThreads + tid;
        if (v >= o.n) { continue; }
        const int64_t t = o.perm ? (int64_t)__ldg(&o.perm[v]) : v;
        const int64_t deg = __ldg(&o.off[v + 1]) - __ldg(&o.off[v]);
        const ull s = __ldcs(&o.seen[t]) & all;
        ull plane[4] = {0ull, 0ull, 0ull, 0ull};
        ull row_lanes = 0;  // lanes read from their rows in the write loop
        if (s) {
            const uint4 *rv = o.rec + t * kRecSlots;
            // the first two slots are read together with the count (they lie
            // in the vertex's record block whatever the count says)
            const uint4 x0 = __ldcs(&rv[0]), x1 = __ldcs(&rv[1]);
            const unsigned cnt = min(__ldcs(&o.rec_cnt[t]), kRecSlots);
            ull left = s;
            for (unsigned k0 = 0; k0 < cnt && left; k0 += 4) {
                uint4 x[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    x[j] = (k0 == 0 && j < 2) ? (j ? x1 : x0)
                                              : (k0 + j < cnt ? __ldcs(&rv[k0 + j])
                                                              : make_uint4(0, 0, 0, 0));
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const ull mask = k0 + j < cnt ? (((ull)x[j].y << 32) | x[j].x) & left : 0ull;
                    if (!mask) { continue; }
                    left &= ~mask;
                    const unsigned k = k0 + j;
                    // (a provider id out of range would only come from a
                    // broken record; it is passed through, not followed)
                    tab[k * kMatThreads + tid] = make_uint2(
                        x[j].w, o.iperm && x[j].z < o.n ? __ldg(&o.iperm[x[j].z]) : x[j].z);
                    mat_set_slot(plane, k, mask);
                }
            }
            // lanes past the records: their rows, four loads in flight; lanes
            // with the (depth, parent) pair of the previous one share its slot
            unsigned used = cnt;
            int32_t last_d = -2;
            uint32_t last_p = 0;
            unsigned last_k = kMatSlots;
            while (left) {
                int rr[4];
                int32_t dd[4];
                uint32_t pp[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    rr[j] = left ? __ffsll((long long)left) - 1 : -1;
                    left &= left ? left - 1 : 0ull;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    dd[j] = rr[j] >= 0 ? __ldcs(&o.depth[t * o.R + rr[j]]) : 0;
                    pp[j] = rr[j] >= 0 ? __ldcs(&o.parent[t * o.R + rr[j]]) : 0u;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (rr[j] < 0) { continue; }
                    if (dd[j] != last_d || pp[j] != last_p) {
                        last_d = dd[j];
                        last_p = pp[j];
                        last_k = kMatSlots;
                        if (used < kMatSlots) {
                            last_k = used++;
                            tab[last_k * kMatThreads + tid] = make_uint2(
                                (uint32_t)dd[j],
                                o.iperm && pp[j] < o.n ? __ldg(&o.iperm[pp[j]]) : pp[j]);
                        }
                    }
                    const ull bit = 1ull << rr[j];
                    if (last_k < kMatSlots) {
                        mat_set_slot(plane, last_k, bit);
                    } else {
                        row_lanes |= bit;
                    }
                }
            }
        }
        const int64_t unreached = deg != 0 ? -deg : -1;
        int32_t *dp = o.depth_out + v;
        int64_t *pq = o.parent_out + v;
        // two halves of 32 lanes, so that the planes shift as 32-bit words
        for (int h = 0; h < 2 && 32 * h < o.lanes; ++h) {
            uint32_t g = (uint32_t)(s >> (32 * h)), rw = (uint32_t)(row_lanes >> (32 * h));
            uint32_t q0 = (uint32_t)(plane[0] >> (32 * h)), q1 = (uint32_t)(plane[1] >> (32 * h));
            uint32_t q2 = (uint32_t)(plane[2] >> (32 * h)), q3 = (uint32_t)(plane[3] >> (32 * h));
            const int end = min(32, o.lanes - 32 * h);
            for (int j = 0; j < end; ++j) {
                const unsigned k = (q0 & 1u) | ((q1 & 1u) << 1) | ((q2 & 1u) << 2) | ((q3 & 1u) << 3);
                const uint2 e = tab[k * kMatThreads + tid];
                int32_t d = (int32_t)e.x;
                int64_t par = (int64_t)e.y;
                if (rw & 1u) {  // more pairs than slots: the lane's own row
                    const int r = 32 * h + j;
                    const uint32_t pr = __ldcs(&o.parent[t * o.R + r]);
                    d = __ldcs(&o.depth[t * o.R + r]);
                    par = (int64_t)(o.iperm && pr < o.n ? __ldg(&o.iperm[pr]) : pr);
                }
                const bool got = g & 1u;
                __stcs(dp, got ? d : -1);
                __stcs(pq, got ? par : unreached);
                dp += o.n;
                pq += o.n;
                g >>= 1;
                rw >>= 1;
                q0 >>= 1;
                q1 >>= 1;
                q2 >>= 1;
                q3 >>= 1;
            }
        }
    }
}

using MsKernel = void (*)(MsParams);

int ms_grid_for(int64_t items)
{
    int64_t b = (items + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

}  // namespace
}  // namespace bd

using namespace bd;

struct bd_msbfs {
    bd_graph *g = nullptr;
    int device = 0;
    int R = 64;          // lanes per group (= lane stride of the output rows)
    int groups = 1;      // result slices
    int max_roots = 64;
    bd_msbfs_opts opts{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ull *seen = nullptr;         // [groups][n]: a group's final words mark its valid lanes
    ull *F[3] = {nullptr, nullptr, nullptr};
    uint32_t *qs[3] = {nullptr, nullptr, nullptr};
    uint32_t *ql[3] = {nullptr, nullptr, nullptr};
    ull *qlb[3] = {nullptr, nullptr, nullptr};
    int32_t *depth = nullptr;    // [groups][n][R]
    uint32_t *parent = nullptr;  // [groups][n][R]
    uint4 *drec = nullptr;       // [groups][n][kRecSlots]
    uint32_t *drec_cnt = nullptr;  // [groups][n]
    uint32_t *done = nullptr;      // [n/32], rewritten for each group
    MsCtrl *ctrl = nullptr;
    bd_step *rec = nullptr;
    int64_t *d_sources = nullptr;         // [max_roots]
    unsigned long long *d_counts = nullptr;  // [groups][128]
    int64_t cap_large = 0;
    int grid = 0;
    int block = 512;
    int count = 0;  // roots in the last run
    std::vector<int64_t> sources;  // roots of the last run
    bool ran = false;
    PolicyBlob *policy = nullptr;  // device copy, or null
    uint32_t *heavy = nullptr;
    ull *heavy_cbase = nullptr;
    int64_t n_heavy = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_count = -1;
    bool graph_ok = true;
    bool frontier_clean = false;  // F is all zero (kernels leave it so)
    MsCtrl last{};
    std::vector<unsigned long long> counts;
    // opts.materialize: every root's results, written by each run
    int32_t *out_depth = nullptr;   // [max_roots][n]
    int64_t *out_parent = nullptr;  // [max_roots][n]
    int mat_grid = 0;
    // otherwise: one root's results, extracted when they are read
    void *xbuf = nullptr;           // 8 n bytes
};

namespace bd {
namespace {

MsKernel ms_pick(int block)
{
    switch (block) {
        case 256: return msbfs_kernel<256, 4>;
        case 1024: return msbfs_kernel<1024, 1>;
        default: return msbfs_kernel<512, 2>;
    }
}

MsParams ms_params(bd_msbfs *b, int group, int count)
{
    MsParams p{};
    p.off = traversal_off(b->g);
    p.adj = traversal_adj(b->g);
    p.perm = b->g->d_perm;
    p.done = b->done;
    p.n = b->g->n;
    p.m = b->g->m;
    p.reach = b->seen + group * b->g->n;
    for (int i = 0; i < 3; ++i) {
        p.F[i] = b->F[i];
        p.qs[i] = b->qs[i];
        p.ql[i] = b->ql[i];
        p.qlb[i] = b->qlb[i];
    }
    const int64_t slice = b->g->n * (int64_t)b->R;
    p.depth = b->depth + group * slice;
    p.drec = b->drec + group * b->g->n * (int64_t)kRecSlots;
    p.drec_cnt = b->drec_cnt + group * b->g->n;
    p.parent = b->parent + group * slice;
    p.R = b->R;
    p.all = count >= 64 ? ~0ull : ((1ull << count) - 1);
    p.ctrl = b->ctrl;
    p.rec = b->rec;
    p.rec_cap = kMsRecCap;
    p.alpha = b->opts.alpha;
    p.large_deg = (uint32_t)b->opts.large_degree;
    p.chunk = (uint32_t)b->opts.chunk_edges;
    p.prefix = b->opts.pull_prefix;
    p.spin_limit = b->opts.spin_limit;
    p.expected_ctas = (unsigned)b->grid;
    p.force_dir = b->opts.force_dir;
    p.policy = b->policy;
    p.heavy = b->heavy;
    p.heavy_cbase = b->heavy_cbase;
    p.n_heavy = b->n_heavy;
    p.heavy_deg = b->opts.heavy_degree;
    p.heavy_chunk = (uint32_t)b->opts.heavy_chunk;
    return p;
}

// Every lane of a finished group into its roots' output rows, and with
// opts.min_parent each root's smallest-parent tree on the caller's CSR.
bd_status ms_enqueue_materialize(bd_msbfs *b, int group, int count)
{
    const int64_t n = b->g->n;
    MsOutParams o{};
    const int64_t slice = n * (int64_t)b->R;
    o.depth = b->depth + group * slice;
    o.parent = b->parent + group * slice;
    o.rec = b->drec + group * n * (int64_t)kRecSlots;
    o.rec_cnt = b->drec_cnt + group * n;
    o.seen = b->seen + group * n;
    o.off = b->g->d_off;
    o.perm = b->g->d_perm;
    o.iperm = b->g->d_iperm;
    o.n = n;
    o.R = b->R;
    o.lanes = count;
    o.depth_out = b->out_depth + (int64_t)group * 64 * n;
    o.parent_out = b->out_parent + (int64_t)group * 64 * n;
    ms_materialize_kernel<<<b->mat_grid, kMatThreads, kMatSmem, b->stream>>>(o);
    BD_CUDA(cudaGetLastError());
    if (b->opts.min_parent) {
        for (int r = 0; r < count; ++r) {
            const int64_t row = ((int64_t)group * 64 + r) * n;
            BD_CUDA(launch_min_parent(b->g->d_off, b->g->d_adj, n, b->out_depth + row,
                                      b->out_parent + row, b->stream));
        }
    }
    return BD_OK;
}

// One group: clear (its seen words, the frontier words), init, the
// persistent kernel, the per-lane counts (and with opts.materialize the
// roots' output rows).
bd_status ms_enqueue_group(bd_msbfs *b, int group, int count)
{
    const int64_t n = b->g->n;
    BD_CUDA(cudaMemsetAsync(b->seen + group * n, 0, sizeof(ull) * n, b->stream));
    BD_CUDA(cudaMemsetAsync(b->drec_cnt + group * n, 0, sizeof(uint32_t) * n, b->stream));
    BD_CUDA(cudaMemcpyAsync(b->done, traversal_isolated(b->g), sizeof(uint32_t) * ((n + 31) / 32),
                            cudaMemcpyDeviceToDevice, b->stream));
    MsParams p = ms_params(b, group, count);
    ms_init_kernel<<<1, 1, 0, b->stream>>>(p, b->d_sources + group * 64, count);
    BD_CUDA(cudaGetLastError());
    void *args[] = {&p};
    BD_CUDA(cudaLaunchCooperativeKernel((const void *)ms_pick(b->block), dim3(b->grid),
                                        dim3(b->block), args, 0, b->stream));
    unsigned long long *dst = b->d_counts + 128 * group;
    BD_CUDA(cudaMemsetAsync(dst, 0, sizeof(unsigned long long) * 128, b->stream));
    ms_count_kernel<<<148 * 8, 256, 0, b->stream>>>(p.reach, p.off, n, p.all, count, dst);
    BD_CUDA(cudaGetLastError());
    if (b->opts.materialize) { BD_TRY(ms_enqueue_materialize(b, group, count)); }
    return BD_OK;
}

bd_status ms_enqueue_all(bd_msbfs *b, int count)
{
    BD_CUDA(cudaMemsetAsync(&b->ctrl->error, 0, sizeof(int), b->stream));
    for (int gi = 0; gi * 64 < count; ++gi) {
        BD_TRY(ms_enqueue_group(b, gi, std::min(64, count - gi * 64)));
    }
    return BD_OK;
}

// Captures the groups of a `count`-root call into one CUDA graph (once per
// count); falls back to plain stream launches if capture is refused.
bd_status ms_launch(bd_msbfs *b, int count)
{
    // The kernels leave F zero; after a first use or an error, zero
    // them here (outside any captured graph).
    if (!b->frontier_clean) {
        const int64_t n = b->g->n;
        for (int i = 0; i < 3; ++i) {
            BD_CUDA(cudaMemsetAsync(b->F[i], 0, sizeof(ull) * n, b->stream));
        }
    }
    b->frontier_clean = false;  // until this call is known to have finished cleanly
    if (b->opts.use_graph && b->graph_ok) {
        if (b->graph_count != count) {
            if (b->graph) {
                cudaGraphExecDestroy(b->graph);
                b->graph = nullptr;
            }
            cudaGraph_t gr = nullptr;
            if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                bd_status st = ms_enqueue_all(b, count);
                cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
                if (st == BD_OK && e == cudaSuccess &&
                    cudaGraphInstantiate(&b->graph, gr, 0) == cudaSuccess) {
                    b->graph_count = count;
                } else {
                    b->graph = nullptr;
                    b->graph_ok = false;
                }
                if (gr) { cudaGraphDestroy(gr); }
            } else {
                b->graph_ok = false;
            }
            cudaGetLastError();  // a refused capture leaves no sticky error
        }
        if (b->graph) {
            BD_CUDA(cudaGraphLaunch(b->graph, b->stream));
            return BD_OK;
        }
    }
    return ms_enqueue_all(b, count);
}

void ms_free(bd_msbfs *b)
{
    if (!b) { return; }
    cudaSetDevice(b->device);
    if (b->stream) { cudaStreamSynchronize(b->stream); }
    if (b->graph) { cudaGraphExecDestroy(b->graph); }
    cudaFree(b->seen);
    cudaFree(b->done);
    for (int i = 0; i < 3; ++i) {
        cudaFree(b->F[i]);
        cudaFree(b->qs[i]);
        cudaFree(b->ql[i]);
        cudaFree(b->qlb[i]);
    }
    cudaFree(b->depth);
    cudaFree(b->parent);
    cudaFree(b->drec);
    cudaFree(b->drec_cnt);
    cudaFree(b->ctrl);
    cudaFree(b->rec);
    cudaFree(b->d_sources);
    cudaFree(b->d_counts);
    cudaFree(b->policy);
    cudaFree(b->heavy);
    cudaFree(b->heavy_cbase);
    cudaFree(b->out_depth);
    cudaFree(b->out_parent);
    cudaFree(b->xbuf);
    if (b->ev0) { cudaEventDestroy(b->ev0); }
    if (b->ev1) { cudaEventDestroy(b->ev1); }
    if (b->stream) { cudaStreamDestroy(b->stream); }
    delete b;
}

bd_status ms_check_root(bd_msbfs *b, int32_t root_index)
{
    if (!b->ran) { return BD_ERR_STATE; }
    if (root_index < 0 || root_index >= b->count) { return BD_ERR_RANGE; }
    return BD_OK;
}

// One root's depths or parents (caller ids, reference encoding) into a
// device buffer of n entries, queued on the handle's stream.
cudaError_t ms_extract_async(bd_msbfs *b, int32_t root_index, int32_t *d_depth, int64_t *d_parent)
{
    const int64_t n = b->g->n;
    const int group = root_index / 64, lane = root_index % 64;
    const int64_t slice = n * (int64_t)b->R;
    ms_extract_kernel<<<ms_grid_for(n), 256, 0, b->stream>>>(
        b->depth + group * slice, b->parent + group * slice, b->drec + group * n * (int64_t)kRecSlots,
        b->drec_cnt + group * n, b->seen + group * n, b->g->d_off, n, b->R, lane, b->g->d_perm,
        b->g->d_iperm, d_depth, d_parent);
    return cudaGetLastError();
}

// One root's depths or parents (caller ids, reference encoding) in device
// memory: its materialized row, or extracted into the handle's buffer.
bd_status ms_root_device(bd_msbfs *b, int32_t root_index, bool want_depth, const void **out)
{
    BD_TRY(ms_check_root(b, root_index));
    BD_CUDA(cudaSetDevice(b->device));
    const int64_t n = b->g->n;
    if (b->opts.materialize) {
        *out = want_depth ? (const void *)(b->out_depth + (int64_t)root_index * n)
                          : (const void *)(b->out_parent + (int64_t)root_index * n);
        return BD_OK;
    }
    BD_CUDA(ms_extract_async(b, root_index, want_depth ? static_cast<int32_t *>(b->xbuf) : nullptr,
                             want_depth ? nullptr : static_cast<int64_t *>(b->xbuf)));
    *out = b->xbuf;
    return BD_OK;
}

bd_status ms_extract(bd_msbfs *b, int32_t root_index, int32_t *depth, int64_t *parent)
{
    const void *src = nullptr;
    BD_TRY(ms_root_device(b, root_index, depth != nullptr, &src));
    const size_t bytes = depth ? sizeof(int32_t) * b->g->n : sizeof(int64_t) * b->g->n;
    BD_CUDA(cudaMemcpyAsync(depth ? (void *)depth : (void *)parent, src, bytes,
                            cudaMemcpyDeviceToHost, b->stream));
    BD_CUDA(cudaStreamSynchronize(b->stream));
    return BD_OK;
}

}  // namespace
}  // namespace bd

extern "C" {

void bd_msbfs_default_opts(bd_msbfs_opts *o)
{
    if (!o) { return; }
    memset(o, 0, sizeof(*o));
    o->alpha = 4;
    o->force_dir = -1;
    o->use_graph = 1;
}

bd_status bd_msbfs_create(bd_graph *g, int32_t max_roots, const bd_msbfs_opts *opts,
                          bd_msbfs **out)
{
    if (!g || !out || max_roots < 1 || max_roots > 65536) { return BD_ERR_INVALID; }
    bd_msbfs_opts o;
    bd_msbfs_default_opts(&o);
    if (opts) { o = *opts; }
    if (o.alpha <= 0 || o.force_dir < -1 || o.force_dir > 1) { return BD_ERR_INVALID; }
    if (o.block_size == 0) { o.block_size = 512; }
    if (o.block_size != 256 && o.block_size != 512 && o.block_size != 1024) { return BD_ERR_INVALID; }
    if (o.large_degree <= 0) { o.large_degree = 32; }
    if (o.large_degree > (1 << 20)) { return BD_ERR_INVALID; }
    if (o.chunk_edges <= 0) { o.chunk_edges = 256; }
    if (o.pull_prefix <= 0) { o.pull_prefix = 16; }
    if (o.heavy_degree <= 0) { o.heavy_degree = 4096; }
    if (o.heavy_chunk <= 0) { o.heavy_chunk = 2048; }
    if (o.spin_limit <= 0) { o.spin_limit = kMsDefaultSpin; }
    if (o.materialize < 0 || o.materialize > 1 || o.min_parent < 0 || o.min_parent > 1) {
        return BD_ERR_INVALID;
    }
    if (o.min_parent) { o.materialize = 1; }
    if (g->n > (int64_t)UINT32_MAX) { return BD_ERR_LIMIT; }
    BD_TRY(ensure_device());
    auto *b = new bd_msbfs();
    b->g = g;
    b->device = current_device();
    b->max_roots = max_roots;
    b->R = std::min(64, (int)max_roots);
    b->groups = (max_roots + 63) / 64;
    b->opts = o;
    b->block = o.block_size;
    const int64_t n = g->n;
    b->cap_large = std::min<int64_t>(n, g->arcs / o.large_degree + 1);
    auto fail = [&](bd_status st) { ms_free(b); return st; };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
        return fail(BD_ERR_CUDA);
    }
    const size_t slots = (size_t)n * b->R * b->groups;
    bool ok = cudaMalloc(&b->seen, sizeof(ull) * n * b->groups) == cudaSuccess &&
              cudaMalloc(&b->done, sizeof(uint32_t) * ((n + 31) / 32)) == cudaSuccess &&
              cudaMalloc(&b->depth, sizeof(int32_t) * slots) == cudaSuccess &&
              cudaMalloc(&b->parent, sizeof(uint32_t) * slots) == cudaSuccess &&
              cudaMalloc(&b->drec, sizeof(uint4) * (size_t)n * kRecSlots * b->groups) == cudaSuccess &&
              cudaMalloc(&b->drec_cnt, sizeof(uint32_t) * (size_t)n * b->groups) == cudaSuccess &&
              cudaMalloc(&b->ctrl, sizeof(MsCtrl)) == cudaSuccess &&
              cudaMalloc(&b->rec, sizeof(bd_step) * kMsRecCap) == cudaSuccess &&
              cudaMalloc(&b->d_sources, sizeof(int64_t) * 64 * b->groups) == cudaSuccess &&
              cudaMalloc(&b->d_counts, sizeof(unsigned long long) * 128 * b->groups) == cudaSuccess;
    for (int i = 0; i < 3 && ok; ++i) {
        ok = cudaMalloc(&b->F[i], sizeof(ull) * n) == cudaSuccess &&
             cudaMalloc(&b->qs[i], sizeof(uint32_t) * n) == cudaSuccess &&
             cudaMalloc(&b->ql[i], sizeof(uint32_t) * b->cap_large) == cudaSuccess &&
             cudaMalloc(&b->qlb[i], sizeof(ull) * b->cap_large) == cudaSuccess;
    }
    if (ok && o.materialize) {
        const size_t rows = (size_t)n * (size_t)max_roots;
        ok = cudaMalloc(&b->out_depth, sizeof(int32_t) * rows) == cudaSuccess &&
             cudaMalloc(&b->out_parent, sizeof(int64_t) * rows) == cudaSuccess;
    } else if (ok) {
        ok = cudaMalloc(&b->xbuf, sizeof(int64_t) * n) == cudaSuccess;
    }
    if (!ok) { return fail(BD_ERR_OOM); }
    if (o.materialize) {
        int per_sm = 0, sms = 0;
        if (cudaFuncSetAttribute(ms_materialize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kMatSmem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_materialize_kernel,
                                                          kMatThreads, kMatSmem) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ||
            per_sm < 1) {
            return fail(BD_ERR_CUDA);
        }
        b->mat_grid = per_sm * sms;
    }
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)ms_pick(b->block),
                                                      b->block, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ||
        per_sm < 1) {
        return fail(BD_ERR_CUDA);
    }
    b->grid = per_sm * sms;
    // heavy vertices and their chunk prefix sums (host, once per handle)
    {
        std::vector<int64_t> off(n + 1);
        if (cudaMemcpy(off.data(), traversal_off(g), sizeof(int64_t) * (n + 1),
                       cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
            return fail(BD_ERR_CUDA);
        }
        std::vector<uint32_t> hv;
        std::vector<ull> hc(1, 0);
        for (int64_t v = 0; v < n; ++v) {
            const int64_t d = off[v + 1] - off[v];
            if (d > o.heavy_degree) {
                hv.push_back((uint32_t)v);
                hc.push_back(hc.back() + (ull)((d + o.heavy_chunk - 1) / o.heavy_chunk));
            }
        }
        b->n_heavy = (int64_t)hv.size();
        if (cudaMalloc(&b->heavy, sizeof(uint32_t) * std::max<size_t>(hv.size(), 1)) != cudaSuccess ||
            cudaMalloc(&b->heavy_cbase, sizeof(ull) * hc.size()) != cudaSuccess ||
            (!hv.empty() && cudaMemcpy(b->heavy, hv.data(), sizeof(uint32_t) * hv.size(),
                                       cudaMemcpyHostToDevice) != cudaSuccess) ||
            cudaMemcpy(b->heavy_cbase, hc.data(), sizeof(ull) * hc.size(), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            return fail(BD_ERR_OOM);
        }
    }
    *out = b;
    return BD_OK;
}

bd_status bd_msbfs_run(bd_msbfs *b, const int64_t *sources, int32_t count, bd_run_stats *stats)
{
    if (!b || !sources || count < 1 || count > b->max_roots) { return BD_ERR_INVALID; }
    for (int i = 0; i < count; ++i) {
        if (sources[i] < 0 || sources[i] >= b->g->n) { return BD_ERR_RANGE; }
    }
    BD_CUDA(cudaSetDevice(b->device));
    // group g's sources start at d_sources + 64 g
    std::vector<int64_t> padded((size_t)64 * b->groups, 0);
    for (int i = 0; i < count; ++i) { padded[(size_t)(i / 64) * 64 + i % 64] = sources[i]; }
    BD_CUDA(cudaMemcpyAsync(b->d_sources, padded.data(), sizeof(int64_t) * padded.size(),
                            cudaMemcpyHostToDevice, b->stream));
    BD_CUDA(cudaEventRecord(b->ev0, b->stream));
    BD_TRY(ms_launch(b, count));
    BD_CUDA(cudaEventRecord(b->ev1, b->stream));
    const int used = (count + 63) / 64;
    b->counts.assign((size_t)128 * used, 0);
    BD_CUDA(cudaMemcpyAsync(b->counts.data(), b->d_counts, sizeof(unsigned long long) * 128 * used,
                            cudaMemcpyDeviceToHost, b->stream));
    BD_CUDA(cudaMemcpyAsync(&b->last, b->ctrl, sizeof(MsCtrl), cudaMemcpyDeviceToHost, b->stream));
    BD_CUDA(cudaStreamSynchronize(b->stream));
    b->count = count;
    b->sources.assign(sources, sources + count);
    b->ran = true;
    b->frontier_clean = b->last.error == 0;
    if (b->last.error) { return (bd_status)b->last.error; }
    if (stats) {
        float ms = 0.f;
        BD_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        stats->ms = ms;
        stats->num_steps = b->last.st.step;
        int64_t edges = 0, reached = 0;
        for (int i = 0; i < count; ++i) {
            const size_t base = (size_t)(i / 64) * 128;
            edges += (int64_t)(b->counts[base + 64 + i % 64] / 2);
            reached += (int64_t)b->counts[base + i % 64];
        }
        stats->traversed_edges = edges;
        stats->reached = reached;
        stats->top_down_steps = b->last.st.push_steps;
        stats->bottom_up_steps = b->last.st.pull_steps;
    }
    return BD_OK;
}

bd_status bd_msbfs_get_depths(bd_msbfs *b, int32_t root_index, int32_t *depth)
{
    if (!b || !depth) { return BD_ERR_INVALID; }
    return ms_extract(b, root_index, depth, nullptr);
}

bd_status bd_msbfs_get_parents(bd_msbfs *b, int32_t root_index, int64_t *parent)
{
    if (!b || !parent) { return BD_ERR_INVALID; }
    return ms_extract(b, root_index, nullptr, parent);
}

// hybrid_bfs::check of one root's parents, extracted and checked in HBM
// (bd_check.cu).
bd_status bd_msbfs_check(bd_msbfs *b, int32_t root_index, int32_t *ok)
{
    if (!b || !ok) { return BD_ERR_INVALID; }
    const void *parent = nullptr;
    BD_TRY(ms_root_device(b, root_index, false, &parent));
    BD_CUDA(cudaStreamSynchronize(b->stream));
    return check_parents_device(b->g, b->sources[root_index], static_cast<const int64_t *>(parent),
                                ok, nullptr);
}

// Borrowed device pointers to one root's materialized results.
bd_status bd_msbfs_device_results(bd_msbfs *b, int32_t root_index, const int32_t **depth,
                                  const int64_t **parent)
{
    if (!b) { return BD_ERR_INVALID; }
    if (!b->opts.materialize) { return BD_ERR_STATE; }
    const void *d = nullptr, *p = nullptr;
    BD_TRY(ms_root_device(b, root_index, true, &d));
    BD_TRY(ms_root_device(b, root_index, false, &p));
    if (depth) { *depth = static_cast<const int32_t *>(d); }
    if (parent) { *parent = static_cast<const int64_t *>(p); }
    return BD_OK;
}

bd_status bd_msbfs_count_traversed_edges(bd_msbfs *b, int32_t root_index, int64_t *edges,
                                         int64_t *reached)
{
    if (!b) { return BD_ERR_INVALID; }
    BD_TRY(ms_check_root(b, root_index));
    const size_t base = (size_t)(root_index / 64) * 128;
    if (edges) { *edges = (int64_t)(b->counts[base + 64 + root_index % 64] / 2); }
    if (reached) { *reached = (int64_t)b->counts[base + root_index % 64]; }
    return BD_OK;
}

bd_status bd_msbfs_get_steps(bd_msbfs *b, bd_step *steps, int64_t capacity, int64_t *count)
{
    if (!b || !count || capacity < 0 || (!steps && capacity)) { return BD_ERR_INVALID; }
    if (!b->ran) { return BD_ERR_STATE; }
    const int64_t have = std::min<int64_t>(b->last.st.step, kMsRecCap);
    const int64_t take = std::min(have, capacity);
    if (take) {
        BD_CUDA(cudaSetDevice(b->device));
        BD_CUDA(cudaMemcpy(steps, b->rec, sizeof(bd_step) * take, cudaMemcpyDeviceToHost));
    }
    *count = have;
    return BD_OK;
}

bd_status bd_msbfs_set_policy(bd_msbfs *b, const float *params, const float *mean,
                              const float *inv_std, const float *lo, const float *hi, float margin)
{
    if (!b) { return BD_ERR_INVALID; }
    BD_CUDA(cudaSetDevice(b->device));
    if (!params || isinf(margin)) {  // +inf margin: the rule decides, nothing is evaluated
        cudaFree(b->policy);
        b->policy = nullptr;
        b->graph_count = -1;  // captured launches hold the old pointer
        return BD_OK;
    }
    PolicyBlob blob;
    BD_TRY(policy_blob(params, mean, inv_std, lo, hi, margin, &blob));
    if (!b->policy) {
        BD_CUDA(cudaMalloc(&b->policy, sizeof(PolicyBlob)));
        b->graph_count = -1;
    }
    BD_CUDA(cudaMemcpy(b->policy, &blob, sizeof(PolicyBlob), cudaMemcpyHostToDevice));
    return BD_OK;
}

bd_status bd_msbfs_destroy(bd_msbfs *b)
{
    if (!b) { return BD_ERR_INVALID; }
    ms_free(b);
    return BD_OK;
}

}  // extern "C"
