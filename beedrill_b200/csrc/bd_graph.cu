// bd_graph.cu -- graphs in HBM: el64 loading, CSR construction, the seeded
// RMAT generator, disjoint unions, the lcg root picker and graph::check.
//
// Reference counterparts:
//   edge_list.cc:20-89 / dist_edge_list.cc:50-143  el64 header + body
//   graph_base.h:335-436                          CSR in insertion order
//   graph_base.h:110-134                          graph::check
//   generator/rmat_generator.h:91-193,
//   generator/rmat_dataset_dump.cc:30-57          RMAT edges + post-processing
//   hybrid_bfs_main.cc:136-144, lcg.h:4-32        root picker
//
// Graph construction is off the BFS hot path; it uses CUB's radix sort,
// unique and scan where a sort or scan is needed.
#include <cub/cub.cuh>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bd_internal.h"

namespace bd {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kMaxAttempts = 4096;  // self-loop re-rolls per edge

int grid_for(int64_t items, int threads = kThreads)
{
    int64_t b = (items + threads - 1) / threads;
    if (b < 1) { b = 1; }
    if (b > 148 * 64) { b = 148 * 64; }  // grid-stride beyond this
    return (int)b;
}

// RAII device buffer for temporaries of the construction pipeline.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t count = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { if (p) { cudaFree(p); } }
    cudaError_t alloc(size_t n)
    {
        count = n;
        return cudaMalloc(&p, sizeof(T) * (n ? n : 1));
    }
    T *release() { T *q = p; p = nullptr; return q; }
    void reset()
    {
        if (p) { cudaFree(p); }
        p = nullptr;
    }
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]);
        uint32_t lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]);
        uint32_t lo1 = 0xCD9E8D57u * c[2];
        uint32_t n0 = hi1 ^ c[1] ^ k0;
        uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Counter-based uniform stream of one (edge, attempt): draw j is half of
// Philox block j/2, top 53 bits scaled into [0, 1).
struct RmatStream {
    uint32_t i_lo, i_hi, t, k0, k1;
    uint32_t block[4];
    uint32_t j = 0;
    __device__ double next()
    {
        if ((j & 1) == 0) {
            block[0] = i_lo;
            block[1] = i_hi;
            block[2] = t;
            block[3] = j >> 1;
            philox(block, k0, k1);
        }
        uint64_t w = (j & 1) ? (((uint64_t)block[2] << 32) | block[3])
                             : (((uint64_t)block[0] << 32) | block[1]);
        ++j;
        return __dmul_rn(__ull2double_rn(w >> 11), 1.0 / 9007199254740992.0);
    }
};

// One attempt of rmat_generator.h:91-140.  Every double operation is an
// explicitly rounded intrinsic so no multiply-add is contracted: the result
// is bit-identical to the step-by-step rounded host restatement.
__device__ void rmat_attempt(int scale, double a, double b, double c, double d, uint64_t seed,
                             int64_t i, uint32_t t, int64_t *src, int64_t *dst)
{
    RmatStream rs;
    rs.i_lo = (uint32_t)(uint64_t)i;
    rs.i_hi = (uint32_t)((uint64_t)i >> 32);
    rs.t = t;
    rs.k0 = (uint32_t)seed;
    rs.k1 = (uint32_t)(seed >> 32);
    double A = a, B = b, C = c, D = d;
    int64_t si = 0, sj = 0;
    int64_t bit = (int64_t)1 << (scale - 1);
    for (;;) {
        double r = rs.next();
        if (r > A) {
            double ab = __dadd_rn(A, B);
            if (r <= ab) {
                sj |= bit;
            } else if (r <= __dadd_rn(ab, C)) {
                si |= bit;
            } else {
                sj |= bit;
                si |= bit;
            }
        }
        if (bit == 1) { break; }
        A = __dmul_rn(A, __ddiv_rn(__dadd_rn(9.5, rs.next()), 10.0));
        B = __dmul_rn(B, __ddiv_rn(__dadd_rn(9.5, rs.next()), 10.0));
        C = __dmul_rn(C, __ddiv_rn(__dadd_rn(9.5, rs.next()), 10.0));
        D = __dmul_rn(D, __ddiv_rn(__dadd_rn(9.5, rs.next()), 10.0));
        double norm = __ddiv_rn(1.0, __dadd_rn(__dadd_rn(__dadd_rn(A, B), C), D));
        A = __dmul_rn(A, norm);
        B = __dmul_rn(B, norm);
        C = __dmul_rn(C, norm);
        D = __dsub_rn(1.0, __dadd_rn(__dadd_rn(A, B), C));
        bit >>= 1;
    }
    *src = si;
    *dst = sj;
}

// Generated edge i -> flipped (src < dst) packed key src << scale | dst.
__global__ void rmat_keys_kernel(int scale, int64_t num_edges, double a, double b, double c,
                                 double d, uint64_t seed, uint64_t *keys)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < num_edges;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t s = 0, t = 0;
        for (uint32_t att = 0; att < kMaxAttempts; ++att) {
            rmat_attempt(scale, a, b, c, d, seed, i, att, &s, &t);
            if (s != t) { break; }
        }
        uint64_t lo = (uint64_t)(s < t ? s : t), hi = (uint64_t)(s < t ? t : s);
        keys[i] = (lo << scale) | hi;
    }
}

// ---------------------------------------------------------------------------
// The reference generator's own random stream (generator/rmat_generator.h,
// generator/prng_engine.hpp), so that edge streams can equal the
// reference's bit for bit.
//
// sitmo::prng_engine (M.A. van den Berg, MIT licence, vendored by the
// reference) is a counter-mode generator: 32-bit output t is half of
// Threefish-256 (Skein 1.3 specification) reduced to 20 rounds, tweak zero,
// key (seed, 0, 0, 0), applied to the 256-bit counter (t / 8, 0, 0, 0) --
// the low half of 64-bit word (t % 8) / 2 when t is even, the high half when
// odd.  Seeding encrypts counter 0, and discard(z) moves the counter, so
// any position of the stream is reached directly.
//
// The reference draws its uniform doubles through libstdc++ (GCC 13)
// std::uniform_real_distribution<double>(0, 1), which calls
// std::generate_canonical<double, 53>: two engine outputs u0, u1 combined
// as (u0 + u1 * 2^32) / 2^64 in double arithmetic (one rounding, at the
// sum), with 1 - 2^-53 in place of a result of 1.
// ---------------------------------------------------------------------------
constexpr uint64_t kThreefishParity = 0x1BD11BDAA9FC1A22ull;

__host__ __device__ __forceinline__ uint64_t rotl64(uint64_t x, int r)
{
    return (x << r) | (x >> (64 - r));
}

// Threefish-256, 20 rounds, zero tweak: the block of counter `ctr` under key
// (key0, 0, 0, 0).  Rotation amounts of round r are kRot[r % 8]; words are
// paired (0,1),(2,3) on even rounds and (0,3),(2,1) on odd rounds (the
// Threefish-256 word permutation); subkey s is injected before rounds
// 4s and after the last round.
__device__ __forceinline__ void threefish20(uint64_t key0, uint64_t ctr, uint64_t o[4])
{
    const uint64_t k[5] = {key0, 0, 0, 0, kThreefishParity ^ key0};
    const int rot[8][2] = {{14, 16}, {52, 57}, {23, 40}, {5, 37},
                           {25, 33}, {46, 12}, {58, 22}, {32, 32}};
    uint64_t x0 = ctr, x1 = 0, x2 = 0, x3 = 0;
#pragma unroll
    for (int r = 0; r < 20; ++r) {
        if ((r & 3) == 0) {
            const int sk = r >> 2;
            x0 += k[sk % 5];
            x1 += k[(sk + 1) % 5];
            x2 += k[(sk + 2) % 5];
            x3 += k[(sk + 3) % 5] + (uint64_t)sk;
        }
        if ((r & 1) == 0) {
            x0 += x1;
            x1 = rotl64(x1, rot[r & 7][0]) ^ x0;
            x2 += x3;
            x3 = rotl64(x3, rot[r & 7][1]) ^ x2;
        } else {
            x0 += x3;
            x3 = rotl64(x3, rot[r & 7][0]) ^ x0;
            x2 += x1;
            x1 = rotl64(x1, rot[r & 7][1]) ^ x2;
        }
    }
    o[0] = x0 + k[0];
    o[1] = x1 + k[1];
    o[2] = x2 + k[2];
    o[3] = x3 + k[3] + 5;
}

// A reader of the stream from any position.
struct SitmoStream {
    uint64_t key0, block;
    uint32_t word;  // next output within the block, 0..8
    uint64_t o[4];
    __device__ void seek(uint64_t t)
    {
        block = t >> 3;
        word = (uint32_t)(t & 7);
        threefish20(key0, block, o);
    }
    __device__ uint32_t next()
    {
        if (word == 8) {
            ++block;
            threefish20(key0, block, o);
            word = 0;
        }
        const uint64_t w = o[word >> 1];
        const uint32_t u = (word & 1) ? (uint32_t)(w >> 32) : (uint32_t)w;
        ++word;
        return u;
    }
    // generate_canonical<double, 53> over two outputs
    __device__ double uniform()
    {
        const double lo = (double)next();
        const double hi = (double)next();
        const double sum = __dadd_rn(lo, __dmul_rn(hi, 4294967296.0));
        const double r = __dmul_rn(sum, 5.42101086242752217e-20);  // 2^-64
        return r >= 1.0 ? 0.99999999999999988898 : r;               // 1 - 2^-53
    }
};

// Engine outputs per edge: next_edge draws 5 uniforms per level but the
// last, which draws 1 (rmat_generator.h:80-89), two outputs per uniform.
__host__ __device__ __forceinline__ uint64_t sitmo_outputs_per_edge(int scale)
{
    return 2ull * (5ull * (uint64_t)(scale - 1) + 1ull);
}

// next_edge (rmat_generator.h:91-140) on the reference stream: the same
// quadrant recursion as rmat_attempt with the uniforms drawn from `rs`.
__device__ void rmat_sitmo_edge(int scale, double a, double b, double c, double d,
                                SitmoStream &rs, int64_t *src, int64_t *dst)
{
    double A = a, B = b, C = c, D = d;
    int64_t si = 0, sj = 0;
    int64_t bit = (int64_t)1 << (scale - 1);
    for (;;) {
        const double r = rs.uniform();
        if (r > A) {
            const double ab = __dadd_rn(A, B);
            if (r <= ab) {
                sj |= bit;
            } else if (r <= __dadd_rn(ab, C)) {
                si |= bit;
            } else {
                sj |= bit;
                si |= bit;
            }
        }
        if (bit == 1) { break; }
        A = __dmul_rn(A, __ddiv_rn(__dadd_rn(9.5, rs.uniform()), 10.0));
        B = __dmul_rn(B, __ddiv_rn(__dadd_rn(9.5, rs.uniform()), 10.0));
        C = __dmul_rn(C, __ddiv_rn(__dadd_rn(9.5, rs.uniform()), 10.0));
        D = __dmul_rn(D, __ddiv_rn(__dadd_rn(9.5, rs.uniform()), 10.0));
        const double norm = __ddiv_rn(1.0, __dadd_rn(__dadd_rn(__dadd_rn(A, B), C), D));
        A = __dmul_rn(A, norm);
        B = __dmul_rn(B, norm);
        C = __dmul_rn(C, norm);
        D = __dsub_rn(1.0, __dadd_rn(__dadd_rn(A, B), C));
        bit >>= 1;
    }
    *src = si;
    *dst = sj;
}

// Edge i of rmat_fill (rmat_generator.h:145-175): drawn from stream position
// i x outputs-per-edge, as the reference's discard() places it.  Self loops
// are flagged for the serial re-roll.
__global__ void rmat_sitmo_kernel(int scale, int64_t num_edges, double a, double b, double c,
                                  double d, uint32_t seed, int64_t *src, int64_t *dst,
                                  uint8_t *self_loop)
{
    const uint64_t per_edge = sitmo_outputs_per_edge(scale);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < num_edges;
         i += (int64_t)gridDim.x * blockDim.x) {
        SitmoStream rs;
        rs.key0 = seed;
        rs.seek((uint64_t)i * per_edge);
        int64_t s = 0, t = 0;
        rmat_sitmo_edge(scale, a, b, c, d, rs, &s, &t);
        src[i] = s;
        dst[i] = t;
        self_loop[i] = s == t ? 1 : 0;
    }
}

// The serial re-roll of rmat_fill (rmat_generator.h:177-189): self loops in
// edge order draw whole edges from the stream after the last generated edge
// until they are not self loops.  One thread: the order is the point, and
// self loops are few (about (a + d)^scale of the edges).  `list` holds the
// self loops' edge indices in ascending order.
__global__ void rmat_sitmo_reroll_kernel(int scale, int64_t num_edges, double a, double b,
                                         double c, double d, uint32_t seed, const int64_t *list,
                                         const int64_t *count, int64_t *src, int64_t *dst,
                                         int *error)
{
    SitmoStream rs;
    rs.key0 = seed;
    rs.seek((uint64_t)num_edges * sitmo_outputs_per_edge(scale));
    const int64_t total = *count;
    uint64_t draws = 0;
    for (int64_t k = 0; k < total; ++k) {
        const int64_t i = list[k];
        int64_t s = 0, t = 0;
        do {
            if (++draws > (uint64_t)kMaxAttempts * (uint64_t)(total + 1)) {
                *error = 1;  // a degenerate A-D that only yields self loops
                return;
            }
            rmat_sitmo_edge(scale, a, b, c, d, rs, &s, &t);
        } while (s == t);
        src[i] = s;
        dst[i] = t;
    }
}

// Generated edge k -> flipped (src < dst) packed key src << scale | dst.
__global__ void flip_keys_kernel(const int64_t *src, const int64_t *dst, int64_t num_edges,
                                 int scale, uint64_t *keys)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < num_edges;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t s = (uint64_t)src[i], t = (uint64_t)dst[i];
        keys[i] = s < t ? (s << scale) | t : (t << scale) | s;
    }
}

__global__ void iota_kernel(int64_t count, int64_t *out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        out[i] = i;
    }
}

// Sort key of item idx in a permutation domain (vertex relabel / shuffle).
__device__ __forceinline__ uint64_t perm_key(uint64_t seed, uint64_t idx, uint32_t tag)
{
    uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), tag, 0u};
    philox(c, (uint32_t)seed ^ 0xA5A5A5A5u, (uint32_t)(seed >> 32) ^ 0x3C3C3C3Cu);
    return ((uint64_t)c[0] << 32) | c[1];
}

constexpr uint32_t kTagRelabel = 0x52454C42u;  // "RELB"
constexpr uint32_t kTagShuffle = 0x53485546u;  // "SHUF"

__global__ void perm_keys_kernel(uint64_t seed, uint32_t tag, int64_t count, uint64_t *keys,
                                 uint32_t *idx)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = perm_key(seed, (uint64_t)i, tag);
        if (idx) { idx[i] = (uint32_t)i; }
    }
}

__global__ void edge_shuffle_keys_kernel(uint64_t seed, int64_t count, uint64_t *keys)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = perm_key(seed, (uint64_t)i, kTagShuffle);
    }
}

__global__ void scatter_rank_kernel(const uint32_t *sorted_v, int64_t n, uint32_t *new_id)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        new_id[sorted_v[k]] = (uint32_t)k;
    }
}

// Packed key k -> edge (new_id of src, new_id of dst); new_id null: the
// generator's own ids.
__global__ void unpack_relabel_kernel(const uint64_t *packed, int64_t m, int scale,
                                      const uint32_t *new_id, int64_t *src, int64_t *dst)
{
    const uint64_t mask = (1ull << scale) - 1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x) {
        uint64_t p = packed[k];
        src[k] = new_id ? (int64_t)new_id[p >> scale] : (int64_t)(p >> scale);
        dst[k] = new_id ? (int64_t)new_id[p & mask] : (int64_t)(p & mask);
    }
}

// ---------------------------------------------------------------------------
// 2-D grid with 4-neighbour edges, a seeded fraction deleted
// ---------------------------------------------------------------------------
constexpr uint32_t kTagGrid = 0x47524944u;  // "GRID"

// Edge e: e < rows*(cols-1) is horizontal (r, c)-(r, c+1) with
// r = e / (cols-1), c = e % (cols-1); the rest are vertical (r, c)-(r+1, c).
// Edge e is kept when the top 53 bits of its Philox key, as a fraction of
// 2^53, are >= delete_frac.
__global__ void grid_keep_kernel(int64_t rows, int64_t cols, double delete_frac, uint64_t seed,
                                 int64_t total, int *keep)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = perm_key(seed, (uint64_t)e, kTagGrid);
        const double u = __dmul_rn(__ull2double_rn(k >> 11), 1.0 / 9007199254740992.0);
        keep[e] = u >= delete_frac ? 1 : 0;
    }
}

__global__ void grid_emit_kernel(int64_t rows, int64_t cols, int64_t total, const int *keep,
                                 const int64_t *pos, int64_t *src, int64_t *dst)
{
    const int64_t horiz = rows * (cols - 1);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        if (!keep[e]) { continue; }
        int64_t a, b;
        if (e < horiz) {
            const int64_t r = e / (cols - 1), c = e % (cols - 1);
            a = r * cols + c;
            b = a + 1;
        } else {
            const int64_t f = e - horiz;
            const int64_t r = f / cols, c = f % cols;
            a = r * cols + c;
            b = a + cols;
        }
        src[pos[e]] = a;
        dst[pos[e]] = b;
    }
}

// ---------------------------------------------------------------------------
// CSR construction
// ---------------------------------------------------------------------------

// Arc 2k = (src_k -> dst_k), arc 2k+1 = (dst_k -> src_k): the insertion
// order of graph_base.h:423-427.  Flags endpoints outside [0, n).
__global__ void make_arcs_kernel(const int64_t *src, const int64_t *dst, int64_t m, int64_t n,
                                 uint32_t *key, uint32_t *val, int *bad)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t s = src[k], d = dst[k];
        if (s < 0 || s >= n || d < 0 || d >= n) {
            atomicExch(bad, 1);
            s = 0;
            d = 0;
        }
        key[2 * k] = (uint32_t)s;
        val[2 * k] = (uint32_t)d;
        key[2 * k + 1] = (uint32_t)d;
        val[2 * k + 1] = (uint32_t)s;
    }
}

__global__ void make_sorted_arcs_kernel(const int64_t *src, const int64_t *dst, int64_t m,
                                        int64_t n, uint64_t *key, int *bad)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t s = src[k], d = dst[k];
        if (s < 0 || s >= n || d < 0 || d >= n) {
            atomicExch(bad, 1);
            s = 0;
            d = 0;
        }
        key[2 * k] = ((uint64_t)s << 32) | (uint64_t)d;
        key[2 * k + 1] = ((uint64_t)d << 32) | (uint64_t)s;
    }
}

__global__ void split_sorted_arcs_kernel(const uint64_t *key, int64_t arcs, uint32_t *src32,
                                         uint32_t *adj)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < arcs;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = key[i];
        src32[i] = (uint32_t)(k >> 32);
        adj[i] = (uint32_t)k;
    }
}

// offsets[v] = first arc whose (sorted) source is >= v.
__global__ void offsets_from_sorted_kernel(const uint32_t *sorted_src, int64_t arcs, int64_t n,
                                           int64_t *off)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= arcs;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t prev = i == 0 ? -1 : (int64_t)sorted_src[i - 1];
        int64_t cur = i == arcs ? n : (int64_t)sorted_src[i];
        for (int64_t v = prev + 1; v <= cur; ++v) { off[v] = i; }
    }
}

// Key of arc i for the degree order: source in the high word, then the
// complement of the neighbour's degree (higher degree sorts first).
__global__ void degree_keys_kernel(const uint32_t *src, const uint32_t *adj, const int64_t *off,
                                   int64_t arcs, uint64_t *key)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < arcs;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = adj[i];
        const int64_t d = off[v + 1] - off[v];
        const uint32_t dc = 0xFFFFFFFFu - (uint32_t)(d < 0xFFFFFFFFll ? d : 0xFFFFFFFFll);
        key[i] = ((uint64_t)src[i] << 32) | dc;
    }
}

__global__ void count_live_kernel(const int64_t *off, int64_t n, unsigned long long *live)
{
    unsigned long long c = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        c += off[v + 1] != off[v];
    }
    for (int d = 16; d > 0; d >>= 1) { c += __shfl_xor_sync(0xFFFFFFFFu, c, d); }
    if ((threadIdx.x & 31) == 0 && c) { atomicAdd(live, c); }
}

__global__ void isolated_bitmap_kernel(const int64_t *off, int64_t n, uint32_t *bits)
{
    int64_t words = (n + 31) / 32;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < words;
         w += (int64_t)gridDim.x * blockDim.x) {
        uint32_t b = 0;
        for (int k = 0; k < 32; ++k) {
            int64_t v = w * 32 + k;
            if (v >= n || off[v + 1] == off[v]) { b |= 1u << k; }
        }
        bits[w] = b;
    }
}

// Hub numbering: sort key of vertex v = (complement of its degree, v), so
// the ascending sort lists vertices by degree, highest first, ties by id.
__global__ void hub_keys_kernel(const int64_t *off, int64_t n, uint64_t *key)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = off[v + 1] - off[v];
        const uint32_t dc = 0xFFFFFFFFu - (uint32_t)(d < 0xFFFFFFFFll ? d : 0xFFFFFFFFll);
        key[v] = ((uint64_t)dc << 32) | (uint64_t)v;
    }
}

// From the sorted keys: iperm (new -> old), perm (old -> new) and the
// degree of each new vertex (the scan input of the new offsets).
__global__ void hub_perm_kernel(const uint64_t *sorted, const int64_t *off, int64_t n,
                                uint32_t *perm, uint32_t *iperm, int64_t *tdeg)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)sorted[i];
        iperm[i] = v;
        perm[v] = (uint32_t)i;
        tdeg[i] = off[v + 1] - off[v];
    }
}

// Neighbour list of new vertex i = the list of old vertex iperm[i], each
// neighbour renamed; one warp per vertex, 32 arcs at a time.
__global__ void hub_adj_kernel(const int64_t *off, const uint32_t *adj, const uint32_t *perm,
                               const uint32_t *iperm, const int64_t *toff, int64_t n,
                               uint32_t *tadj)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const uint32_t v = iperm[i];
        const int64_t b = off[v], e = off[v + 1], t = toff[i];
        for (int64_t k = b + lane; k < e; k += 32) { tadj[t + (k - b)] = perm[adj[k]]; }
    }
}

__global__ void validate_csr_kernel(const int64_t *off, const uint32_t *adj, int64_t n,
                                    int64_t arcs, int *bad)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        int64_t b = off[v], e = off[v + 1];
        if (b < 0 || e < b || e > arcs) { atomicExch(bad, 1); continue; }
        if (v == 0 && b != 0) { atomicExch(bad, 1); }
        if (v == n - 1 && e != arcs) { atomicExch(bad, 1); }
        for (int64_t k = b; k < e; ++k) {
            if ((int64_t)adj[k] >= n) { atomicExch(bad, 1); break; }
        }
    }
}

__global__ void split_pairs_kernel(const int64_t *pairs, int64_t count, int64_t *src,
                                   int64_t *dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        src[i] = pairs[2 * i];
        dst[i] = pairs[2 * i + 1];
    }
}

__global__ void shift_csr_kernel(const int64_t *off_in, const uint32_t *adj_in, int64_t n,
                                 int64_t arcs, int64_t vbase, int64_t abase, int64_t *off_out,
                                 uint32_t *adj_out)
{
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t v = t; v < n; v += stride) { off_out[vbase + v] = off_in[v] + abase; }
    for (int64_t e = t; e < arcs; e += stride) {
        adj_out[abase + e] = adj_in[e] + (uint32_t)vbase;
    }
}

__global__ void set_last_offset_kernel(int64_t *off, int64_t n, int64_t arcs) { off[n] = arcs; }

// graph::check: each edge present in both lists; no equal adjacent entries.
__global__ void graph_check_kernel(const int64_t *src, const int64_t *dst, int64_t m,
                                   const int64_t *off, const uint32_t *adj, int64_t arcs,
                                   int sorted, int *bad)
{
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t k = t; k < m; k += stride) {
        for (int dir = 0; dir < 2; ++dir) {
            int64_t u = dir ? dst[k] : src[k];
            uint32_t v = (uint32_t)(dir ? src[k] : dst[k]);
            int64_t b = off[u], e = off[u + 1];
            bool found = false;
            if (sorted) {
                while (b < e) {
                    int64_t mid = (b + e) / 2;
                    if (adj[mid] < v) { b = mid + 1; } else { e = mid; }
                }
                found = b < off[u + 1] && adj[b] == v;
            } else {
                for (int64_t i = b; i < e && !found; ++i) { found = adj[i] == v; }
            }
            if (!found) { atomicExch(bad, 1); }
        }
    }
    (void)arcs;
}

__global__ void adjacent_dup_kernel(const int64_t *off, const uint32_t *adj, int64_t n, int *bad)
{
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += stride) {
        for (int64_t i = off[v] + 1; i < off[v + 1]; ++i) {
            if (adj[i] == adj[i - 1]) { atomicExch(bad, 1); break; }
        }
    }
}

// lcg(seed) (lcg.h:11-27) and pick_random_vertex (hybrid_bfs_main.cc:136-144):
// rng() % n until the vertex has nonzero degree.  Bounded so a pathological
// graph cannot loop forever; *status gets 1 if the bound was hit.
__global__ void pick_roots_kernel(const int64_t *off, int64_t n, uint64_t seed, int64_t k,
                                  int64_t *roots, int *status)
{
    const uint64_t mul = 6364136223846793005ull;
    uint64_t mul_k = mul, add_k = 1, ran = 1;
    for (uint64_t un = seed; un; un >>= 1) {
        if (un & 1) { ran = mul_k * ran + add_k; }
        add_k *= (mul_k + 1);
        mul_k *= mul_k;
    }
    uint64_t state = ran;
    int64_t budget = (int64_t)1 << 34;
    for (int64_t s = 0; s < k; ++s) {
        int64_t v;
        do {
            if (--budget < 0) { *status = 1; return; }
            state = mul * state + 1;
            v = (int64_t)(state % (uint64_t)n);
        } while (off[v + 1] == off[v]);
        roots[s] = v;
    }
}

// Runs a CUB algorithm in the usual two calls: size query, then work.
template <typename F>
cudaError_t cub_run(F &&f, cudaStream_t s)
{
    size_t bytes = 0;
    cudaError_t e = f(nullptr, bytes);
    if (e != cudaSuccess) { return e; }
    void *tmp = nullptr;
    e = cudaMalloc(&tmp, bytes ? bytes : 1);
    if (e != cudaSuccess) { return e; }
    e = f(tmp, bytes);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(tmp);
    return e != cudaSuccess ? e : e2;
}

int bits_for(int64_t n)
{
    int b = 1;
    while (b < 32 && ((int64_t)1 << b) < n) { ++b; }
    return b;
}

bd_status read_flag(const int *d_flag, int *out)
{
    BD_CUDA(cudaMemcpy(out, d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    return BD_OK;
}

// ---------------------------------------------------------------------------
// el64 header (edge_list.cc:20-89): one text line shorter than 256 bytes
// ending in '\n', parsed like a long-option command line; then the checks
// of dist_edge_list.cc:56-76.
// ---------------------------------------------------------------------------
bd_status parse_el64_header(FILE *fp, int64_t *nv, int64_t *ne)
{
    char line[256];
    if (!fgets(line, sizeof line, fp)) { return BD_ERR_FORMAT; }
    size_t len = strlen(line);
    if (len == 0 || line[len - 1] != '\n') { return BD_ERR_FORMAT; }
    line[len - 1] = '\0';
    int64_t num_v = -1, num_e = -1;
    bool deduped = false, el64 = false;
    std::vector<std::string> tok;
    for (char *save = nullptr, *t = strtok_r(line, " ", &save); t; t = strtok_r(nullptr, " ", &save)) {
        tok.emplace_back(t);
    }
    for (size_t i = 0; i < tok.size(); ++i) {
        const std::string &t = tok[i];
        auto value = [&](int64_t *dst) -> bool {
            if (i + 1 >= tok.size()) { return false; }
            *dst = atoll(tok[++i].c_str());
            return true;
        };
        if (t == "--num_vertices") {
            if (!value(&num_v)) { return BD_ERR_FORMAT; }
        } else if (t == "--num_edges") {
            if (!value(&num_e)) { return BD_ERR_FORMAT; }
        } else if (t == "--format") {
            if (i + 1 >= tok.size()) { return BD_ERR_FORMAT; }
            el64 = tok[++i] == "el64";
        } else if (t == "--is_deduped") {
            deduped = true;
        } else if (t == "--is_sorted" || t == "--is_permuted" || t == "--is_directed" ||
                   t == "--is_undirected") {
        } else {
            return BD_ERR_FORMAT;
        }
    }
    if (num_v <= 0 || num_e <= 0 || !el64 || !deduped) { return BD_ERR_FORMAT; }
    *nv = num_v;
    *ne = num_e;
    return BD_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Construction pipeline shared by every graph source
// ---------------------------------------------------------------------------

void graph_free(bd_graph *g)
{
    if (!g) { return; }
    cudaFree(g->d_off);
    cudaFree(g->d_adj);
    cudaFree(g->d_isolated);
    cudaFree(g->d_src);
    cudaFree(g->d_dst);
    cudaFree(g->d_toff);
    cudaFree(g->d_tadj);
    cudaFree(g->d_tisolated);
    cudaFree(g->d_perm);
    cudaFree(g->d_iperm);
    delete g;
}

bd_status graph_build_hub(bd_graph *g, cudaStream_t s)
{
    const int64_t n = g->n;
    const int64_t words = bitmap_words(n);
    if (cudaMalloc(&g->d_toff, sizeof(int64_t) * (n + 1)) != cudaSuccess ||
        cudaMalloc(&g->d_tadj, sizeof(uint32_t) * (g->arcs ? g->arcs : 1)) != cudaSuccess ||
        cudaMalloc(&g->d_tisolated, sizeof(uint32_t) * (words ? words : 1)) != cudaSuccess ||
        cudaMalloc(&g->d_perm, sizeof(uint32_t) * (n ? n : 1)) != cudaSuccess ||
        cudaMalloc(&g->d_iperm, sizeof(uint32_t) * (n ? n : 1)) != cudaSuccess) {
        return BD_ERR_OOM;
    }
    DevBuf<uint64_t> key, sorted;
    DevBuf<int64_t> tdeg;
    if (key.alloc(n) != cudaSuccess || sorted.alloc(n) != cudaSuccess ||
        tdeg.alloc(n + 1) != cudaSuccess) {
        return BD_ERR_OOM;
    }
    hub_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(g->d_off, n, key.p);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
        return cub::DeviceRadixSort::SortKeys(tmp, bytes, key.p, sorted.p, n, 0, 64, s);
    }, s));
    hub_perm_kernel<<<grid_for(n), kThreads, 0, s>>>(sorted.p, g->d_off, n, g->d_perm, g->d_iperm,
                                                     tdeg.p);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaMemsetAsync(tdeg.p + n, 0, sizeof(int64_t), s));
    BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
        return cub::DeviceScan::ExclusiveSum(tmp, bytes, tdeg.p, g->d_toff, n + 1, s);
    }, s));
    hub_adj_kernel<<<grid_for(n * 32), kThreads, 0, s>>>(g->d_off, g->d_adj, g->d_perm, g->d_iperm,
                                                          g->d_toff, n, g->d_tadj);
    BD_CUDA(cudaGetLastError());
    isolated_bitmap_kernel<<<grid_for(words), kThreads, 0, s>>>(g->d_toff, n, g->d_tisolated);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaStreamSynchronize(s));
    return BD_OK;
}

bd_status graph_finish(bd_graph *g, cudaStream_t s)
{
    int64_t words = bitmap_words(g->n);
    BD_CUDA(cudaMalloc(&g->d_isolated, sizeof(uint32_t) * (words ? words : 1)));
    isolated_bitmap_kernel<<<grid_for(words), kThreads, 0, s>>>(g->d_off, g->n, g->d_isolated);
    BD_CUDA(cudaGetLastError());
    DevBuf<unsigned long long> live;
    if (live.alloc(1) != cudaSuccess) { return BD_ERR_OOM; }
    BD_CUDA(cudaMemsetAsync(live.p, 0, sizeof(unsigned long long), s));
    count_live_kernel<<<grid_for(g->n), kThreads, 0, s>>>(g->d_off, g->n, live.p);
    BD_CUDA(cudaGetLastError());
    unsigned long long nl = 0;
    BD_CUDA(cudaMemcpyAsync(&nl, live.p, sizeof(nl), cudaMemcpyDeviceToHost, s));
    BD_CUDA(cudaStreamSynchronize(s));
    g->n_live = (int64_t)nl;
    return BD_OK;
}

bd_status graph_from_device_edges(int64_t n, int64_t m, int64_t *d_src, int64_t *d_dst,
                                  int32_t order, bd_graph **out)
{
    auto *g = new bd_graph();
    g->device = current_device();
    g->n = n;
    g->m = m;
    g->arcs = 2 * m;
    g->order = order;
    g->symmetric = true;  // every edge is stored in both directions
    g->d_src = d_src;
    g->d_dst = d_dst;
    cudaStream_t s = 0;
    const int64_t arcs = g->arcs;
    DevBuf<int> bad;
    auto fail = [&](bd_status st) { graph_free(g); return st; };
    if (bad.alloc(1) != cudaSuccess) { return fail(BD_ERR_OOM); }
    if (cudaMemset(bad.p, 0, sizeof(int)) != cudaSuccess) { return fail(BD_ERR_CUDA); }
    if (cudaMalloc(&g->d_off, sizeof(int64_t) * (n + 1)) != cudaSuccess ||
        cudaMalloc(&g->d_adj, sizeof(uint32_t) * (arcs ? arcs : 1)) != cudaSuccess) {
        return fail(BD_ERR_OOM);
    }
    DevBuf<uint32_t> sorted_src;
    if (sorted_src.alloc(arcs) != cudaSuccess) { return fail(BD_ERR_OOM); }
    if (order == BD_ORDER_SORTED) {
        DevBuf<uint64_t> k_in, k_out;
        if (k_in.alloc(arcs) != cudaSuccess || k_out.alloc(arcs) != cudaSuccess) {
            return fail(BD_ERR_OOM);
        }
        make_sorted_arcs_kernel<<<grid_for(m), kThreads, 0, s>>>(d_src, d_dst, m, n, k_in.p, bad.p);
        cudaError_t e = cub_run([&](void *tmp, size_t &bytes) {
            return cub::DeviceRadixSort::SortKeys(tmp, bytes, k_in.p, k_out.p, arcs, 0, 64, s);
        }, s);
        if (e != cudaSuccess) { return fail(cuda_fail(e, "SortKeys(arcs)", __FILE__, __LINE__)); }
        split_sorted_arcs_kernel<<<grid_for(arcs), kThreads, 0, s>>>(k_out.p, arcs, sorted_src.p,
                                                                     g->d_adj);
    } else {
        DevBuf<uint32_t> k_in, v_in;
        if (k_in.alloc(arcs) != cudaSuccess || v_in.alloc(arcs) != cudaSuccess) {
            return fail(BD_ERR_OOM);
        }
        make_arcs_kernel<<<grid_for(m), kThreads, 0, s>>>(d_src, d_dst, m, n, k_in.p, v_in.p, bad.p);
        int end_bit = bits_for(n);
        // Radix sort is stable: arcs with the same source keep insertion order.
        cudaError_t e = cub_run([&](void *tmp, size_t &bytes) {
            return cub::DeviceRadixSort::SortPairs(tmp, bytes, k_in.p, sorted_src.p, v_in.p,
                                                   g->d_adj, arcs, 0, end_bit, s);
        }, s);
        if (e != cudaSuccess) { return fail(cuda_fail(e, "SortPairs(arcs)", __FILE__, __LINE__)); }
    }
    offsets_from_sorted_kernel<<<grid_for(arcs + 1), kThreads, 0, s>>>(sorted_src.p, arcs, n,
                                                                        g->d_off);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
        return fail(BD_ERR_CUDA);
    }
    int flag = 0;
    if (read_flag(bad.p, &flag) != BD_OK) { return fail(BD_ERR_CUDA); }
    if (flag) { return fail(BD_ERR_RANGE); }
    if (order == BD_ORDER_DEGREE || order == BD_ORDER_HUB) {
        // Re-sort every list by neighbour degree, highest first; the stable
        // sort keeps insertion order among equal degrees.
        DevBuf<uint64_t> k_in, k_out;
        DevBuf<uint32_t> v_out;
        if (k_in.alloc(arcs) != cudaSuccess || k_out.alloc(arcs) != cudaSuccess ||
            v_out.alloc(arcs) != cudaSuccess) {
            return fail(BD_ERR_OOM);
        }
        degree_keys_kernel<<<grid_for(arcs), kThreads, 0, s>>>(sorted_src.p, g->d_adj, g->d_off,
                                                               arcs, k_in.p);
        const int end_bit = 32 + bits_for(n);
        cudaError_t e = cub_run([&](void *tmp, size_t &bytes) {
            return cub::DeviceRadixSort::SortPairs(tmp, bytes, k_in.p, k_out.p, g->d_adj, v_out.p,
                                                   arcs, 0, end_bit, s);
        }, s);
        if (e != cudaSuccess) { return fail(cuda_fail(e, "SortPairs(degree)", __FILE__, __LINE__)); }
        if (cudaMemcpyAsync(g->d_adj, v_out.p, sizeof(uint32_t) * arcs, cudaMemcpyDeviceToDevice,
                            s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            return fail(BD_ERR_CUDA);
        }
    }
    bd_status st = graph_finish(g, s);
    if (st == BD_OK && order == BD_ORDER_HUB) { st = graph_build_hub(g, s); }
    if (st != BD_OK) { return fail(st); }
    *out = g;
    return BD_OK;
}

}  // namespace bd

using namespace bd;

extern "C" {

bd_status bd_graph_from_edges(int64_t num_vertices, int64_t num_edges, const int64_t *src,
                              const int64_t *dst, int32_t adjacency_order, bd_graph **out)
{
    if (!out || (!src && num_edges) || (!dst && num_edges) || num_vertices <= 0 || num_edges < 0) {
        return BD_ERR_INVALID;
    }
    if (adjacency_order < BD_ORDER_INSERTION || adjacency_order > BD_ORDER_HUB) {
        return BD_ERR_INVALID;
    }
    if (num_vertices > (int64_t)UINT32_MAX) { return BD_ERR_LIMIT; }
    BD_TRY(ensure_device());
    int64_t *d_src = nullptr, *d_dst = nullptr;
    size_t bytes = sizeof(int64_t) * (num_edges ? num_edges : 1);
    if (cudaMalloc(&d_src, bytes) != cudaSuccess || cudaMalloc(&d_dst, bytes) != cudaSuccess) {
        cudaFree(d_src);
        cudaFree(d_dst);
        return BD_ERR_OOM;
    }
    if (num_edges) {
        cudaError_t e1 = cudaMemcpy(d_src, src, bytes, cudaMemcpyHostToDevice);
        cudaError_t e2 = cudaMemcpy(d_dst, dst, bytes, cudaMemcpyHostToDevice);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            cudaFree(d_src);
            cudaFree(d_dst);
            return cuda_fail(e1 != cudaSuccess ? e1 : e2, "cudaMemcpy(edges)", __FILE__, __LINE__);
        }
    }
    return graph_from_device_edges(num_vertices, num_edges, d_src, d_dst, adjacency_order, out);
}

bd_status bd_graph_from_el64(const char *path, int32_t adjacency_order, bd_graph **out)
{
    if (!path || !out) { return BD_ERR_INVALID; }
    if (adjacency_order < BD_ORDER_INSERTION || adjacency_order > BD_ORDER_HUB) {
        return BD_ERR_INVALID;
    }
    FILE *fp = fopen(path, "rb");
    if (!fp) { return BD_ERR_IO; }
    int64_t nv = 0, ne = 0;
    bd_status st = parse_el64_header(fp, &nv, &ne);
    if (st != BD_OK) { fclose(fp); return st; }
    if (nv > (int64_t)UINT32_MAX) { fclose(fp); return BD_ERR_LIMIT; }
    st = ensure_device();
    if (st != BD_OK) { fclose(fp); return st; }
    // Stream the body through two pinned staging buffers into a device array
    // of (src, dst) pairs, then split it.
    int64_t *d_pairs = nullptr, *d_src = nullptr, *d_dst = nullptr;
    const size_t chunk_pairs = (size_t)1 << 22;  // 64 MiB per staging buffer
    int64_t *stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaStream_t s = nullptr;
    auto cleanup = [&]() {
        if (s) { cudaStreamSynchronize(s); }
        for (int i = 0; i < 2; ++i) {
            if (stage[i]) { cudaFreeHost(stage[i]); }
            if (done[i]) { cudaEventDestroy(done[i]); }
        }
        if (s) { cudaStreamDestroy(s); }
        cudaFree(d_pairs);
        fclose(fp);
    };
    if (cudaMalloc(&d_pairs, sizeof(int64_t) * 2 * ne) != cudaSuccess ||
        cudaHostAlloc(&stage[0], sizeof(int64_t) * 2 * chunk_pairs, 0) != cudaSuccess ||
        cudaHostAlloc(&stage[1], sizeof(int64_t) * 2 * chunk_pairs, 0) != cudaSuccess ||
        cudaEventCreate(&done[0]) != cudaSuccess || cudaEventCreate(&done[1]) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cleanup();
        return BD_ERR_OOM;
    }
    int64_t pos = 0;
    int which = 0;
    while (pos < ne) {
        size_t want = (size_t)std::min<int64_t>((int64_t)chunk_pairs, ne - pos);
        if (cudaEventSynchronize(done[which]) != cudaSuccess) { cleanup(); return BD_ERR_CUDA; }
        size_t got = fread(stage[which], sizeof(int64_t) * 2, want, fp);
        if (got != want) { cleanup(); return BD_ERR_FORMAT; }  // unexpected EOF
        if (cudaMemcpyAsync(d_pairs + 2 * pos, stage[which], sizeof(int64_t) * 2 * want,
                            cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaEventRecord(done[which], s) != cudaSuccess) {
            cleanup();
            return BD_ERR_CUDA;
        }
        pos += (int64_t)want;
        which ^= 1;
    }
    if (cudaMalloc(&d_src, sizeof(int64_t) * ne) != cudaSuccess ||
        cudaMalloc(&d_dst, sizeof(int64_t) * ne) != cudaSuccess) {
        cudaFree(d_src);
        cudaFree(d_dst);
        cleanup();
        return BD_ERR_OOM;
    }
    split_pairs_kernel<<<grid_for(ne), kThreads, 0, s>>>(d_pairs, ne, d_src, d_dst);
    cudaError_t e = cudaGetLastError();
    cleanup();
    if (e != cudaSuccess) {
        cudaFree(d_src);
        cudaFree(d_dst);
        return cuda_fail(e, "split_pairs_kernel", __FILE__, __LINE__);
    }
    return graph_from_device_edges(nv, ne, d_src, d_dst, adjacency_order, out);
}

bd_status bd_graph_from_csr(int64_t num_vertices, int64_t num_arcs, const int64_t *offsets,
                            const uint32_t *adjacency, bd_graph **out)
{
    if (!out || !offsets || (!adjacency && num_arcs) || num_vertices <= 0 || num_arcs < 0) {
        return BD_ERR_INVALID;
    }
    if (num_vertices > (int64_t)UINT32_MAX) { return BD_ERR_LIMIT; }
    BD_TRY(ensure_device());
    auto *g = new bd_graph();
    g->device = current_device();
    g->n = num_vertices;
    g->arcs = num_arcs;
    g->m = num_arcs / 2;
    if (cudaMalloc(&g->d_off, sizeof(int64_t) * (num_vertices + 1)) != cudaSuccess ||
        cudaMalloc(&g->d_adj, sizeof(uint32_t) * (num_arcs ? num_arcs : 1)) != cudaSuccess) {
        graph_free(g);
        return BD_ERR_OOM;
    }
    DevBuf<int> bad;
    if (bad.alloc(1) != cudaSuccess || cudaMemset(bad.p, 0, sizeof(int)) != cudaSuccess ||
        cudaMemcpy(g->d_off, offsets, sizeof(int64_t) * (num_vertices + 1),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        (num_arcs && cudaMemcpy(g->d_adj, adjacency, sizeof(uint32_t) * num_arcs,
                                cudaMemcpyHostToDevice) != cudaSuccess)) {
        graph_free(g);
        return BD_ERR_CUDA;
    }
    validate_csr_kernel<<<grid_for(num_vertices), kThreads>>>(g->d_off, g->d_adj, num_vertices,
                                                             num_arcs, bad.p);
    int flag = 0;
    if (cudaDeviceSynchronize() != cudaSuccess || read_flag(bad.p, &flag) != BD_OK) {
        graph_free(g);
        return BD_ERR_CUDA;
    }
    if (flag) { graph_free(g); return BD_ERR_FORMAT; }
    bd_status st = graph_finish(g, 0);
    if (st == BD_OK && g->order == BD_ORDER_HUB) { st = graph_build_hub(g, 0); }
    if (st != BD_OK) { graph_free(g); return st; }
    *out = g;
    return BD_OK;
}

}  // extern "C"

namespace bd {
namespace {

bd_status check_rmat_args(int32_t scale, int64_t edge_factor, double a, double b, double c,
                          double d, int32_t adjacency_order, bd_graph **out)
{
    if (!out || scale < 1 || scale > 30 || edge_factor < 1 || edge_factor > 1024) {
        return BD_ERR_INVALID;
    }
    if (!(a >= 0 && b >= 0 && c >= 0 && d >= 0 && a <= 1 && b <= 1 && c <= 1 && d <= 1)) {
        return BD_ERR_INVALID;
    }
    if (adjacency_order < BD_ORDER_INSERTION || adjacency_order > BD_ORDER_HUB) {
        return BD_ERR_INVALID;
    }
    return BD_OK;
}

// rmat_dataset_dump.cc:48-57 from flipped packed keys (keys.p, E of them):
// sort + dedup, then either the seeded vertex relabel and edge shuffle
// (permute) or the sorted list as it is, then the CSR.
bd_status rmat_finish(int32_t scale, int64_t E, DevBuf<uint64_t> &keys,
                      DevBuf<uint64_t> &keys_sorted, bool permute, uint64_t seed,
                      int32_t adjacency_order, bd_graph **out)
{
    const int64_t n = (int64_t)1 << scale;
    cudaStream_t s = 0;
    BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
        return cub::DeviceRadixSort::SortKeys(tmp, bytes, keys.p, keys_sorted.p, E, 0, 2 * scale, s);
    }, s));
    DevBuf<int64_t> num_unique;
    if (num_unique.alloc(1) != cudaSuccess) { return BD_ERR_OOM; }
    BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
        return cub::DeviceSelect::Unique(tmp, bytes, keys_sorted.p, keys.p, num_unique.p, E, s);
    }, s));
    int64_t m = 0;
    BD_CUDA(cudaMemcpy(&m, num_unique.p, sizeof(int64_t), cudaMemcpyDeviceToHost));
    const uint64_t *packed = keys.p;  // sorted, deduplicated
    DevBuf<uint64_t> vkeys, vkeys_sorted, ekeys, ekeys_sorted;
    DevBuf<uint32_t> vidx, vidx_sorted, new_id;
    if (permute) {
        // relabel (rmat_dataset_dump.cc:55): vertex with the k-th smallest key -> k
        if (vkeys.alloc(n) != cudaSuccess || vkeys_sorted.alloc(n) != cudaSuccess ||
            vidx.alloc(n) != cudaSuccess || vidx_sorted.alloc(n) != cudaSuccess ||
            new_id.alloc(n) != cudaSuccess) {
            return BD_ERR_OOM;
        }
        perm_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(seed, kTagRelabel, n, vkeys.p, vidx.p);
        BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
            return cub::DeviceRadixSort::SortPairs(tmp, bytes, vkeys.p, vkeys_sorted.p, vidx.p,
                                                   vidx_sorted.p, n, 0, 64, s);
        }, s));
        scatter_rank_kernel<<<grid_for(n), kThreads, 0, s>>>(vidx_sorted.p, n, new_id.p);
        // shuffle (rmat_dataset_dump.cc:57): order edges by a keyed permutation
        if (ekeys.alloc(m) != cudaSuccess || ekeys_sorted.alloc(m) != cudaSuccess) {
            return BD_ERR_OOM;
        }
        edge_shuffle_keys_kernel<<<grid_for(m), kThreads, 0, s>>>(seed, m, ekeys.p);
        BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
            return cub::DeviceRadixSort::SortPairs(tmp, bytes, ekeys.p, ekeys_sorted.p, keys.p,
                                                   keys_sorted.p, m, 0, 64, s);
        }, s));
        packed = keys_sorted.p;
    }
    int64_t *d_src = nullptr, *d_dst = nullptr;
    if (cudaMalloc(&d_src, sizeof(int64_t) * (m ? m : 1)) != cudaSuccess ||
        cudaMalloc(&d_dst, sizeof(int64_t) * (m ? m : 1)) != cudaSuccess) {
        cudaFree(d_src);
        cudaFree(d_dst);
        return BD_ERR_OOM;
    }
    unpack_relabel_kernel<<<grid_for(m), kThreads, 0, s>>>(packed, m, scale,
                                                           permute ? new_id.p : nullptr, d_src,
                                                           d_dst);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) { e = cudaStreamSynchronize(s); }
    if (e != cudaSuccess) {
        cudaFree(d_src);
        cudaFree(d_dst);
        return cuda_fail(e, "unpack_relabel_kernel", __FILE__, __LINE__);
    }
    // free the generator temporaries before the CSR build needs its memory
    keys.reset();
    keys_sorted.reset();
    ekeys.reset();
    ekeys_sorted.reset();
    vkeys.reset();
    vkeys_sorted.reset();
    return graph_from_device_edges(n, m, d_src, d_dst, adjacency_order, out);
}

}  // namespace
}  // namespace bd

extern "C" {

bd_status bd_graph_rmat(int32_t scale, int64_t edge_factor, double a, double b, double c,
                        double d, uint64_t seed, int32_t adjacency_order, bd_graph **out)
{
    BD_TRY(check_rmat_args(scale, edge_factor, a, b, c, d, adjacency_order, out));
    BD_TRY(ensure_device());
    const int64_t E = edge_factor << scale;
    DevBuf<uint64_t> keys, keys_sorted;
    if (keys.alloc(E) != cudaSuccess || keys_sorted.alloc(E) != cudaSuccess) { return BD_ERR_OOM; }
    rmat_keys_kernel<<<grid_for(E), kThreads, 0, 0>>>(scale, E, a, b, c, d, seed, keys.p);
    BD_CUDA(cudaGetLastError());
    return rmat_finish(scale, E, keys, keys_sorted, true, seed, adjacency_order, out);
}

bd_status bd_graph_rmat_stream(int32_t scale, int64_t edge_factor, double a, double b, double c,
                               double d, uint32_t stream_seed, int32_t permute,
                               uint64_t permute_seed, int32_t adjacency_order, bd_graph **out)
{
    BD_TRY(check_rmat_args(scale, edge_factor, a, b, c, d, adjacency_order, out));
    if (permute != 0 && permute != 1) { return BD_ERR_INVALID; }
    BD_TRY(ensure_device());
    const int64_t E = edge_factor << scale;
    cudaStream_t s = 0;
    DevBuf<int64_t> src, dst, loops, num_loops;
    DevBuf<uint8_t> flag;
    DevBuf<int> err;
    if (src.alloc(E) != cudaSuccess || dst.alloc(E) != cudaSuccess || flag.alloc(E) != cudaSuccess ||
        loops.alloc(E) != cudaSuccess || num_loops.alloc(1) != cudaSuccess ||
        err.alloc(1) != cudaSuccess) {
        return BD_ERR_OOM;
    }
    BD_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    rmat_sitmo_kernel<<<grid_for(E), kThreads, 0, s>>>(scale, E, a, b, c, d, stream_seed, src.p,
                                                       dst.p, flag.p);
    BD_CUDA(cudaGetLastError());
    // the self loops' edge indices, in ascending order, for the serial re-roll
    iota_kernel<<<grid_for(E), kThreads, 0, s>>>(E, loops.p);
    BD_CUDA(cudaGetLastError());
    DevBuf<int64_t> seq;
    if (seq.alloc(E) != cudaSuccess) { return BD_ERR_OOM; }
    BD_CUDA(cudaMemcpyAsync(seq.p, loops.p, sizeof(int64_t) * E, cudaMemcpyDeviceToDevice, s));
    BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
        return cub::DeviceSelect::Flagged(tmp, bytes, seq.p, flag.p, loops.p, num_loops.p, E, s);
    }, s));
    seq.reset();
    rmat_sitmo_reroll_kernel<<<1, 1, 0, s>>>(scale, E, a, b, c, d, stream_seed, loops.p,
                                             num_loops.p, src.p, dst.p, err.p);
    BD_CUDA(cudaGetLastError());
    int bad = 0;
    BD_CUDA(cudaMemcpy(&bad, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (bad) { return BD_ERR_INVALID; }
    DevBuf<uint64_t> keys, keys_sorted;
    if (keys.alloc(E) != cudaSuccess) { return BD_ERR_OOM; }
    flip_keys_kernel<<<grid_for(E), kThreads, 0, s>>>(src.p, dst.p, E, scale, keys.p);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaStreamSynchronize(s));
    src.reset();
    dst.reset();
    loops.reset();
    flag.reset();
    if (keys_sorted.alloc(E) != cudaSuccess) { return BD_ERR_OOM; }
    return rmat_finish(scale, E, keys, keys_sorted, permute != 0, permute_seed, adjacency_order,
                       out);
}

bd_status bd_graph_grid(int64_t rows, int64_t cols, double delete_frac, uint64_t seed,
                        int32_t adjacency_order, bd_graph **out)
{
    if (!out || rows < 1 || cols < 1 || !(delete_frac >= 0.0 && delete_frac <= 1.0)) {
        return BD_ERR_INVALID;
    }
    if (adjacency_order < BD_ORDER_INSERTION || adjacency_order > BD_ORDER_HUB) {
        return BD_ERR_INVALID;
    }
    if (rows * cols > (int64_t)UINT32_MAX) { return BD_ERR_LIMIT; }
    BD_TRY(ensure_device());
    const int64_t n = rows * cols;
    const int64_t total = rows * (cols - 1) + (rows - 1) * cols;
    DevBuf<int> keep;
    DevBuf<int64_t> pos, count;
    if (keep.alloc(total) != cudaSuccess || pos.alloc(total + 1) != cudaSuccess ||
        count.alloc(1) != cudaSuccess) {
        return BD_ERR_OOM;
    }
    cudaStream_t s = 0;
    if (total > 0) {
        grid_keep_kernel<<<grid_for(total), kThreads, 0, s>>>(rows, cols, delete_frac, seed, total,
                                                               keep.p);
        BD_CUDA(cudaGetLastError());
        BD_CUDA(cub_run([&](void *tmp, size_t &bytes) {
            return cub::DeviceScan::ExclusiveSum(tmp, bytes, keep.p, pos.p, total, s);
        }, s));
    }
    int64_t m = 0;
    if (total > 0) {
        int last_keep = 0;
        int64_t last_pos = 0;
        BD_CUDA(cudaMemcpy(&last_keep, keep.p + total - 1, sizeof(int), cudaMemcpyDeviceToHost));
        BD_CUDA(cudaMemcpy(&last_pos, pos.p + total - 1, sizeof(int64_t), cudaMemcpyDeviceToHost));
        m = last_pos + last_keep;
    }
    int64_t *d_src = nullptr, *d_dst = nullptr;
    if (cudaMalloc(&d_src, sizeof(int64_t) * (m ? m : 1)) != cudaSuccess ||
        cudaMalloc(&d_dst, sizeof(int64_t) * (m ? m : 1)) != cudaSuccess) {
        cudaFree(d_src);
        cudaFree(d_dst);
        return BD_ERR_OOM;
    }
    if (total > 0) {
        grid_emit_kernel<<<grid_for(total), kThreads, 0, s>>>(rows, cols, total, keep.p, pos.p,
                                                               d_src, d_dst);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) { e = cudaStreamSynchronize(s); }
    if (e != cudaSuccess) {
        cudaFree(d_src);
        cudaFree(d_dst);
        return cuda_fail(e, "grid_emit_kernel", __FILE__, __LINE__);
    }
    return graph_from_device_edges(n, m, d_src, d_dst, adjacency_order, out);
}

bd_status bd_graph_concat(bd_graph *const *graphs, int64_t count, bd_graph **out,
                          int64_t *vertex_base)
{
    if (!graphs || count <= 0 || !out) { return BD_ERR_INVALID; }
    int64_t n = 0, arcs = 0, m = 0;
    for (int64_t i = 0; i < count; ++i) {
        if (!graphs[i]) { return BD_ERR_INVALID; }
        if (vertex_base) { vertex_base[i] = n; }
        n += graphs[i]->n;
        arcs += graphs[i]->arcs;
        m += graphs[i]->m;
    }
    if (vertex_base) { vertex_base[count] = n; }
    if (n > (int64_t)UINT32_MAX) { return BD_ERR_LIMIT; }
    BD_TRY(ensure_device());
    auto *g = new bd_graph();
    g->device = current_device();
    g->n = n;
    g->arcs = arcs;
    g->m = m;
    g->order = graphs[0]->order;
    g->symmetric = true;
    for (int64_t i = 0; i < count; ++i) { g->symmetric = g->symmetric && graphs[i]->symmetric; }
    if (cudaMalloc(&g->d_off, sizeof(int64_t) * (n + 1)) != cudaSuccess ||
        cudaMalloc(&g->d_adj, sizeof(uint32_t) * (arcs ? arcs : 1)) != cudaSuccess) {
        graph_free(g);
        return BD_ERR_OOM;
    }
    int64_t vb = 0, ab = 0;
    for (int64_t i = 0; i < count; ++i) {
        const bd_graph *p = graphs[i];
        shift_csr_kernel<<<grid_for(std::max(p->n, p->arcs)), kThreads>>>(
            p->d_off, p->d_adj, p->n, p->arcs, vb, ab, g->d_off, g->d_adj);
        vb += p->n;
        ab += p->arcs;
    }
    set_last_offset_kernel<<<1, 1>>>(g->d_off, n, arcs);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        graph_free(g);
        return BD_ERR_CUDA;
    }
    bd_status st = graph_finish(g, 0);
    if (st != BD_OK) { graph_free(g); return st; }
    *out = g;
    return BD_OK;
}

bd_status bd_graph_info(const bd_graph *g, int64_t *num_vertices, int64_t *num_edges)
{
    if (!g) { return BD_ERR_INVALID; }
    if (num_vertices) { *num_vertices = g->n; }
    if (num_edges) { *num_edges = g->m; }
    return BD_OK;
}

bd_status bd_graph_copy_csr(const bd_graph *g, int64_t *offsets, uint32_t *adjacency)
{
    if (!g) { return BD_ERR_INVALID; }
    BD_TRY(ensure_device());
    if (offsets) {
        BD_CUDA(cudaMemcpy(offsets, g->d_off, sizeof(int64_t) * (g->n + 1), cudaMemcpyDeviceToHost));
    }
    if (adjacency && g->arcs) {
        BD_CUDA(cudaMemcpy(adjacency, g->d_adj, sizeof(uint32_t) * g->arcs, cudaMemcpyDeviceToHost));
    }
    return BD_OK;
}

bd_status bd_graph_copy_edges(const bd_graph *g, int64_t *src, int64_t *dst)
{
    if (!g) { return BD_ERR_INVALID; }
    if (!g->d_src || !g->d_dst) { return BD_ERR_STATE; }
    BD_TRY(ensure_device());
    if (src && g->m) {
        BD_CUDA(cudaMemcpy(src, g->d_src, sizeof(int64_t) * g->m, cudaMemcpyDeviceToHost));
    }
    if (dst && g->m) {
        BD_CUDA(cudaMemcpy(dst, g->d_dst, sizeof(int64_t) * g->m, cudaMemcpyDeviceToHost));
    }
    return BD_OK;
}

// Same layout as dump_bin (generator/edge_list_utils.h:170-197).
bd_status bd_graph_write_el64(const bd_graph *g, const char *path)
{
    if (!g || !path) { return BD_ERR_INVALID; }
    if (!g->d_src || !g->d_dst) { return BD_ERR_STATE; }
    BD_TRY(ensure_device());
    FILE *fp = fopen(path, "wb");
    if (!fp) { return BD_ERR_IO; }
    fprintf(fp, " --format el64 --num_edges %lld --num_vertices %lld --is_undirected"
                " --is_deduped --is_permuted\n",
            (long long)g->m, (long long)g->n);
    const int64_t chunk = (int64_t)1 << 22;
    std::vector<int64_t> s(chunk), d(chunk), pairs(2 * chunk);
    for (int64_t pos = 0; pos < g->m; pos += chunk) {
        int64_t cnt = std::min(chunk, g->m - pos);
        if (cudaMemcpy(s.data(), g->d_src + pos, sizeof(int64_t) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(d.data(), g->d_dst + pos, sizeof(int64_t) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess) {
            fclose(fp);
            return BD_ERR_CUDA;
        }
        for (int64_t i = 0; i < cnt; ++i) {
            pairs[2 * i] = s[i];
            pairs[2 * i + 1] = d[i];
        }
        if (fwrite(pairs.data(), sizeof(int64_t) * 2, cnt, fp) != (size_t)cnt) {
            fclose(fp);
            return BD_ERR_IO;
        }
    }
    if (fclose(fp) != 0) { return BD_ERR_IO; }
    return BD_OK;
}

bd_status bd_graph_check(const bd_graph *g, int32_t *ok)
{
    if (!g || !ok) { return BD_ERR_INVALID; }
    if (!g->d_src || !g->d_dst) { return BD_ERR_STATE; }
    BD_TRY(ensure_device());
    DevBuf<int> bad;
    if (bad.alloc(1) != cudaSuccess) { return BD_ERR_OOM; }
    BD_CUDA(cudaMemset(bad.p, 0, sizeof(int)));
    graph_check_kernel<<<grid_for(g->m), kThreads>>>(g->d_src, g->d_dst, g->m, g->d_off, g->d_adj,
                                                     g->arcs, g->order == BD_ORDER_SORTED, bad.p);
    adjacent_dup_kernel<<<grid_for(g->n), kThreads>>>(g->d_off, g->d_adj, g->n, bad.p);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaDeviceSynchronize());
    int flag = 0;
    BD_TRY(read_flag(bad.p, &flag));
    *ok = flag ? 0 : 1;
    return BD_OK;
}

bd_status bd_graph_pick_roots(const bd_graph *g, uint64_t seed, int64_t k, int64_t *roots)
{
    if (!g || k < 0 || (!roots && k)) { return BD_ERR_INVALID; }
    if (k == 0) { return BD_OK; }
    if (g->arcs == 0) { return BD_ERR_INVALID; }  // no vertex of nonzero degree
    BD_TRY(ensure_device());
    DevBuf<int64_t> d_roots;
    DevBuf<int> status;
    if (d_roots.alloc(k) != cudaSuccess || status.alloc(1) != cudaSuccess) { return BD_ERR_OOM; }
    BD_CUDA(cudaMemset(status.p, 0, sizeof(int)));
    pick_roots_kernel<<<1, 1>>>(g->d_off, g->n, seed, k, d_roots.p, status.p);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaDeviceSynchronize());
    int flag = 0;
    BD_TRY(read_flag(status.p, &flag));
    if (flag) { return BD_ERR_LIMIT; }
    BD_CUDA(cudaMemcpy(roots, d_roots.p, sizeof(int64_t) * k, cudaMemcpyDeviceToHost));
    return BD_OK;
}

bd_status bd_graph_device_csr(const bd_graph *g, const int64_t **offsets,
                              const uint32_t **adjacency)
{
    if (!g) { return BD_ERR_INVALID; }
    if (offsets) { *offsets = g->d_off; }
    if (adjacency) { *adjacency = g->d_adj; }
    return BD_OK;
}

bd_status bd_graph_destroy(bd_graph *g)
{
    if (!g) { return BD_ERR_INVALID; }
    cudaSetDevice(g->device);
    graph_free(g);
    return BD_OK;
}

}  // extern "C"
