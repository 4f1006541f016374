// bd_bfs_device.cuh -- device-side pieces of the direction-optimizing BFS.
//
// One cooperative ("persistent") kernel runs a whole BFS: every CTA loops
// over levels; each level is a top-down step (frontier queue -> CAS claims)
// or a bottom-up step (visited-bitmap scan with early exit), followed by a
// grid barrier (one release-add per CTA, acquire polling) after which every
// CTA reads the step's counters and makes the same direction decision for
// the next level.  No host round trip happens inside a BFS.
//
// Reference counterparts:
//   run_beamer                hybrid_bfs.cc:152-191   (decide_next / beamer_*)
//   top-down step             hybrid_bfs.cc:71-100    (td_step)
//   bottom-up step            hybrid_bfs.cc:111-143   (bu_step)
//   sliding_queue windows     sliding_queue.h:77-99   (queue ping-pong)
#pragma once

#include <stdint.h>

#include "beedrill_b200.h"
#include "bd_policy.cuh"

namespace bd {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kDirTD = BD_DIR_TOP_DOWN;
constexpr int kDirBU = BD_DIR_BOTTOM_UP;
constexpr int kDirDone = 2;
constexpr int kLargeShift = 38;  // large-queue counter: count << 38 | chunks
constexpr unsigned long long kChunkMask = (1ull << kLargeShift) - 1;

// Counters the CTAs accumulate during one step, in a ring of three slots:
// step s uses slot s % 3, CTA 0 clears slot (s + 1) % 3 during step s (every
// CTA finished reading it before arriving at the barrier of step s - 1).
struct Acc {
    unsigned long long found;
    unsigned long long degsum;
    unsigned long long small_cnt;
    unsigned long long large_packed;
    unsigned long long t_end;  // max over CTAs of their arrival time
    unsigned long long pad[3];
};

// The traversal state between steps.  The init kernel writes the first one
// into Ctrl; every CTA then keeps an identical copy in shared memory and
// advances it with the same function of the same counters after each
// barrier; CTA 0 writes the final one back for the host.
struct LevelState {
    int dir;        // direction of the step about to run, or kDirDone
    int level;      // depth of the current frontier
    int vis_cur;    // parity of the visited bitmap that is current
    int q_cur;      // parity of the queues holding the current frontier
    int step;       // index of the step about to run
    int bu_sparse;  // next bottom-up step uses the lane-owned layout
    int in_bu;      // inside Beamer's bottom-up do-while
    int prev_dir;
    long long etc;        // Beamer edges_to_check
    long long scout;      // Beamer scout_count
    long long awake;      // Beamer awake_count
    long long old_awake;
    long long prev_ns;    // duration of the previous step
    long long t_last;     // end of the previous step (globaltimer)
    long long f_count, f_degsum, f_small, f_large, f_chunks;
    long long visited_degsum;
    long long reached;
    long long td_steps, bu_steps;
    long long policy_overrides;  // learned decisions that differed from Beamer
};

// Device-resident control block of one BFS handle.
struct Ctrl {
    unsigned long long bar;      // barrier arrivals; step s is complete at (s+1) * CTAs
    int error;
    int pad0;
    unsigned long long t_start;  // min over CTAs of their start time
    LevelState st;
    Acc acc[3];
};

struct BfsParams {
    const int64_t *off;
    const uint32_t *adj;
    int64_t n;
    int64_t m;
    int32_t *depth;
    int64_t *parent;
    uint32_t *vis[2];
    int64_t words;
    int64_t n_live;  // vertices of nonzero degree
    uint32_t *qs[2];
    uint32_t *ql[2];
    unsigned long long *qlb[2];
    Ctrl *ctrl;
    bd_step *rec;
    int64_t rec_cap;
    int alg;
    int64_t alpha;
    int64_t beta;
    uint32_t large_deg;
    uint32_t chunk;
    int bu_prefix;
    long long spin_limit;
    unsigned expected_ctas;
    const PolicyBlob *policy;  // null: no learned policy loaded
    const uint32_t *perm;      // caller id -> traversal id (BD_ORDER_HUB), or null
};

}  // namespace bd
