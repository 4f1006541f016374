/* Serial-elision stand-in for <cilk/cilk.h>.
 *
 * Test infrastructure only: lets the reference's own BFS sources
 * (hybrid_bfs.cc, graph.cc, edge_list.cc, dist_edge_list.cc,
 * hybrid_bfs_main.cc) compile with plain g++, which has no Cilk support.
 * Dropping cilk_spawn/cilk_sync yields the serial elision, which is by
 * definition a legal execution of the Cilk program.
 */
#pragma once
#define cilk_spawn
#define cilk_sync
#define cilk_for for
static inline int __cilkrts_get_worker_number(void) { return 0; }
