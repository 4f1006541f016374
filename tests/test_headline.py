"""The headline configuration, pinned root by root.

The benchmark's own workload: the seeded RMAT scale-24 graph (edge factor
16, A=.57 B=C=.19 D=.05, graph seed 24, hub numbering) and its 64 lcg(0)
roots (hybrid_bfs_main.cc:136-144), run three ways -- batched with the
shipped push/pull policy and materialized results, one launch per root
under the plain Beamer switch, and one launch per root under the shipped
learned policy.  For EVERY root and every way, as the reference checks every
trial under --check_results (hybrid_bfs_main.cc:283-292): depths bit-exact
against the oracle's serial BFS, the parent tree passes the oracle's
check() (hybrid_bfs.cc:281-379), and m_c and n_c equal the oracle's.

The oracle runs on the host cores in a thread pool (its C calls release the
GIL); results are fetched from the device in chunks of roots so the host
holds a few GB at a time.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")
torch = pytest.importorskip("torch")

SCALE, EDGE_FACTOR, GRAPH_SEED, ROOTS = 24, 16, 24, 64
CHUNK = 8


def _verify(off, adj, root, ways):
    """Oracle verdicts for one root: ways maps a name to (depth, parent,
    m_c, n_c) from the device.  Returns a list of failure strings."""
    want = O.bfs_depth(off, adj, root)
    n_c = int((want >= 0).sum())
    bad = []
    for name, (depth, parent, m_c, reached) in ways.items():
        if not np.array_equal(depth, want):
            bad.append(f"{name}: depths differ")
        if not O.check(off, adj, root, parent):
            bad.append(f"{name}: check() failed")
        if O.count_traversed(off, parent) != m_c:
            bad.append(f"{name}: m_c differs")
        if reached != n_c:
            bad.append(f"{name}: n_c differs")
    return bad


def test_headline_every_root_every_way():
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from beedrill_b200 import policy as P
    torch.cuda.set_device(0)
    bd.lib().bd_set_device(0)
    g = bd.Graph.rmat(SCALE, EDGE_FACTOR, seed=GRAPH_SEED, order=bd.ORDER_HUB)
    n = g.num_vertices()
    off, adj = g.csr()
    roots = g.pick_roots(0, ROOTS)

    batched = bd.BatchedBFS(g, ROOTS, materialize=True)
    if os.path.exists(P.BATCHED_PATH):
        P.Policy.load(P.BATCHED_PATH).install(batched)
    batched.run(roots)
    b_mc, b_nc = batched.counts()

    singles = {}
    for name, alg in (("plain", "beamer_hybrid"), ("learned", "learned")):
        h = bd.HybridBFS(g, alg=alg)
        if alg == "learned" and os.path.exists(P.DEFAULT_PATH):
            P.Policy.load().install(h)
        depth = torch.empty((ROOTS, n), dtype=torch.int32, device="cuda:0")
        parent = torch.empty((ROOTS, n), dtype=torch.int64, device="cuda:0")
        _, m_c, n_c, _ = h.run_many_into(roots, depth.data_ptr(), parent.data_ptr())
        singles[name] = (depth, parent, m_c, n_c)
        h.close()

    failures = []
    workers = max(1, min(16, os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as pool:
        for lo in range(0, ROOTS, CHUNK):
            jobs = []
            for i in range(lo, min(lo + CHUNK, ROOTS)):
                ways = {"batched": (batched.depths(i), batched.parents(i), int(b_mc[i]), int(b_nc[i]))}
                for name, (depth, parent, m_c, n_c) in singles.items():
                    ways[name] = (depth[i].cpu().numpy(), parent[i].cpu().numpy(), int(m_c[i]),
                                  int(n_c[i]))
                jobs.append((i, pool.submit(_verify, off, adj, int(roots[i]), ways)))
            for i, job in jobs:
                failures += [f"root {i} ({int(roots[i])}): {msg}" for msg in job.result()]
    assert not failures, failures[:10]
    batched.close()
    g.close()
