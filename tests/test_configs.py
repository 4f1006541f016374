"""The evaluation workloads at their stated sizes.

  * RMAT scale 22, 64 roots, one root per launch (plain Beamer).
  * Batched: 256 roots on RMAT scale 20 (four 64-lane groups in one captured
    graph), and 512 independent RMAT graphs (scales 10-18, edge factors 4-32)
    packed into one CSR and traversed from one root each in one launch.
  * The largest single-GPU case: RMAT scale 26 with 64 roots batched.

Depths are compared bit-exactly with the oracle's BFS and every root's
parents go through the oracle's check() (the oracle runs in a thread pool on
the host cores; its C calls release the GIL).  At scale 26 the 64 batched
roots are compared with the single-source kernel (a different kernel with a
different traversal order), and four of them with the oracle as well.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")


def _pool():
    return ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1)))


def _oracle_verdict(off, adj, root, depth, parent, m_c, n_c):
    """Failure strings for one root's device results against the oracle."""
    want = O.bfs_depth(off, adj, root)
    bad = []
    if not np.array_equal(depth, want):
        bad.append("depths differ")
    if not O.check(off, adj, root, parent):
        bad.append("check() failed")
    if m_c is not None and O.count_traversed(off, parent) != m_c:
        bad.append("m_c differs")
    if n_c is not None and int((want >= 0).sum()) != n_c:
        bad.append("n_c differs")
    return bad


def _batched(g, roots):
    from beedrill_b200 import policy as P
    ms = bd.BatchedBFS(g, len(roots))
    if os.path.exists(P.BATCHED_PATH):
        P.Policy.load(P.BATCHED_PATH).install(ms)
    return ms


def test_scale22_64_roots_one_launch_each():
    g = bd.Graph.rmat(22, seed=22)
    off, adj = g.csr()
    roots = g.pick_roots(0, 64)
    bfs = bd.HybridBFS(g)
    _, edges, _ = bfs.run_many(roots)
    failures = []
    with _pool() as pool:
        jobs = []
        for i, root in enumerate(roots):
            root = int(root)
            bfs.clear()
            bfs.run(root)
            jobs.append((i, pool.submit(_oracle_verdict, off, adj, root, bfs.depths(),
                                        bfs.parents(), int(edges[i]), None)))
        for i, job in jobs:
            failures += [f"root {i}: {msg}" for msg in job.result()]
    assert not failures, failures[:10]


def test_batched_256_roots_scale20():
    g = bd.Graph.rmat(20, seed=20, order=bd.ORDER_DEGREE)
    off, adj = g.csr()
    roots = g.pick_roots(1, 256)
    ms = _batched(g, roots)
    st = ms.run(roots)
    assert st.ms > 0
    m_c, n_c = ms.counts()
    failures = []
    with _pool() as pool:
        jobs = [(i, pool.submit(_oracle_verdict, off, adj, int(root), ms.depths(i), ms.parents(i),
                                int(m_c[i]), int(n_c[i])))
                for i, root in enumerate(roots)]
        for i, job in jobs:
            failures += [f"root {i}: {msg}" for msg in job.result()]
    assert not failures, failures[:10]


def test_packed_512_graphs_one_root_each():
    rng = np.random.default_rng(512)
    scales = rng.integers(10, 19, 512)
    factors = rng.integers(4, 33, 512)
    parts = [bd.Graph.rmat(int(s), int(f), seed=5000 + i) for i, (s, f) in enumerate(zip(scales, factors))]
    g, base = bd.Graph.concat(parts)
    roots = [int(p.pick_roots(i, 1)[0]) + int(base[i]) for i, p in enumerate(parts)]
    bfs = bd.HybridBFS(g)
    bfs.run_multi(roots)
    depth = bfs.depths()
    parent = bfs.parents()
    for i, p in enumerate(parts):
        off, adj = p.csr()
        lo, hi = int(base[i]), int(base[i + 1])
        r = roots[i] - lo
        assert np.array_equal(depth[lo:hi], O.bfs_depth(off, adj, r)), i
        local = parent[lo:hi].copy()
        local[local >= 0] -= lo
        assert O.check(off, adj, r, local), i
        p.close()


def test_scale26_batched_64_roots():
    g = bd.Graph.rmat(26, seed=26, order=bd.ORDER_DEGREE)
    roots = g.pick_roots(0, 64)
    ms = _batched(g, roots)
    ms.run(roots)
    m_c, n_c = ms.counts()
    bfs = bd.HybridBFS(g)
    for i, root in enumerate(roots):
        bfs.clear()
        bfs.run(int(root))
        depth = bfs.depths()
        assert np.array_equal(ms.depths(i), depth), i
        assert m_c[i] == bfs.count_num_traversed_edges(), i
        assert n_c[i] == int((depth >= 0).sum()), i
    ms.close()
    bfs.close()
    off, adj = g.csr()
    ms = _batched(g, roots)
    ms.run(roots)
    m_c, n_c = ms.counts()
    picks = (0, 21, 42, 63)
    with _pool() as pool:
        jobs = [(i, pool.submit(_oracle_verdict, off, adj, int(roots[i]), ms.depths(i),
                                ms.parents(i), int(m_c[i]), int(n_c[i]))) for i in picks]
        failures = [f"root {i}: {msg}" for i, job in jobs for msg in job.result()]
    assert not failures, failures
