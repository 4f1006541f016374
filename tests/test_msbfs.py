"""Batched traversal (64 roots per pass, one bit lane per root): every
root's results must equal a single-source BFS -- depths bit-exact, parents
pass the reference's check(), m_c and n_c exact."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")


def _check_all(ms, off, adj, roots, limit=None):
    idx = range(len(roots)) if limit is None else range(0, len(roots), max(1, len(roots) // limit))
    m_c, n_c = ms.counts()
    for i in idx:
        root = int(roots[i])
        want = O.bfs_depth(off, adj, root)
        got = ms.depths(i)
        assert np.array_equal(got, want), f"lane {i} root {root}: depths differ"
        par = ms.parents(i)
        assert O.check(off, adj, root, par), f"lane {i}: check() failed"
        assert m_c[i] == O.count_traversed(off, par)
        assert n_c[i] == int((want >= 0).sum())


@pytest.mark.parametrize("force_dir", [-1, 0, 1])
def test_64_roots_every_lane_matches(force_dir):
    g = bd.Graph.rmat(14, seed=41)
    off, adj = g.csr()
    roots = g.pick_roots(0, 64)
    ms = bd.BatchedBFS(g, 64, force_dir=force_dir)
    ms.run(roots)
    _check_all(ms, off, adj, roots)


@pytest.mark.parametrize("heavy", [(64, 32), (256, 100), (1 << 30, 2048)])
def test_heavy_vertex_chunked_pull(heavy):
    """Pull scans of long lists cut into chunks shared by all warps (a
    tiny threshold makes most vertices take that path)."""
    g = bd.Graph.rmat(15, seed=45, order=bd.ORDER_DEGREE)
    off, adj = g.csr()
    roots = g.pick_roots(2, 64)
    ms = bd.BatchedBFS(g, 64, force_dir=1, heavy_degree=heavy[0], heavy_chunk=heavy[1],
                       tuned=False)
    ms.run(roots)
    _check_all(ms, off, adj, roots, limit=16)


def test_partial_groups_duplicates_and_isolated_roots():
    g = bd.Graph.rmat(13, 8, seed=42)
    off, adj = g.csr()
    deg = np.diff(off)
    roots = list(g.pick_roots(3, 90))
    roots[5] = roots[4]                        # same vertex in two lanes
    roots[70] = int(np.flatnonzero(deg == 0)[0])  # a root with no edges
    ms = bd.BatchedBFS(g, 100)
    ms.run(roots)
    _check_all(ms, off, adj, roots)


def test_graph_replay_equals_plain_launches():
    g = bd.Graph.rmat(15, seed=43)
    off, adj = g.csr()
    roots = g.pick_roots(1, 130)
    a = bd.BatchedBFS(g, 130, use_graph=True)
    b = bd.BatchedBFS(g, 130, use_graph=False)
    for _ in range(2):  # second call replays the captured graph
        a.run(roots)
    b.run(roots)
    for i in range(0, 130, 13):
        assert np.array_equal(a.depths(i), b.depths(i))
    _check_all(a, off, adj, roots, limit=12)


def test_256_roots_scale18():
    g = bd.Graph.rmat(18, seed=44)
    off, adj = g.csr()
    roots = g.pick_roots(0, 256)
    ms = bd.BatchedBFS(g, 256)
    st = ms.run(roots)
    assert st.ms > 0
    _check_all(ms, off, adj, roots, limit=16)
    # m_c of every root against the single-source path
    single = bd.HybridBFS(g)
    _, edges, _ = single.run_many(roots)
    m_c, _ = ms.counts()
    assert np.array_equal(m_c, edges)
