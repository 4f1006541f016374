"""Graphs with the hub numbering (BD_ORDER_HUB): the traversal kernels run on
a CSR whose vertices are renumbered by degree, and every result comes back
in the caller's numbering -- identical to the oracle's on the caller's
graph, for every direction policy, min-parent trees, many sources, batched
roots, and the exported CSR."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")


@pytest.fixture(scope="module")
def pair():
    hub = bd.Graph.rmat(16, seed=1616, order=bd.ORDER_HUB)
    deg = bd.Graph.rmat(16, seed=1616, order=bd.ORDER_DEGREE)
    return hub, deg


def test_exported_csr_is_the_degree_ordered_one(pair):
    hub, deg = pair
    oh, ah = hub.csr()
    od, ad = deg.csr()
    assert np.array_equal(oh, od) and np.array_equal(ah, ad)
    assert np.array_equal(hub.pick_roots(0, 8), deg.pick_roots(0, 8))
    assert hub.check()


@pytest.mark.parametrize("alg", ["beamer_hybrid", "top_down", "bottom_up", "learned"])
def test_results_in_caller_numbering(pair, alg):
    hub, _ = pair
    off, adj = hub.csr()
    m = hub.num_edges()
    bfs = bd.HybridBFS(hub, alg=alg)
    for root in hub.pick_roots(3, 6):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        depth = bfs.depths()
        assert np.array_equal(depth, O.bfs_depth(off, adj, root))
        par = bfs.parents()
        assert O.check(off, adj, root, par)
        assert bfs.check(root)
        assert bfs.count_num_traversed_edges() == O.count_traversed(off, par)
        if alg == "beamer_hybrid":
            dirs, found = O.beamer_sequence(off, depth, root, m)
            assert bfs.directions() == dirs
            assert [s["found"] for s in bfs.steps()] == found.tolist()


def test_min_parent_bit_exact(pair):
    hub, _ = pair
    off, adj = hub.csr()
    bfs = bd.HybridBFS(hub, min_parent=True)
    for root in hub.pick_roots(5, 4):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        depth = O.bfs_depth(off, adj, root)
        assert np.array_equal(bfs.parents(), O.min_parent(off, adj, root, depth))


def test_run_many_and_run_multi(pair):
    hub, deg = pair
    roots = hub.pick_roots(9, 5)
    a = bd.HybridBFS(hub)
    b = bd.HybridBFS(deg)
    _, ea, _ = a.run_many(roots)
    _, eb, _ = b.run_many(roots)
    assert np.array_equal(ea, eb)
    a.clear()
    a.run_multi(roots)
    b.clear()
    b.run_multi(roots)
    assert np.array_equal(a.depths(), b.depths())


def test_batched_roots(pair):
    hub, _ = pair
    off, adj = hub.csr()
    roots = hub.pick_roots(11, 100)
    ms = bd.BatchedBFS(hub, 100)
    ms.run(roots)
    m_c, n_c = ms.counts()
    for i in range(0, 100, 9):
        r = int(roots[i])
        depth = O.bfs_depth(off, adj, r)
        assert np.array_equal(ms.depths(i), depth)
        par = ms.parents(i)
        assert O.check(off, adj, r, par)
        assert ms.check(i)
        assert m_c[i] == O.count_traversed(off, par) and n_c[i] == int((depth >= 0).sum())


def test_packed_hub_graphs():
    parts = [bd.Graph.rmat(s, 8, seed=70 + s, order=bd.ORDER_HUB) for s in (9, 11, 12)]
    g, base = bd.Graph.concat(parts)
    roots = [int(p.pick_roots(i, 1)[0]) + int(base[i]) for i, p in enumerate(parts)]
    bfs = bd.HybridBFS(g)
    bfs.run_multi(roots)
    depth = bfs.depths()
    for i, p in enumerate(parts):
        off, adj = p.csr()
        lo, hi = int(base[i]), int(base[i + 1])
        assert np.array_equal(depth[lo:hi], O.bfs_depth(off, adj, roots[i] - lo))
