"""Degenerate and irregular inputs through every path: graphs with no edges,
one edge, an isolated source, a star (one vertex adjacent to all), a long
path, several components, and a source in a small component; for each
direction policy, each adjacency order including the hub layout, min-parent
trees, and the batched kernel.  Expected values come from the oracle; the
device check() must pass every tree the oracle's check passes."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")

ORDERS = ["insertion", "sorted", "degree", "hub"]
ALGS = ["beamer_hybrid", "top_down", "bottom_up"]


def _cases():
    rng = np.random.default_rng(77)
    cases = {}
    cases["no_edges"] = (6, [], [])
    cases["one_edge"] = (2, [0], [1])
    cases["isolated_source"] = (5, [1, 2], [2, 3])  # vertex 0 has no edge
    n = 300
    cases["star"] = (n, [0] * (n - 1), list(range(1, n)))
    n = 2000
    cases["path"] = (n, list(range(n - 1)), list(range(1, n)))
    # three components of different sizes plus isolated vertices
    src, dst = [], []
    for base, size in ((0, 500), (600, 40), (700, 3)):
        for _ in range(size * 3):
            a, b = rng.integers(base, base + size, 2)
            if a != b:
                src.append(int(a))
                dst.append(int(b))
    # deduplicate undirected pairs (the el64 contract: deduplicated edges)
    pairs = sorted({(min(a, b), max(a, b)) for a, b in zip(src, dst)})
    cases["components"] = (800, [a for a, _ in pairs], [b for _, b in pairs])
    return cases


CASES = _cases()


def _graph(name, order):
    n, src, dst = CASES[name]
    code = {"insertion": bd.ORDER_INSERTION, "sorted": bd.ORDER_SORTED,
            "degree": bd.ORDER_DEGREE, "hub": bd.ORDER_HUB}[order]
    return bd.Graph.from_edges(n, np.array(src, np.int64), np.array(dst, np.int64), order=code)


def _sources(name):
    n = CASES[name][0]
    return sorted({0, 1, n - 1, n // 2})


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("name", sorted(CASES))
def test_single_source_every_policy(name, order):
    g = _graph(name, order)
    off, adj = g.csr()
    for alg in ALGS:
        bfs = bd.HybridBFS(g, alg=alg)
        for s in _sources(name):
            bfs.clear()
            bfs.run(s)
            depth = O.bfs_depth(off, adj, s)
            assert np.array_equal(bfs.depths(), depth), (name, order, alg, s)
            par = bfs.parents()
            assert O.check(off, adj, s, par), (name, order, alg, s)
            assert bfs.check(s) and g.check_parents(s, par) == (True, -1), (name, order, alg, s)
            assert bfs.count_num_traversed_edges() == O.count_traversed(off, par)
        bfs.close()
    g.close()


@pytest.mark.parametrize("order", ["insertion", "hub"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_min_parent_and_batched(name, order):
    g = _graph(name, order)
    off, adj = g.csr()
    srcs = _sources(name)
    mp = bd.HybridBFS(g, min_parent=True)
    for s in srcs:
        mp.clear()
        mp.run(s)
        depth = O.bfs_depth(off, adj, s)
        assert np.array_equal(mp.parents(), O.min_parent(off, adj, s, depth)), (name, order, s)
    ms = bd.BatchedBFS(g, len(srcs))
    ms.run(np.array(srcs, np.int64))
    m_c, n_c = ms.counts()
    for i, s in enumerate(srcs):
        depth = O.bfs_depth(off, adj, s)
        assert np.array_equal(ms.depths(i), depth), (name, order, s)
        par = ms.parents(i)
        assert O.check(off, adj, s, par)
        assert ms.check(i), (name, order, s)
        assert m_c[i] == O.count_traversed(off, par) and n_c[i] == int((depth >= 0).sum())
    g.close()
