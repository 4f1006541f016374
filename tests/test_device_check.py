"""hybrid_bfs::check (hybrid_bfs.cc:281-379) on the device.

bd_graph_check_parents checks any parent array; bd_bfs_check and
bd_msbfs_check run the same kernels on the parents a traversal left in HBM.
Verdicts and the reported vertex (the one at which the reference's
ascending loop stops) must equal the oracle's restatement of the serial
check, for correct trees and for mistakes planted in a parent array on the
CPU.  At RMAT scale 24 a single planted mistake must be reported at the
vertex where it was planted.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")


def _planted(off, adj, root, good, depth, rng):
    """(what, parent array) pairs, each with mistakes made on the CPU."""
    n = len(off) - 1
    reached = np.flatnonzero(depth > 1)
    v = int(rng.choice(reached))
    nbrs = adj[off[v]:off[v + 1]]
    out = []

    def plant(what, **changes):
        bad = good.copy()
        for k, val in changes.items():
            bad[int(k[1:])] = val
        out.append((what, bad))

    non = np.setdiff1d(np.arange(n), nbrs)
    plant("not a neighbour", **{f"v{v}": int(non[non != v][0])})
    for what, d in (("neighbour on the same level", depth[v]), ("neighbour one level down", depth[v] + 1)):
        cand = [int(u) for u in nbrs if depth[u] == d]
        if cand:
            plant(what, **{f"v{v}": cand[0]})
    plant("reached without a parent", **{f"v{v}": -1})
    plant("its own parent", **{f"v{v}": v})
    plant("parent id past n", **{f"v{v}": n + 5})
    plant("parent id far past n", **{f"v{v}": 1 << 40})
    unreached = np.flatnonzero(depth < 0)
    if len(unreached):
        plant("unreached with a parent", **{f"v{int(unreached[-1])}": root})
    plant("source not its own parent", **{f"v{root}": int(adj[off[root]])})
    w = int(rng.choice(reached[reached != v]))
    plant("two mistakes", **{f"v{v}": -1, f"v{w}": -1})
    return out


@pytest.mark.parametrize("order", [bd.ORDER_INSERTION, bd.ORDER_HUB])
def test_check_parents_matches_the_serial_check(order):
    g = bd.Graph.rmat(14, seed=3, order=order)
    off, adj = g.csr()
    bfs = bd.HybridBFS(g)
    rng = np.random.default_rng(14)
    for root in g.pick_roots(0, 4):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        good = bfs.parents()
        assert bfs.check(root)
        assert g.check_parents(root, good) == (True, -1)
        assert O.check(off, adj, root, good)
        depth = O.bfs_depth(off, adj, root)
        for what, bad in _planted(off, adj, root, good, depth, rng):
            want = O.check_first_bad(off, adj, root, bad)
            assert want >= 0, what
            assert g.check_parents(root, bad) == (False, want), what
    bfs.close()
    g.close()


def test_check_parents_equals_the_reference_check():
    """The reference's own check() (tests/golden/ref_check.npz) on its trees
    of graph500-scale10 and on copies with planted mistakes: same verdict,
    and the reported vertex is the one its LOG lines name."""
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    d = np.load(os.path.join(here, "golden", "ref_check.npz"))
    g = bd.Graph.from_el64(os.path.join(here, "golden", "graph500-scale10.el64"))
    for i, (s, p, v, w) in enumerate(zip(d["sources"], d["parents"], d["verdict"], d["stop"])):
        assert g.check_parents(int(s), p) == (bool(v), int(w)), i
    g.close()


def test_check_parents_small_graphs():
    # no edges: only the source is reached
    g = bd.Graph.from_edges(5, np.zeros(0, np.int64), np.zeros(0, np.int64))
    par = np.full(5, -1, np.int64)
    par[2] = 2
    assert g.check_parents(2, par) == (True, -1)
    par[3] = 2
    assert g.check_parents(2, par) == (False, 3)
    # a path 0-1-2-3 and an isolated vertex 4
    g = bd.Graph.from_edges(5, np.array([0, 1, 2], np.int64), np.array([1, 2, 3], np.int64))
    off, adj = g.csr()
    par = np.array([0, 0, 1, 2, -1], np.int64)
    assert g.check_parents(0, par) == (True, -1)
    for bad, want in (([0, 0, 0, 2, -1], 2), ([0, 0, 1, 2, 0], 4), ([1, 0, 1, 2, -1], 0),
                      ([0, 0, 1, -2, -1], 3), ([0, 2, 1, 2, -1], 1)):
        bad = np.array(bad, np.int64)
        assert O.check_first_bad(off, adj, 0, bad) == want
        assert g.check_parents(0, bad) == (False, want)
    with pytest.raises(bd.BeedrillError):
        g.check_parents(5, par)
    with pytest.raises(ValueError):
        g.check_parents(0, par[:4])


def test_check_parents_high_diameter_grid():
    g = bd.Graph.grid(300, 300, 0.01, seed=7)
    off, adj = g.csr()
    bfs = bd.HybridBFS(g)
    root = int(g.pick_roots(0, 1)[0])
    bfs.run(root)
    good = bfs.parents()
    assert bfs.check(root)
    depth = O.bfs_depth(off, adj, root)
    far = int(np.argmax(depth))
    bad = good.copy()
    bad[far] = -1
    assert g.check_parents(root, bad) == (False, O.check_first_bad(off, adj, root, bad))
    bfs.close()


def test_batched_check_matches_the_serial_check():
    g = bd.Graph.rmat(18, seed=18, order=bd.ORDER_HUB)
    off, adj = g.csr()
    roots = g.pick_roots(0, 64)
    ms = bd.BatchedBFS(g, 64)
    ms.run(roots)
    for i in range(0, 64, 9):
        par = ms.parents(i)
        assert ms.check(i), i
        assert O.check(off, adj, int(roots[i]), par), i
    ms.close()


def test_scale24_check_and_a_planted_mistake():
    g = bd.Graph.rmat(24, seed=24, order=bd.ORDER_HUB)
    roots = g.pick_roots(0, 2)
    bfs = bd.HybridBFS(g)
    ms = bd.BatchedBFS(g, 2)
    ms.run(roots)
    for i, root in enumerate(roots):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        assert bfs.check(root)
        assert ms.check(i)
    good = bfs.parents()
    root = int(roots[-1])
    assert g.check_parents(root, good) == (True, -1)
    reached = np.flatnonzero(good >= 0)
    reached = reached[reached != root]
    # one mistake: the check stops exactly there (no self loops, so a vertex
    # is never its own neighbour)
    for v in (int(reached[0]), int(reached[len(reached) // 2]), int(reached[-1])):
        for wrong in (-1, v):
            bad = good.copy()
            bad[v] = wrong
            assert g.check_parents(root, bad) == (False, v), (v, wrong)
    ms.close()
    bfs.close()
    g.close()
