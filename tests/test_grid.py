"""The high-diameter contrast graph: a rows x cols 4-neighbour grid with a
seeded fraction of its edges deleted.  Generator bytes against the oracle;
depths bit-exact, check() and m_c for every direction policy, single-source
and batched; run_beamer's direction sequence on a grid."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")


def test_grid_edges_match_oracle():
    for rows, cols, frac, seed in [(7, 9, 0.1, 3), (64, 40, 0.01, 11), (1, 50, 0.0, 0)]:
        g = bd.Graph.grid(rows, cols, frac, seed)
        n, src, dst = O.grid_graph(rows, cols, frac, seed)
        gs, gd = g.edges()
        assert g.num_vertices() == n
        assert np.array_equal(gs, src) and np.array_equal(gd, dst)


@pytest.mark.parametrize("alg", ["beamer_hybrid", "top_down", "bottom_up", "learned"])
def test_grid_depths_all_directions(alg):
    g = bd.Graph.grid(96, 120, 0.01, 5)
    off, adj = g.csr()
    bfs = bd.HybridBFS(g, alg=alg)
    if alg == "learned":
        from beedrill_b200 import policy as P
        import os
        if os.path.exists(P.DEFAULT_PATH):
            P.Policy.load().install(bfs)
    for root in g.pick_roots(0, 3):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        depth = O.bfs_depth(off, adj, root)
        assert np.array_equal(bfs.depths(), depth)
        assert O.check(off, adj, root, bfs.parents())
        if alg == "beamer_hybrid":
            # run_beamer's own sequence: top-down until the unexplored edges
            # run out near the far side of the grid
            dirs, found = O.beamer_sequence(off, depth, root, g.num_edges())
            assert bfs.directions() == dirs
            assert [s["found"] for s in bfs.steps()] == found.tolist()


def test_grid_batched_64_roots():
    g = bd.Graph.grid(80, 100, 0.01, 6)
    off, adj = g.csr()
    roots = g.pick_roots(4, 64)
    ms = bd.BatchedBFS(g, 64)
    from beedrill_b200 import policy as P
    if os.path.exists(P.BATCHED_PATH):
        P.Policy.load(P.BATCHED_PATH).install(ms)
    ms.run(roots)
    m_c, _ = ms.counts()
    for i in range(0, 64, 7):
        depth = O.bfs_depth(off, adj, int(roots[i]))
        assert np.array_equal(ms.depths(i), depth)
        par = ms.parents(i)
        assert O.check(off, adj, int(roots[i]), par)
        assert m_c[i] == O.count_traversed(off, par)
