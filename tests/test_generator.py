"""The reference generator's edge stream on the device (bd_graph_rmat_stream).

RMAT edges drawn from the reference's own random stream -- sitmo's
counter-mode engine through libstdc++'s uniform doubles, next_edge's
quadrant recursion, rmat_fill's serial self-loop re-roll
(generator/rmat_generator.h:70-193) -- then flipped, sorted and deduplicated
(rmat_dataset_dump.cc:48-53).  The deduplicated list must equal, byte for
byte, what the reference's own generator produced for the fixture cases
(tests/golden/ref_gen.npz, written by oracle/_ref/ref_gen_edges), and what
the oracle's restatement produces at larger scales.  The reference's later
relabel and shuffle depend on its thread count, so the permuted graph is
checked through what a relabel keeps (edge count, degree multiset).
"""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")

HERE = os.path.dirname(os.path.abspath(__file__))


def _cases():
    d = np.load(os.path.join(HERE, "golden", "ref_gen.npz"))
    out = []
    for i, ((scale, ef, seed), prm) in enumerate(zip(d["cases"], d["params"])):
        out.append((i, int(scale), int(ef), tuple(float(x) for x in prm), int(seed)))
    return d, out


FIXTURE, CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=[f"case{c[0]}-scale{c[1]}" for c in CASES])
def test_device_stream_equals_the_reference_generator(case):
    i, scale, ef, (a, b, c, d), seed = case
    g = bd.Graph.rmat_stream(scale, ef, a, b, c, d, stream_seed=seed)
    src, dst = g.edges()
    ded = np.stack([src, dst], axis=1)
    assert len(ded) == FIXTURE[f"{i}.counts"][2]
    assert hashlib.sha256(ded.tobytes()).digest() == bytes(FIXTURE[f"{i}.ded_sha"])
    if i == 0:
        assert np.array_equal(ded, FIXTURE["0.ded"])
    g.close()


@pytest.mark.parametrize("scale,seed", [(16, 0), (18, 5)])
def test_device_stream_equals_the_oracle_at_larger_scales(scale, seed):
    n, s, t = O.rmat_stream_graph(scale, 16, seed=seed)
    g = bd.Graph.rmat_stream(scale, 16, stream_seed=seed)
    assert g.num_vertices() == n
    src, dst = g.edges()
    assert np.array_equal(src, s) and np.array_equal(dst, t)
    off, adj = g.csr()
    assert np.array_equal(off, O.csr_build(n, s, t)[0])
    g.close()


def test_permuted_stream_graph_is_a_relabel():
    n, s, t = O.rmat_stream_graph(14, 16, seed=2)
    g = bd.Graph.rmat_stream(14, 16, stream_seed=2, permute=True, permute_seed=99)
    src, dst = g.edges()
    assert len(src) == len(s)
    deg = np.bincount(np.concatenate([s, t]), minlength=n)
    deg2 = np.bincount(np.concatenate([src, dst]), minlength=n)
    assert np.array_equal(np.sort(deg), np.sort(deg2))
    assert not np.array_equal(src, s)
    g.close()


def test_stream_graph_bfs_matches_the_reference_build_order():
    """A BFS on the stream graph (scale 12, the reference's default seed)
    gives the oracle's depths: the graph is usable like any other."""
    n, s, t = O.rmat_stream_graph(12, 16, seed=0)
    off, adj = O.csr_build(n, s, t)
    g = bd.Graph.rmat_stream(12, 16, stream_seed=0)
    bfs = bd.HybridBFS(g)
    root = int(g.pick_roots(0, 1)[0])
    bfs.run(root)
    assert np.array_equal(bfs.depths(), O.bfs_depth(off, adj, root))
    assert O.check(off, adj, root, bfs.parents())
    bfs.close()
    g.close()
