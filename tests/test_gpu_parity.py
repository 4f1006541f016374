"""Parity of the CUDA path with the oracle and the reference's own outputs.

Every call goes through the C ABI (beedrill_b200 -> libbeedrill_b200.so).
The bar: depth arrays bit-exact, every parent tree passes the reference's
check(), min-parent trees bit-exact, direction sequences and per-step counts
equal to the reference's run_beamer, m_c equal to
count_num_traversed_edges().
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")


@pytest.fixture(scope="module")
def golden(golden_dir):
    with open(os.path.join(golden_dir, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def scale10(golden_dir):
    path = os.path.join(golden_dir, "graph500-scale10.el64")
    g = bd.Graph.from_el64(path)
    n, src, dst = O.el64_load(path)
    off, adj = O.csr_build(n, src, dst)
    ref = dict(np.load(os.path.join(golden_dir, "ref_scale10.npz")))
    return g, off, adj, len(src), ref


def _sha(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a).astype(dtype).tobytes()).hexdigest()


def _assert_run_matches(bfs, off, adj, m, root, alg):
    depth = bfs.depths()
    want = O.bfs_depth(off, adj, root)
    assert np.array_equal(depth, want), f"{alg} root {root}: depth mismatch"
    parent = bfs.parents()
    assert O.check(off, adj, root, parent), f"{alg} root {root}: check() failed"
    assert bfs.check(root)
    m_c = O.count_traversed(off, parent)
    assert bfs.count_num_traversed_edges() == m_c
    if alg == "beamer_hybrid":
        dirs, found = O.beamer_sequence(off, want, root, m)
        assert bfs.directions() == dirs
        assert [s["found"] for s in bfs.steps()] == found.tolist()
    return depth, parent


def test_csr_matches_reference_build(scale10):
    g, off, adj, m, ref = scale10
    goff, gadj = g.csr()
    assert np.array_equal(goff, ref["offsets"])
    assert np.array_equal(gadj, ref["adj"])
    assert g.check()


def test_roots_match_reference(scale10):
    g, off, adj, m, ref = scale10
    assert np.array_equal(g.pick_roots(0, 8), ref["beamer_hybrid.roots"])


@pytest.mark.parametrize("alg", ["beamer_hybrid", "top_down", "bottom_up", "remote_writes_hybrid",
                                 "migrating_threads", "remote_writes"])
def test_scale10_all_algorithms(scale10, alg):
    g, off, adj, m, ref = scale10
    bfs = bd.HybridBFS(g, alg=alg)
    for i, root in enumerate(ref["beamer_hybrid.roots"]):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        _assert_run_matches(bfs, off, adj, m, root, "beamer_hybrid" if "hybrid" in alg else alg)
        assert bfs.count_num_traversed_edges() == ref["beamer_hybrid.m_c"][i]


def test_generator_bytes_match_oracle(golden, tmp_path):
    for key in ("gen12", "gen16"):
        spec = golden[key]
        g = bd.Graph.rmat(spec["scale"], seed=spec["seed"])
        path = str(tmp_path / f"{key}.el64")
        g.write_el64(path)
        h = hashlib.sha256(open(path, "rb").read()).hexdigest()
        assert h == spec["el64_sha256"], key
        assert g.num_edges() == spec["num_edges"]


def test_generator_other_parameters_match_oracle():
    for scale, ef, a, seed in [(9, 4, 0.45, 7), (11, 32, 0.65, 123), (6, 8, 0.57, 1 << 40)]:
        d = 0.05
        b = c = (1 - a - d) / 2
        g = bd.Graph.rmat(scale, ef, a, b, c, d, seed)
        n, src, dst = O.rmat_graph(scale, ef, a, b, c, d, seed)
        gs, gd = g.edges()
        assert np.array_equal(gs, src) and np.array_equal(gd, dst)


def test_scale16_against_reference_hashes(golden):
    spec = golden["gen16"]
    g = bd.Graph.rmat(16, seed=spec["seed"])
    off, adj = g.csr()
    h = hashlib.sha256(off.astype("<i8").tobytes() + adj.astype("<u4").tobytes()).hexdigest()
    assert h == spec["csr_sha256"]
    bfs = bd.HybridBFS(g)
    roots = g.pick_roots(0, len(spec["roots"]))
    for r, root in zip(spec["roots"], roots):
        assert int(root) == r["root"]
        bfs.clear()
        st = bfs.run_beamer(int(root), 15, 18)
        depth = bfs.depths()
        assert _sha(depth, "<i4") == r["depth_sha256"]
        assert st.traversed_edges == r["m_c"]
        assert [s["found"] for s in bfs.steps()] == r["found"]
        assert bfs.directions()[: int(depth.max())] == r["level_dirs"]
        assert O.check(off, adj, int(root), bfs.parents())


def test_min_parent_bit_exact(golden):
    g = bd.Graph.rmat(14, seed=5)
    off, adj = g.csr()
    m = g.num_edges()
    for alg in ("beamer_hybrid", "top_down", "bottom_up"):
        bfs = bd.HybridBFS(g, alg=alg, min_parent=True)
        for root in g.pick_roots(3, 4):
            root = int(root)
            bfs.clear()
            bfs.run(root)
            depth = O.bfs_depth(off, adj, root)
            assert np.array_equal(bfs.depths(), depth)
            assert np.array_equal(bfs.parents(), O.min_parent(off, adj, root, depth))


def test_sorted_adjacency_bottom_up_gives_min_parents():
    g = bd.Graph.rmat(13, seed=9, order=bd.ORDER_SORTED)
    off, adj = g.csr()
    for v in range(len(off) - 1):
        assert np.all(np.diff(adj[off[v]:off[v + 1]].astype(np.int64)) > 0)
    bfs = bd.HybridBFS(g, alg="bottom_up")
    root = int(g.pick_roots(0, 1)[0])
    bfs.run(root)
    depth = O.bfs_depth(off, adj, root)
    assert np.array_equal(bfs.depths(), depth)
    assert np.array_equal(bfs.parents(), O.min_parent(off, adj, root, depth))


def test_graph_from_host_csr_and_edges():
    n, src, dst = O.rmat_graph(11, seed=2)
    off, adj = O.csr_build(n, src, dst)
    g1 = bd.Graph.from_csr(off, adj)
    g2 = bd.Graph.from_edges(n, src, dst)
    for g in (g1, g2):
        goff, gadj = g.csr()
        assert np.array_equal(goff, off) and np.array_equal(gadj, adj)
        bfs = bd.HybridBFS(g)
        root = int(O.pick_roots(off, 0, 1)[0])
        bfs.run(root)
        assert np.array_equal(bfs.depths(), O.bfs_depth(off, adj, root))


def test_packed_graphs_multi_source():
    rng = np.random.default_rng(4)
    parts = []
    for i in range(12):
        parts.append(bd.Graph.rmat(int(rng.integers(5, 11)), int(rng.integers(2, 20)), seed=100 + i))
    g, base = bd.Graph.concat(parts)
    roots = []
    for i, p in enumerate(parts):
        roots.append(int(p.pick_roots(i, 1)[0]) + int(base[i]))
    bfs = bd.HybridBFS(g)
    bfs.run_multi(roots)
    depth = bfs.depths()
    parent = bfs.parents()
    for i, p in enumerate(parts):
        off, adj = p.csr()
        lo, hi = int(base[i]), int(base[i + 1])
        want = O.bfs_depth(off, adj, roots[i] - lo)
        assert np.array_equal(depth[lo:hi], want)
        local = parent[lo:hi].copy()
        local[local >= 0] -= lo
        assert O.check(off, adj, roots[i] - lo, local)


def test_scale20_depths_and_check():
    g = bd.Graph.rmat(20, seed=20)
    off, adj = g.csr()
    m = g.num_edges()
    bfs = bd.HybridBFS(g)
    for root in g.pick_roots(0, 3):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        _assert_run_matches(bfs, off, adj, m, root, "beamer_hybrid")


def test_run_many_matches_single_runs():
    g = bd.Graph.rmat(15, seed=3)
    roots = g.pick_roots(0, 6)
    bfs = bd.HybridBFS(g)
    ms, edges, e2e = bfs.run_many(roots)
    assert np.all(ms > 0) and e2e >= ms.sum() * 0.5
    for r, e in zip(roots, edges):
        bfs.clear()
        assert bfs.run(int(r)).traversed_edges == e


def test_errors_are_status_codes(tmp_path):
    g = bd.Graph.rmat(8, seed=1)
    bfs = bd.HybridBFS(g)
    with pytest.raises(bd.BeedrillError) as ei:
        bfs.run(g.num_vertices())
    assert ei.value.status == -7  # BD_ERR_RANGE
    with pytest.raises(bd.BeedrillError) as ei:
        bd.Graph.from_el64(str(tmp_path / "missing.el64"))
    assert ei.value.status == -2
    bad = tmp_path / "bad.el64"
    bad.write_bytes(b" --format el64 --num_edges 1 --num_vertices 2\n" + bytes(16))
    with pytest.raises(bd.BeedrillError) as ei:
        bd.Graph.from_el64(str(bad))
    assert ei.value.status == -3
    short = tmp_path / "short.el64"
    short.write_bytes(b" --format el64 --num_edges 4 --num_vertices 8 --is_deduped\n" + bytes(16))
    with pytest.raises(bd.BeedrillError) as ei:
        bd.Graph.from_el64(str(short))
    assert ei.value.status == -3
    oob = tmp_path / "oob.el64"
    oob.write_bytes(b" --format el64 --num_edges 1 --num_vertices 2 --is_deduped\n"
                    + np.array([0, 5], np.int64).tobytes())
    with pytest.raises(bd.BeedrillError) as ei:
        bd.Graph.from_el64(str(oob))
    assert ei.value.status == -7


def test_barrier_timeout_is_reported_and_recoverable():
    """The grid barrier waits for one CTA more than the launch has, so it can
    never complete: every CTA gives up after its short poll limit, the kernel
    returns and the host reads BD_ERR_TIMEOUT.  The context stays usable."""
    g = bd.Graph.rmat(10, seed=1)
    off, adj = g.csr()
    root = int(g.pick_roots(0, 1)[0])
    stuck = bd.HybridBFS(g, spin_limit=2000, test_extra_ctas=1)
    with pytest.raises(bd.BeedrillError) as ei:
        stuck.run(root)
    assert ei.value.status == -6  # BD_ERR_TIMEOUT
    stuck.close()
    bfs = bd.HybridBFS(g)
    bfs.run(root)
    assert np.array_equal(bfs.depths(), O.bfs_depth(off, adj, root))


def test_degree_order_lists_and_results():
    g = bd.Graph.rmat(14, seed=15, order=bd.ORDER_DEGREE)
    ref = bd.Graph.rmat(14, seed=15)
    off, adj = g.csr()
    roff, radj = ref.csr()
    assert np.array_equal(off, roff)
    deg = np.diff(off)
    for v in range(0, len(off) - 1, 97):
        lst = adj[off[v]:off[v + 1]]
        assert np.array_equal(np.sort(lst), np.sort(radj[roff[v]:roff[v + 1]]))
        assert np.all(np.diff(deg[lst]) <= 0)
    m = g.num_edges()
    for alg in ("beamer_hybrid", "bottom_up", "top_down"):
        bfs = bd.HybridBFS(g, alg=alg)
        for root in g.pick_roots(0, 3):
            root = int(root)
            bfs.clear()
            bfs.run(root)
            _assert_run_matches(bfs, off, adj, m, root, alg)
    ms = bd.BatchedBFS(g, 64)
    roots = g.pick_roots(1, 64)
    ms.run(roots)
    for i in range(0, 64, 9):
        assert np.array_equal(ms.depths(i), O.bfs_depth(off, adj, int(roots[i])))
        assert O.check(off, adj, int(roots[i]), ms.parents(i))
