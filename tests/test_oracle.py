"""The CPU oracle, pinned against outputs of the reference itself.

The fixtures in tests/golden/ were produced by running the reference's own
sources (oracle/_ref, see tests/golden/make_golden.py).  These tests run on
CPU only and are the reason the oracle may be trusted as the parity checker
for the device path.
"""
import ctypes
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

REF_ALGS = ["beamer_hybrid", "migrating_threads", "remote_writes", "remote_writes_hybrid"]


@pytest.fixture(scope="module")
def scale10(golden_dir):
    path = os.path.join(golden_dir, "graph500-scale10.el64")
    n, src, dst = O.el64_load(path)
    off, adj = O.csr_build(n, src, dst)
    ref = dict(np.load(os.path.join(golden_dir, "ref_scale10.npz")))
    return n, src, dst, off, adj, ref


@pytest.fixture(scope="module")
def golden(golden_dir):
    with open(os.path.join(golden_dir, "golden.json")) as f:
        return json.load(f)


def test_el64_file_matches_fixture_hash(golden_dir, golden):
    path = os.path.join(golden_dir, "graph500-scale10.el64")
    h = hashlib.sha256(open(path, "rb").read()).hexdigest()
    assert h == golden["graph500-scale10.el64"]["sha256"]


def test_csr_insertion_order_matches_reference(scale10):
    n, src, dst, off, adj, ref = scale10
    assert np.array_equal(off, ref["offsets"])
    assert np.array_equal(adj, ref["adj"])
    assert O.graph_check(n, src, dst, off, adj)


def test_roots_match_reference_lcg(scale10):
    n, src, dst, off, adj, ref = scale10
    assert np.array_equal(O.pick_roots(off, 0, 8), ref["beamer_hybrid.roots"])


@pytest.mark.parametrize("alg", REF_ALGS)
def test_check_accepts_every_reference_tree(scale10, alg):
    n, src, dst, off, adj, ref = scale10
    for i, root in enumerate(ref[f"{alg}.roots"]):
        parent = ref[f"{alg}.parent"][i]
        assert ref[f"{alg}.check"][i]
        assert O.check(off, adj, int(root), parent)
        depth = O.bfs_depth(off, adj, int(root))
        assert np.array_equal(depth, O.depth_from_parents(parent, int(root)))
        assert O.count_traversed(off, parent) == ref[f"{alg}.m_c"][i]


def _ref_steps(heads):
    heads = heads[heads >= 0]
    return np.diff(heads)


def _ref_level_dirs(parent, flags, root):
    depth = O.depth_from_parents(parent, root)
    return "".join("B" if flags[depth == lv][0] else "T" for lv in range(1, depth.max() + 1))


def test_beamer_sequence_matches_reference(scale10):
    n, src, dst, off, adj, ref = scale10
    for alg in ("beamer_hybrid", "remote_writes_hybrid"):
        for i, root in enumerate(ref[f"{alg}.roots"]):
            root = int(root)
            depth = O.bfs_depth(off, adj, root)
            dirs, found = O.beamer_sequence(off, depth, root, len(src))
            assert np.array_equal(found, _ref_steps(ref[f"{alg}.heads"][i]))
            if alg == "beamer_hybrid":
                nonempty = dirs[: int(depth.max())]
                assert nonempty == _ref_level_dirs(ref[f"{alg}.parent"][i],
                                                   ref[f"{alg}.bottom_up"][i], root)


def test_serial_restatement_matches_reference(golden_dir):
    ref = dict(np.load(os.path.join(golden_dir, "ref_gen12.npz")))
    n, src, dst = O.rmat_graph(12, seed=12)
    assert len(src) == ref["num_edges"][0]
    off, adj = O.csr_build(n, src, dst)
    for i, root in enumerate(ref["roots"]):
        root = int(root)
        parent, depth, dirs = O.run_bfs(off, adj, root, len(src))
        rparent = ref["parent"][i]
        assert np.array_equal(depth, O.depth_from_parents(rparent, root))
        assert O.check(off, adj, root, parent)
        assert O.count_traversed(off, parent) == ref["m_c"][i]
        assert dirs[: int(depth.max())] == _ref_level_dirs(rparent, ref["bottom_up"][i], root)
        # bottom-up discoveries follow find.h's scan order, so they must pick
        # the very same parents as the serial reference
        bu = ref["bottom_up"][i].astype(bool)
        assert np.array_equal(parent[bu], rparent[bu])


def test_generator_scale12_bytes(golden):
    n, src, dst = O.rmat_graph(12, seed=12)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "g.el64")
        O.el64_write(path, n, src, dst)
        h = hashlib.sha256(open(path, "rb").read()).hexdigest()
    assert h == golden["gen12"]["el64_sha256"]


def test_scale16_depths_and_sequences(golden):
    g = golden["gen16"]
    n, src, dst = O.rmat_graph(16, seed=g["seed"])
    assert len(src) == g["num_edges"]
    off, adj = O.csr_build(n, src, dst)
    h = hashlib.sha256(off.astype("<i8").tobytes() + adj.astype("<u4").tobytes()).hexdigest()
    assert h == g["csr_sha256"]
    roots = O.pick_roots(off, 0, len(g["roots"]))
    for r, root in zip(g["roots"], roots):
        assert r["root"] == root
        depth = O.bfs_depth(off, adj, int(root))
        assert hashlib.sha256(depth.astype("<i4").tobytes()).hexdigest() == r["depth_sha256"]
        dirs, found = O.beamer_sequence(off, depth, int(root), len(src))
        assert found.tolist() == r["found"]
        assert dirs[: int(depth.max())] == r["level_dirs"]
        mp = O.min_parent(off, adj, int(root), depth)
        assert O.check(off, adj, int(root), mp)
        assert O.count_traversed(off, mp) == r["m_c"]


def test_check_equals_the_reference_check_on_planted_trees(scale10, golden_dir):
    """Verdict and stopping vertex of the oracle's check() equal the
    reference's own check() (oracle/_ref/ref_check, its LOG lines) on the
    reference's trees and on 63 copies with planted mistakes."""
    n, src, dst, off, adj, ref = scale10
    d = np.load(os.path.join(golden_dir, "ref_check.npz"))
    assert len(d["sources"]) > 60 and d["verdict"].sum() == 8
    for i, (s, p, v, w) in enumerate(zip(d["sources"], d["parents"], d["verdict"], d["stop"])):
        assert O.check(off, adj, int(s), p) == bool(v), i
        assert O.check_first_bad(off, adj, int(s), p) == w, i


def test_check_rejects_planted_mistakes(scale10):
    """Mistakes planted in a parent array on the CPU must fail check()."""
    n, src, dst, off, adj, ref = scale10
    root = int(ref["beamer_hybrid.roots"][0])
    good = ref["beamer_hybrid.parent"][0]
    depth = O.bfs_depth(off, adj, root)
    rng = np.random.default_rng(0)
    reached = np.flatnonzero((depth > 1))
    v = int(rng.choice(reached))
    # parent that is not a neighbour
    bad = good.copy()
    non_nbrs = np.setdiff1d(np.arange(n), adj[off[v]:off[v + 1]])
    bad[v] = int(non_nbrs[non_nbrs != v][0])
    assert not O.check(off, adj, root, bad)
    assert O.check_first_bad(off, adj, root, bad) == v
    # neighbour at the wrong depth
    same = [u for u in adj[off[v]:off[v + 1]] if depth[u] == depth[v]]
    if same:
        bad = good.copy()
        bad[v] = int(same[0])
        assert not O.check(off, adj, root, bad)
        assert O.check_first_bad(off, adj, root, bad) == v
    # reachable vertex left without a parent
    bad = good.copy()
    bad[v] = -1
    assert not O.check(off, adj, root, bad)
    assert O.check_first_bad(off, adj, root, bad) == v
    # source not its own parent
    bad = good.copy()
    bad[root] = int(adj[off[root]])
    assert not O.check(off, adj, root, bad)
    assert O.check_first_bad(off, adj, root, bad) == root
    # two mistakes: the check stops at the lower vertex
    w = int(rng.choice(reached[reached != v]))
    bad = good.copy()
    bad[v] = -1
    bad[w] = -1
    assert O.check_first_bad(off, adj, root, bad) == min(v, w)
    assert O.check_first_bad(off, adj, root, good) == -1


def test_el64_header_rules(tmp_path):
    def write(header, body=b""):
        p = tmp_path / "h.el64"
        p.write_bytes(header + body)
        return str(p)

    pair = np.array([[0, 1]], np.int64).tobytes()
    ok = b" --format el64 --num_edges 1 --num_vertices 2 --is_deduped\n"
    assert O.el64_header(write(ok, pair))[0] == 0
    assert O.el64_header(write(b" --format el32 --num_edges 1 --num_vertices 2 --is_deduped\n"))[0] == -4
    assert O.el64_header(write(b" --format el64 --num_edges 1 --num_vertices 2\n"))[0] == -5
    assert O.el64_header(write(b" --format el64 --num_edges 0 --num_vertices 2 --is_deduped\n"))[0] == -3
    assert O.el64_header(write(b" --format el64 --num_edges 1 --num_vertices 2 --is_deduped"))[0] == -2
    assert O.el64_header(write(b" --format el64 --bogus --num_edges 1 --num_vertices 2 --is_deduped\n"))[0] == -2


def _gen_cases(golden_dir):
    d = np.load(os.path.join(golden_dir, "ref_gen.npz"))
    for i, ((scale, ef, seed), (a, b, c, dd)) in enumerate(zip(d["cases"], d["params"])):
        yield i, int(scale), int(ef), float(a), float(b), float(c), float(dd), int(seed), d


def test_reference_stream_restatement_matches_the_reference_generator(golden_dir):
    """The oracle's restatement of the reference generator (sitmo stream,
    libstdc++ uniform doubles, next_edge, rmat_fill's serial self-loop
    re-roll; then flip / sort / dedup) gives, on every fixture case, the
    reference's own generated list and deduplicated list (ref_gen_edges,
    tests/golden/ref_gen.npz) byte for byte."""
    import hashlib
    for i, scale, ef, a, b, c, d, seed, fx in _gen_cases(golden_dir):
        src, dst = O.rmat_stream_edges(scale, ef << scale, a, b, c, d, seed)
        gen = np.stack([src, dst], axis=1)
        counts = fx[f"{i}.counts"]
        assert len(gen) == counts[1] and (src != dst).all(), i
        assert hashlib.sha256(gen.tobytes()).digest() == bytes(fx[f"{i}.gen_sha"]), i
        s, t = O.dedup_sorted(src, dst)
        ded = np.stack([s, t], axis=1)
        assert len(ded) == counts[2], i
        assert hashlib.sha256(ded.tobytes()).digest() == bytes(fx[f"{i}.ded_sha"]), i
        if i == 0:
            assert np.array_equal(gen, fx["0.gen"]) and np.array_equal(ded, fx["0.ded"])


def test_reference_stream_and_the_reference_el64_file(golden_dir):
    """graph500-scale10.el64, written by the reference's rmat_dataset_dump,
    is the oracle's deduplicated scale-10 list after a vertex relabel and an
    edge shuffle: same edge count, same multiset of degrees, same multiset
    of per-edge degree pairs."""
    n, src, dst = O.rmat_stream_graph(10, 16, seed=0)
    n2, s2, d2 = O.el64_load(os.path.join(golden_dir, "graph500-scale10.el64"))
    assert n == n2 and len(src) == len(s2)
    deg = np.bincount(np.concatenate([src, dst]), minlength=n)
    deg2 = np.bincount(np.concatenate([s2, d2]), minlength=n)
    assert np.array_equal(np.sort(deg), np.sort(deg2))
    pairs = np.sort(np.sort(np.stack([deg[src], deg[dst]], 1), axis=1), axis=0)
    pairs2 = np.sort(np.sort(np.stack([deg2[s2], deg2[d2]], 1), axis=1), axis=0)
    assert np.array_equal(np.sort(pairs.view([("a", np.int64), ("b", np.int64)]), axis=0),
                          np.sort(pairs2.view([("a", np.int64), ("b", np.int64)]), axis=0))


def test_threefish20_stream_positions():
    """Output t of the engine is half of block t / 8: the sequential reader
    and direct access by position agree, across block boundaries."""
    ts = [0, 1, 2, 7, 8, 9, 15, 16, 1 << 20, (1 << 33) + 5]
    for seed in (0, 1, 0xFFFFFFFF):
        for t in ts:
            out = (ctypes.c_uint64 * 4)()
            O.lib().or_threefish20(seed, t >> 3, out)
            w = out[(t & 7) >> 1]
            want = (w >> 32) if t & 1 else (w & 0xFFFFFFFF)
            assert O.lib().or_sitmo_output(seed, t) == want
