"""Connected components on the device (components.cc:38-118, :155-200).

Labels must equal the reference's exactly (each vertex labelled with the
smallest id of its component): against the reference's own output on the
fixture graphs (tests/golden/ref_components.npz), and against the oracle's
restatement of components::run elsewhere.  The device check() must give the
reference's own verdict on the fixtures' planted labellings and the
oracle's elsewhere, on correct and wrong labellings alike.  At RMAT scale 24
size-independent properties stand in: labels are minimum ids and fixed
points, sizes add up, the count equals the number of distinct labels,
check() passes, and a BFS from any vertex reaches exactly its label's
vertices.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")

HERE = os.path.dirname(os.path.abspath(__file__))


def _edges_from_csr(off, adj):
    src = np.repeat(np.arange(len(off) - 1, dtype=np.int64), np.diff(off))
    keep = src < adj
    return src[keep], adj[keep].astype(np.int64)


def _run(g):
    cc = bd.Components(g)
    st = cc.run()
    out = cc.labels(), cc.sizes(), st.num_components, cc.check()
    cc.close()
    return out


@pytest.mark.parametrize("name", ["scale10", "rmat12_ef2", "grid48", "tail_isolated", "tail_path"])
def test_labels_equal_the_reference(name):
    ref = np.load(os.path.join(HERE, "golden", "ref_components.npz"))
    off, adj = ref[f"{name}.offsets"], ref[f"{name}.adj"]
    want = ref[f"{name}.labels"]
    count = int(ref[f"{name}.summary"][0])
    src, dst = _edges_from_csr(off, adj)
    for g in (bd.Graph.from_csr(off, adj),  # no symmetry assumed: every arc joins
              bd.Graph.from_edges(len(off) - 1, src, dst),
              bd.Graph.from_edges(len(off) - 1, src, dst, order=bd.ORDER_HUB)):
        labels, sizes, k, ok = _run(g)
        assert np.array_equal(labels, want), name
        assert k == count and ok
        assert np.array_equal(sizes, np.bincount(want, minlength=len(want)))
        # the reference's own check() verdicts on planted labellings
        for i, (lab, v) in enumerate(zip(ref[f"{name}.planted"], ref[f"{name}.planted_verdict"])):
            assert g.check_components(lab)[0] == bool(v), (name, i)
        g.close()


@pytest.mark.parametrize("order", [bd.ORDER_INSERTION, bd.ORDER_HUB])
def test_rmat_and_grid_against_the_oracle(order):
    for g in (bd.Graph.rmat(14, seed=41, order=order), bd.Graph.rmat(13, 2, seed=42, order=order),
              bd.Graph.grid(120, 150, 0.45, seed=43, order=order)):
        off, adj = g.csr()
        want, want_sizes, count, _ = O.components(off, adj)
        labels, sizes, k, ok = _run(g)
        assert np.array_equal(labels, want)
        assert np.array_equal(sizes, want_sizes)
        assert k == count and ok
        g.close()


def test_heavy_vertices_and_small_graphs():
    # a star of 10,000 leaves around its highest id (a vertex split over the
    # grid: every join of the star comes from its arcs), a path, and isolated
    # vertices, packed into one graph
    star = bd.Graph.from_edges(10001, np.arange(10000, dtype=np.int64), np.full(10000, 10000, np.int64))
    path = bd.Graph.from_edges(3000, np.arange(2999, dtype=np.int64), np.arange(1, 3000, dtype=np.int64))
    alone = bd.Graph.from_edges(7, np.zeros(0, np.int64), np.zeros(0, np.int64))
    g, base = bd.Graph.concat([alone, star, path, alone])
    off, adj = g.csr()
    want, _, count, _ = O.components(off, adj)
    labels, sizes, k, ok = _run(g)
    assert np.array_equal(labels, want) and k == count == 7 + 1 + 1 + 7 and ok
    assert sizes[base[1]] == 10001 and sizes[base[2]] == 3000
    # no edges at all: every vertex is its own component
    labels, sizes, k, ok = _run(alone)
    assert np.array_equal(labels, np.arange(7)) and k == 7 and ok and (sizes == 1).all()


def test_relabelled_and_chain_graphs_against_the_oracle():
    # Ids in random order: the largest component's minimum id is no longer
    # a hub, so its root moves under smaller ones while joins race (the
    # finds read parent words that may be stale); a path over a random
    # permutation builds long chains of links; many small random cycles
    # give many roots.  Labels must still be the oracle's.
    rng = np.random.default_rng(77)
    base = bd.Graph.rmat(16, seed=61)
    src, dst = base.edges()
    n = base.num_vertices()
    perm = rng.permutation(n).astype(np.int64)
    graphs = [bd.Graph.from_edges(n, perm[src], perm[dst])]
    k = 50000
    walk = rng.permutation(k).astype(np.int64)
    graphs.append(bd.Graph.from_edges(k, walk[:-1], walk[1:]))
    sizes_c = rng.integers(3, 40, size=2000)
    order = rng.permutation(int(sizes_c.sum())).astype(np.int64)
    cs, cd, at = [], [], 0
    for c in sizes_c:
        ring = order[at:at + c]
        cs.append(ring)
        cd.append(np.roll(ring, 1))
        at += c
    graphs.append(bd.Graph.from_edges(int(sizes_c.sum()), np.concatenate(cs), np.concatenate(cd)))
    for g in graphs:
        off, adj = g.csr()
        want, want_sizes, count, _ = O.components(off, adj)
        labels, sizes, kk, ok = _run(g)
        assert np.array_equal(labels, want)
        assert np.array_equal(sizes, want_sizes)
        assert kk == count and ok
        g.close()
    base.close()


def test_check_agrees_with_the_oracle_on_planted_labels():
    g = bd.Graph.grid(60, 60, 0.4, seed=5)
    off, adj = g.csr()
    good, _, _, _ = O.components(off, adj)
    uniq, counts = np.unique(good, return_counts=True)
    big = int(uniq[np.argmax(counts)])
    other = int(uniq[uniq != big][0])
    members = np.flatnonzero(good == big)
    cases = {"good": good}
    bad = good.copy()
    bad[members[len(members) // 2]] = -7
    cases["one vertex relabelled"] = bad
    bad = good.copy()
    bad[good == other] = big
    cases["two components share a label"] = bad
    cases["distinct arbitrary labels"] = good * 3 + (1 << 40)
    swapped = good.copy()
    swapped[good == big], swapped[good == other] = other, big
    cases["labels swapped"] = swapped
    cases["all one label"] = np.zeros_like(good)
    for what, lab in cases.items():
        ok, where = g.check_components(lab)
        assert ok == O.components_check(off, adj, lab), what
        assert (where == -1) == ok, what
    with pytest.raises(ValueError):
        g.check_components(good[:-1])


def test_scale24_properties():
    g = bd.Graph.rmat(24, seed=24, order=bd.ORDER_HUB)
    cc = bd.Components(g)
    st = cc.run()
    st = cc.run()  # a second run starts over
    labels, sizes = cc.labels(), cc.sizes()
    assert cc.check()
    n = len(labels)
    v = np.arange(n)
    assert (labels <= v).all() and np.array_equal(labels[labels], labels)
    roots = np.flatnonzero(labels == v)
    assert st.num_components == len(roots) == len(np.unique(labels))
    assert sizes.sum() == n and np.array_equal(np.flatnonzero(sizes), roots)
    bfs = bd.HybridBFS(g)
    for root in g.pick_roots(0, 2):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        reached = bfs.depths() >= 0
        assert np.array_equal(reached, labels == labels[root])
        assert reached.sum() == sizes[labels[root]]
    print(f"scale 24: {st.num_components} components in {st.ms:.3f} ms")
    bfs.close()
    cc.close()
    g.close()


@pytest.mark.parametrize("name", ["scale10", "tail_path"])
def test_cli_matches_the_reference_output(name, tmp_path):
    """The components CLI on a fixture graph: counts, check() and the
    --dump_results text byte for byte as the reference's CLI printed it
    (on tail_path the last line has no newline, as in the reference)."""
    import re
    import subprocess
    cli = os.path.join(os.path.dirname(HERE), "beedrill_b200", "bin", "components")
    if not os.path.exists(cli):
        pytest.skip("CLI not built")
    ref = np.load(os.path.join(HERE, "golden", "ref_components.npz"))
    if name == "scale10":
        path = os.path.join(HERE, "golden", "graph500-scale10.el64")
    else:
        off, adj = ref[f"{name}.offsets"], ref[f"{name}.adj"]
        src, dst = _edges_from_csr(off, adj)
        path = str(tmp_path / f"{name}.el64")
        O.el64_write(path, len(off) - 1, src, dst)
    count = int(ref[f"{name}.summary"][0])
    out = subprocess.run([cli, "--graph_filename", path,
                          "--num_trials", "3", "--check_results", "--dump_results"],
                         stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=120)
    assert out.returncode == 0, out.stdout
    text = out.stdout
    assert text.count(f"Found {count} components in 1 iterations") == 3
    assert "Checking results...PASS" in text
    n = len(ref[f"{name}.labels"])
    labels = np.full(n, -1, np.int64)
    for m in re.finditer(r"Component (\d+): ((?:\d+(?:-\d+)?)(?:, \d+(?:-\d+)?)*)", text):
        for part in m.group(2).split(", "):
            lo, _, hi = part.partition("-")
            labels[int(lo): int(hi or lo) + 1] = int(m.group(1))
    assert np.array_equal(labels, ref[f"{name}.labels"])
    verdict = "Checking results...PASS\n"
    dump = text[text.rindex(verdict) + len(verdict):]
    assert dump.encode() == bytes(ref[f"{name}.dump"])