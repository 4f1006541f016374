"""The connected-components oracle against the reference's own build.

tests/golden/ref_components.npz holds what the reference's components CLI
(components_main.cc, built from its sources by oracle/Makefile) printed on
three graphs: labels (from --dump_results), component count, iteration
count and its check() verdict, plus the verdicts of the reference's own
components::check on planted labellings.  The oracle's restatement of
components::run must reproduce all of them, and its restatement of
components::check must give the reference's verdict on every labelling.
CPU only.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["scale10", "rmat12_ef2", "grid48", "tail_isolated", "tail_path"]


@pytest.fixture(scope="module")
def ref():
    O.build()
    return np.load(os.path.join(HERE, "golden", "ref_components.npz"))


@pytest.mark.parametrize("name", NAMES)
def test_components_match_the_reference(ref, name):
    off, adj = ref[f"{name}.offsets"], ref[f"{name}.adj"]
    count, iters, passed = ref[f"{name}.summary"].tolist()
    labels, sizes, k, it = O.components(off, adj)
    assert np.array_equal(labels, ref[f"{name}.labels"])
    assert (k, it) == (count, iters)
    assert passed == 1 and O.components_check(off, adj, labels)
    assert sizes.sum() == len(labels) and int((sizes > 0).sum()) == k
    assert np.array_equal(np.flatnonzero(sizes), np.unique(labels))


@pytest.mark.parametrize("name", NAMES)
def test_check_verdicts_equal_the_reference(ref, name):
    """The oracle's components::check gives the reference's own verdict
    (oracle/_ref/ref_components_check) on every planted labelling."""
    off, adj = ref[f"{name}.offsets"], ref[f"{name}.adj"]
    planted, want = ref[f"{name}.planted"], ref[f"{name}.planted_verdict"]
    assert len(planted) >= 6 and want.min() == 0 and want.max() == 1
    for i, (lab, v) in enumerate(zip(planted, want)):
        assert O.components_check(off, adj, lab) == bool(v), i


@pytest.mark.parametrize("name", NAMES)
def test_check_rule(ref, name):
    """components::check accepts any labelling that gives each component one
    label of its own, and nothing else."""
    off, adj = ref[f"{name}.offsets"], ref[f"{name}.adj"]
    good = ref[f"{name}.labels"]
    uniq, counts = np.unique(good, return_counts=True)
    big = int(uniq[np.argmax(counts)])
    other = int(uniq[uniq != big][0])
    members = np.flatnonzero(good == big)
    # one vertex of a component relabelled: its edges cross labels
    bad = good.copy()
    bad[members[len(members) // 2]] = -7
    assert not O.components_check(off, adj, bad)
    # two components share one label: the second is never visited
    bad = good.copy()
    bad[good == other] = big
    assert not O.components_check(off, adj, bad)
    # arbitrary but distinct labels per component pass
    relabel = good * 3 + (1 << 40)
    assert O.components_check(off, adj, relabel)
    swapped = good.copy()
    swapped[good == big], swapped[good == other] = other, big
    assert O.components_check(off, adj, swapped)


def _random_graph(rng, n, m):
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    keep = src != dst
    pairs = np.unique(np.sort(np.stack([src[keep], dst[keep]], 1), axis=1), axis=0)
    return O.csr_build(n, pairs[:, 0].astype(np.int64), pairs[:, 1].astype(np.int64))


@pytest.mark.parametrize("seed", range(6))
def test_components_against_scipy(seed):
    """Labels equal the minimum vertex id of each component as scipy's
    connected_components finds them, on sparse random graphs."""
    sp = pytest.importorskip("scipy.sparse")
    csgraph = pytest.importorskip("scipy.sparse.csgraph")
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 3000))
    off, adj = _random_graph(rng, n, int(rng.integers(0, 2 * n)))
    mat = sp.csr_matrix((np.ones(len(adj)), adj.astype(np.int64), off), shape=(n, n))
    k, comp = csgraph.connected_components(mat, directed=False)
    first = np.full(k, n, np.int64)
    np.minimum.at(first, comp, np.arange(n))
    labels, sizes, count, iters = O.components(off, adj)
    assert count == k and iters >= 1
    assert np.array_equal(labels, first[comp])
    assert np.array_equal(sizes[first], np.bincount(comp, minlength=k))
    # any one-to-one relabelling of the components passes the check
    perm = rng.permutation(k)
    assert O.components_check(off, adj, perm[comp] * 7 - 3)
    if k > 1:
        merged = comp.copy()
        merged[comp == 1] = 0
        assert not O.components_check(off, adj, merged)
