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


@pytest.mark.parametrize("order", [bd.ORDER_INSERTION, bd.ORDER_HUB])
def test_materialized_rows_equal_the_oracle(order):
    """materialize=True: the run itself leaves every root's depths and
    parents (caller ids, the reference's encoding) in device memory, written
    by one pass over each group's state.  Every lane of three groups (a
    partial last group, a duplicate root and a root of degree zero) must
    equal the oracle, and the rows read through the device pointers must
    equal the rows the copy-out path returns."""
    g = bd.Graph.rmat(15, 8, seed=48, order=order)
    off, adj = g.csr()
    deg = np.diff(off)
    roots = list(g.pick_roots(4, 150))
    roots[7] = roots[6]
    roots[140] = int(np.flatnonzero(deg == 0)[0])
    ms = bd.BatchedBFS(g, 150, materialize=True)
    for _ in range(2):  # the second run replays the captured graph
        ms.run(roots)
    _check_all(ms, off, adj, roots)
    n = g.num_vertices()
    for i in (0, 63, 64, 149):
        dp, pp = ms.device_results(i)
        assert np.array_equal(_device_to_host(dp, n, np.int32), ms.depths(i))
        assert np.array_equal(_device_to_host(pp, n, np.int64), ms.parents(i))


def _device_to_host(addr, n, dtype):
    """n elements at a borrowed device address, copied to a host array
    (through torch, which reads the CUDA array interface)."""
    torch = pytest.importorskip("torch")

    class View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str,
                                    "data": (addr, False), "version": 3}

    return torch.as_tensor(View(), device="cuda:0").cpu().numpy()


@pytest.mark.parametrize("order", [bd.ORDER_DEGREE, bd.ORDER_HUB])
def test_batched_min_parent_bit_exact(order):
    """min_parent=True: every root's parent tree is the smallest neighbour
    one level up, bit-exact against the oracle's min-parent tree, on 64
    roots at scale 16 (both numberings)."""
    g = bd.Graph.rmat(16, seed=49, order=order)
    off, adj = g.csr()
    roots = g.pick_roots(0, 64)
    ms = bd.BatchedBFS(g, 64, min_parent=True)
    ms.run(roots)
    m_c, _ = ms.counts()
    for i, root in enumerate(roots):
        root = int(root)
        depth = O.bfs_depth(off, adj, root)
        assert np.array_equal(ms.depths(i), depth)
        want = O.min_parent(off, adj, root, depth)
        got = ms.parents(i)
        assert np.array_equal(got, want), f"lane {i}: min-parent tree differs"
        assert m_c[i] == O.count_traversed(off, got)
