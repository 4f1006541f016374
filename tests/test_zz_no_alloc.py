"""bd_bfs_run_noalloc: the BFS entry point that allocates no device memory.

It serves callers that must not allocate on the call path (device memory
reserved up front by their own pool allocator, or no tolerance for the
device-wide synchronisation cudaMalloc / cudaFree can cause).  Its
temporaries live in a fixed array inside the library; the caller brings the
CSR and the output arrays.

This file is collected last on purpose.  The test calls the new entry point
through the C ABI twice in a row (different roots, so stale scratch from the
first call would show) and compares each result with the regular entry point
(bd_bfs_run on a HybridBFS handle) and with the oracle on the same graph and
root: depths bit-exact against both, m_c equal, and the parent tree must
pass the reference's check().  The device's free memory must be the same
before and after the second call (the first one only looks the scratch
array up).
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

bd = pytest.importorskip("beedrill_b200")
torch = pytest.importorskip("torch")

MAX_VERTICES = 524288
BD_ERR_LIMIT = -10


def _fn():
    f = bd.lib().bd_bfs_run_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                  ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.POINTER(ctypes.c_int64)]
    return f


def _device_csr(g):
    off_p = ctypes.c_void_p()
    adj_p = ctypes.c_void_p()
    assert bd.lib().bd_graph_device_csr(g._h, ctypes.byref(off_p), ctypes.byref(adj_p)) == 0
    return off_p.value, adj_p.value


@pytest.mark.parametrize("scale", [16, 19])
def test_noalloc_matches_regular_entry_point(scale):
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    torch.cuda.set_device(0)
    bd.lib().bd_set_device(0)
    g = bd.Graph.rmat(scale, 16, seed=77 + scale)
    n, m = g.num_vertices(), g.num_edges()
    assert n <= MAX_VERTICES
    off, adj = g.csr()
    d_off, d_adj = _device_csr(g)
    depth = torch.empty(n, dtype=torch.int32, device="cuda:0")
    parent = torch.empty(n, dtype=torch.int64, device="cuda:0")
    regular = bd.HybridBFS(g, alg="beamer_hybrid")
    run = _fn()
    for i, root in enumerate(g.pick_roots(5, 2)):  # two calls in a row
        root = int(root)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        edges = ctypes.c_int64(-1)
        st = run(d_off, d_adj, n, len(adj), root, 15, 18, depth.data_ptr(), parent.data_ptr(),
                 None, ctypes.byref(edges))
        assert st == 0, bd.lib().bd_status_string(st)
        torch.cuda.synchronize()
        if i == 1:
            assert torch.cuda.mem_get_info(0)[0] == free_before, "the call allocated device memory"
        got_depth = depth.cpu().numpy()
        got_parent = parent.cpu().numpy()
        assert np.array_equal(got_depth, O.bfs_depth(off, adj, root))
        regular.clear()
        stats = regular.run(root)
        assert np.array_equal(got_depth, regular.depths())
        assert edges.value == stats.traversed_edges
        assert O.check(off, adj, root, got_parent)
        assert O.count_traversed(off, got_parent) == edges.value


def test_noalloc_rejects_graphs_beyond_its_limit():
    run = _fn()
    edges = ctypes.c_int64(0)
    # sizes are checked before anything touches the pointers
    st = run(16, 16, MAX_VERTICES + 1, 2, 0, 15, 18, 16, 16, None, ctypes.byref(edges))
    assert st == BD_ERR_LIMIT
