"""ctypes view of the CPU oracle (liboracle.so, built from bfs_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product package
(beedrill_b200) never imports it.

Every wrapper takes and returns numpy arrays; the C functions cite the
reference lines they restate.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int64, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build() -> None:
    """Compile liboracle.so (and the reference builds when the reference
    sources are present) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        i64p = POINTER(c_int64)
        u32p = POINTER(c_uint32)
        i32p = POINTER(ctypes.c_int32)
        L.or_el64_header.argtypes = [c_char_p, i64p, i64p, i64p]
        L.or_el64_load.argtypes = [c_char_p, i64p, i64p, c_int64]
        L.or_el64_write.argtypes = [c_char_p, c_int64, c_int64, i64p, i64p]
        L.or_csr_build.argtypes = [c_int64, c_int64, i64p, i64p, i64p, u32p]
        L.or_graph_check.argtypes = [c_int64, c_int64, i64p, i64p, i64p, u32p]
        L.or_pick_roots.argtypes = [c_int64, i64p, c_uint64, c_int64, i64p]
        L.or_pick_roots.restype = None
        L.or_bfs_depth.argtypes = [c_int64, i64p, u32p, c_int64, i32p]
        L.or_bfs_depth.restype = None
        L.or_check.argtypes = [c_int64, i64p, u32p, c_int64, i64p, i32p]
        L.or_check_first_bad.argtypes = [c_int64, i64p, u32p, c_int64, i64p, i32p]
        L.or_check_first_bad.restype = c_int64
        L.or_components.argtypes = [c_int64, i64p, u32p, i64p, i64p, i64p]
        L.or_components.restype = c_int64
        L.or_components_check.argtypes = [c_int64, i64p, u32p, i64p]
        L.or_min_parent.argtypes = [c_int64, i64p, u32p, c_int64, i32p, i64p]
        L.or_min_parent.restype = None
        L.or_count_traversed.argtypes = [c_int64, i64p, i64p]
        L.or_count_traversed.restype = c_int64
        L.or_beamer_sequence.argtypes = [c_int64, c_int64, i64p, i32p, c_int64, c_int64,
                                         c_int64, c_char_p, i64p, c_int]
        L.or_run_bfs.argtypes = [c_int64, c_int64, i64p, u32p, c_int64, c_int64, c_int64,
                                 c_int, i64p, i32p, c_char_p, c_int]
        L.or_philox4x32.argtypes = [u32p, u32p, u32p]
        L.or_philox4x32.restype = None
        L.or_rmat_edges.argtypes = [c_int, c_int64, c_double, c_double, c_double, c_double,
                                    c_uint64, i64p, i64p]
        L.or_rmat_edges.restype = None
        L.or_rmat_finish.argtypes = [c_int, c_int64, c_uint64, i64p, i64p]
        L.or_rmat_finish.restype = c_int64
        L.or_grid_edges.argtypes = [c_int64, c_int64, c_double, c_uint64, i64p, i64p]
        L.or_grid_edges.restype = c_int64
        L.or_threefish20.argtypes = [c_uint64, c_uint64, POINTER(c_uint64)]
        L.or_threefish20.restype = None
        L.or_sitmo_output.argtypes = [ctypes.c_uint32, c_uint64]
        L.or_sitmo_output.restype = ctypes.c_uint32
        L.or_rmat_stream_edges.argtypes = [c_int, c_int64, c_double, c_double, c_double,
                                           c_double, ctypes.c_uint32, i64p, i64p]
        L.or_rmat_stream_edges.restype = c_int
        _lib = L
    return _lib


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(POINTER(ct))


# --------------------------------------------------------------------------
# el64 / graph construction
# --------------------------------------------------------------------------

def el64_header(path: str):
    n, m, hb = c_int64(), c_int64(), c_int64()
    rc = lib().or_el64_header(path.encode(), ctypes.byref(n), ctypes.byref(m), ctypes.byref(hb))
    return rc, n.value, m.value, hb.value


def el64_load(path: str):
    rc, n, m, _ = el64_header(path)
    if rc:
        raise ValueError(f"el64 header rejected ({rc}): {path}")
    src = np.empty(m, np.int64)
    dst = np.empty(m, np.int64)
    rc = lib().or_el64_load(path.encode(), _p(src, c_int64), _p(dst, c_int64), m)
    if rc:
        raise ValueError(f"el64 body rejected ({rc}): {path}")
    return n, src, dst


def el64_write(path: str, n: int, src: np.ndarray, dst: np.ndarray) -> None:
    src = np.ascontiguousarray(src, np.int64)
    dst = np.ascontiguousarray(dst, np.int64)
    rc = lib().or_el64_write(path.encode(), n, len(src), _p(src, c_int64), _p(dst, c_int64))
    if rc:
        raise OSError(f"el64 write failed ({rc}): {path}")


def csr_build(n: int, src: np.ndarray, dst: np.ndarray):
    src = np.ascontiguousarray(src, np.int64)
    dst = np.ascontiguousarray(dst, np.int64)
    off = np.empty(n + 1, np.int64)
    adj = np.empty(2 * len(src), np.uint32)
    rc = lib().or_csr_build(n, len(src), _p(src, c_int64), _p(dst, c_int64),
                            _p(off, c_int64), _p(adj, c_uint32))
    if rc:
        raise ValueError(f"edge endpoint out of range ({rc})")
    return off, adj


def graph_check(n, src, dst, off, adj) -> bool:
    return bool(lib().or_graph_check(n, len(src), _p(src, c_int64), _p(dst, c_int64),
                                     _p(off, c_int64), _p(adj, c_uint32)))


def pick_roots(off: np.ndarray, seed: int, k: int) -> np.ndarray:
    roots = np.empty(k, np.int64)
    lib().or_pick_roots(len(off) - 1, _p(off, c_int64), seed, k, _p(roots, c_int64))
    return roots


# --------------------------------------------------------------------------
# BFS oracles
# --------------------------------------------------------------------------

def bfs_depth(off, adj, source: int) -> np.ndarray:
    depth = np.empty(len(off) - 1, np.int32)
    lib().or_bfs_depth(len(off) - 1, _p(off, c_int64), _p(adj, c_uint32), source,
                       _p(depth, ctypes.c_int32))
    return depth


def check(off, adj, source: int, parent: np.ndarray) -> bool:
    parent = np.ascontiguousarray(parent, np.int64)
    scratch = np.empty(len(off) - 1, np.int32)
    return bool(lib().or_check(len(off) - 1, _p(off, c_int64), _p(adj, c_uint32), source,
                               _p(parent, c_int64), _p(scratch, ctypes.c_int32)))


def check_first_bad(off, adj, source: int, parent: np.ndarray) -> int:
    """The vertex at which hybrid_bfs::check stops (hybrid_bfs.cc:331-376), or -1."""
    parent = np.ascontiguousarray(parent, np.int64)
    scratch = np.empty(len(off) - 1, np.int32)
    return int(lib().or_check_first_bad(len(off) - 1, _p(off, c_int64), _p(adj, c_uint32), source,
                                        _p(parent, c_int64), _p(scratch, ctypes.c_int32)))


def components(off, adj):
    """(labels, sizes, num_components, num_iters) of components::run
    (components.cc:38-118) in its serial-elision order."""
    n = len(off) - 1
    comp = np.empty(n, np.int64)
    size = np.empty(n, np.int64)
    count = c_int64()
    iters = lib().or_components(n, _p(off, c_int64), _p(adj, c_uint32), _p(comp, c_int64),
                                _p(size, c_int64), ctypes.byref(count))
    return comp, size, int(count.value), int(iters)


def components_check(off, adj, labels: np.ndarray) -> bool:
    """components::check (components.cc:155-200) of any labelling."""
    labels = np.ascontiguousarray(labels, np.int64)
    return bool(lib().or_components_check(len(off) - 1, _p(off, c_int64), _p(adj, c_uint32),
                                          _p(labels, c_int64)))


def min_parent(off, adj, source: int, depth: np.ndarray) -> np.ndarray:
    depth = np.ascontiguousarray(depth, np.int32)
    parent = np.empty(len(off) - 1, np.int64)
    lib().or_min_parent(len(off) - 1, _p(off, c_int64), _p(adj, c_uint32), source,
                        _p(depth, ctypes.c_int32), _p(parent, c_int64))
    return parent


def count_traversed(off, parent) -> int:
    parent = np.ascontiguousarray(parent, np.int64)
    return int(lib().or_count_traversed(len(off) - 1, _p(off, c_int64), _p(parent, c_int64)))


def beamer_sequence(off, depth, source: int, m: int, alpha: int = 15, beta: int = 18):
    """(direction string, per-step discovered counts) of run_beamer."""
    depth = np.ascontiguousarray(depth, np.int32)
    cap = int(depth.max()) + 8
    buf = ctypes.create_string_buffer(cap + 1)
    found = np.zeros(cap, np.int64)
    steps = lib().or_beamer_sequence(len(off) - 1, m, _p(off, c_int64),
                                     _p(depth, ctypes.c_int32), source, alpha, beta,
                                     buf, _p(found, c_int64), cap)
    if steps < 0:
        raise RuntimeError("step buffer too small")
    return buf.value.decode(), found[:steps].copy()


MODES = {"beamer_hybrid": 0, "top_down": 1, "bottom_up": 2}


def run_bfs(off, adj, source: int, m: int, mode: str = "beamer_hybrid",
            alpha: int = 15, beta: int = 18):
    """Serial restatement of run_beamer / top-down / bottom-up.
    Returns (parent, depth, direction string)."""
    n = len(off) - 1
    parent = np.empty(n, np.int64)
    depth = np.empty(n, np.int32)
    cap = n + 8
    buf = ctypes.create_string_buffer(cap + 1)
    steps = lib().or_run_bfs(n, m, _p(off, c_int64), _p(adj, c_uint32), source, alpha, beta,
                             MODES[mode], _p(parent, c_int64), _p(depth, ctypes.c_int32),
                             buf, cap)
    if steps < 0:
        raise MemoryError("oracle BFS allocation failed")
    return parent, depth, buf.value.decode()


# --------------------------------------------------------------------------
# Seeded RMAT generator (the project's generator, restated)
# --------------------------------------------------------------------------

def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.empty(4, np.uint32)
    lib().or_philox4x32(_p(c, c_uint32), _p(k, c_uint32), _p(out, c_uint32))
    return out


def rmat_edges(scale: int, num_edges: int, a=0.57, b=0.19, c=0.19, d=0.05, seed: int = 0):
    src = np.empty(num_edges, np.int64)
    dst = np.empty(num_edges, np.int64)
    lib().or_rmat_edges(scale, num_edges, a, b, c, d, seed, _p(src, c_int64), _p(dst, c_int64))
    return src, dst


def rmat_graph(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, d=0.05,
               seed: int = 0):
    """Edge list of the seeded RMAT graph: (n, src, dst) after flip, sort,
    dedup, relabel and shuffle."""
    num_edges = edge_factor << scale
    src, dst = rmat_edges(scale, num_edges, a, b, c, d, seed)
    m = lib().or_rmat_finish(scale, num_edges, seed, _p(src, c_int64), _p(dst, c_int64))
    if m < 0:
        raise MemoryError("oracle generator allocation failed")
    return 1 << scale, src[:m].copy(), dst[:m].copy()


def rmat_stream_edges(scale: int, num_edges: int, a=0.57, b=0.19, c=0.19, d=0.05,
                      seed: int = 0):
    """Edges of the reference generator (rmat_edge_generator(2^scale, a, b,
    c, d, seed) + rmat_fill, rmat_generator.h:70-193, run serially) in
    generation order, self loops re-rolled."""
    src = np.empty(num_edges, np.int64)
    dst = np.empty(num_edges, np.int64)
    if lib().or_rmat_stream_edges(scale, num_edges, a, b, c, d, seed, _p(src, c_int64),
                                  _p(dst, c_int64)):
        raise ValueError("self loops never end for these RMAT parameters")
    return src, dst


def dedup_sorted(src: np.ndarray, dst: np.ndarray):
    """flip_edges, sort_edges, dedup_edges (edge_list_utils.h:14-56): the
    edge list with src < dst, sorted by (src, dst), without repeats."""
    lo = np.minimum(src, dst)
    hi = np.maximum(src, dst)
    pairs = np.unique(np.stack([lo, hi], axis=1), axis=0)
    return pairs[:, 0].copy(), pairs[:, 1].copy()


def rmat_stream_graph(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, d=0.05,
                      seed: int = 0):
    """(n, src, dst): the reference generator's deduplicated, sorted edge
    list (rmat_dataset_dump.cc:43-53), before its relabel and shuffle."""
    src, dst = rmat_stream_edges(scale, edge_factor << scale, a, b, c, d, seed)
    s, t = dedup_sorted(src, dst)
    return 1 << scale, s, t


def grid_graph(rows: int, cols: int, delete_frac: float = 0.01, seed: int = 0):
    """Edge list of the project's seeded grid graph: (n, src, dst)."""
    total = rows * (cols - 1) + (rows - 1) * cols
    src = np.empty(max(total, 1), np.int64)
    dst = np.empty(max(total, 1), np.int64)
    m = lib().or_grid_edges(rows, cols, delete_frac, seed, _p(src, c_int64), _p(dst, c_int64))
    return rows * cols, src[:m].copy(), dst[:m].copy()


def depth_from_parents(parent: np.ndarray, source: int) -> np.ndarray:
    """Depth of every vertex in a parent tree (reference encoding);
    -1 for unreached vertices."""
    n = len(parent)
    depth = np.full(n, -1, np.int32)
    depth[source] = 0
    reached = np.flatnonzero(parent >= 0)
    pending = reached[reached != source]
    # Resolve level by level: a vertex gets depth once its parent has one.
    while len(pending):
        par = parent[pending]
        ready = depth[par] >= 0
        if not ready.any():
            raise ValueError("parent tree has a cycle or dangling parent")
        depth[pending[ready]] = depth[par[ready]] + 1
        pending = pending[~ready]
    return depth


# --------------------------------------------------------------------------
# Reference runs (oracle/_ref, built from the reference sources)
# --------------------------------------------------------------------------

def read_ref_dump(path: str):
    """Parse the file written by oracle/_ref/ref_dump (layout in ref_dump.cc)."""
    raw = open(path, "rb").read()
    if raw[:8] != b"BDREF001":
        raise ValueError("not a ref_dump file")
    pos = 8

    def i64(count=1):
        nonlocal pos
        a = np.frombuffer(raw, np.int64, count, pos)
        pos += 8 * count
        return a

    n, m, k, has_graph = (int(x) for x in i64(4))
    out = {"n": n, "m": m, "roots": []}
    if has_graph:
        out["offsets"] = i64(n + 1).copy()
        out["adj"] = i64(2 * m).astype(np.uint32)
    for _ in range(k):
        root, ok, mc = (int(x) for x in i64(3))
        ms = float(np.frombuffer(raw, np.float64, 1, pos)[0])
        pos += 8
        nw = int(i64()[0])
        heads = i64(nw).copy()
        parent = i64(n).copy()
        flag = np.frombuffer(raw, np.uint8, n, pos).copy()
        pos += n
        out["roots"].append({"root": root, "check": bool(ok), "m_c": mc, "ms": ms,
                             "heads": heads, "parent": parent, "bottom_up": flag})
    return out
