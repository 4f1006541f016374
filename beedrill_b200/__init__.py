"""beedrill_b200 -- Python view of the B200 direction-optimizing BFS.

A thin ctypes layer over the C ABI in include/beedrill_b200.h
(beedrill_b200/lib/libbeedrill_b200.so).  Class and method names follow the
reference's hybrid_bfs class (hybrid_bfs.h:11-47) so code written against the
reference reads the same:

    g = Graph.from_el64("graph500-scale16")
    bfs = HybridBFS(g)                      # hybrid_bfs(graph&)
    bfs.clear()                             # hybrid_bfs::clear
    bfs.run_beamer(src, 15, 18)             # hybrid_bfs::run_beamer
    assert bfs.check(src)                   # hybrid_bfs::check
    m_c = bfs.count_num_traversed_edges()   # hybrid_bfs::count_num_traversed_edges

Every call runs on the GPU through the shared library; there is no CPU
fallback.  If the library is missing or no sm_100 device is present the
calls raise BeedrillError.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, byref, c_char_p, c_double, c_float, c_int, c_int32, c_int64,
                    c_uint32, c_uint64, c_void_p)

import numpy as np

__all__ = ["BeedrillError", "Graph", "HybridBFS", "BatchedBFS", "Components", "Step", "ALGORITHMS", "lib", "LIB_PATH",
           "tuned_options", "format_tree",
           "policy_forward", "policy_loss_grad", "policy_train"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbeedrill_b200.so")

BD_OK = 0
STATUS_NAMES = {
    0: "BD_OK", -1: "BD_ERR_INVALID", -2: "BD_ERR_IO", -3: "BD_ERR_FORMAT", -4: "BD_ERR_OOM",
    -5: "BD_ERR_CUDA", -6: "BD_ERR_TIMEOUT", -7: "BD_ERR_RANGE", -8: "BD_ERR_STATE",
    -9: "BD_ERR_NODEV", -10: "BD_ERR_LIMIT",
}
ORDER_INSERTION, ORDER_SORTED, ORDER_DEGREE, ORDER_HUB = 0, 1, 2, 3
ALG_BEAMER, ALG_TOP_DOWN, ALG_BOTTOM_UP, ALG_LEARNED = 0, 1, 2, 3

# The reference's --algorithm values (hybrid_bfs_main.cc:228-245) plus the
# directions and the learned policy of this implementation.
ALGORITHMS = {
    "beamer_hybrid": ALG_BEAMER,
    "remote_writes_hybrid": ALG_BEAMER,
    "migrating_threads": ALG_TOP_DOWN,
    "remote_writes": ALG_TOP_DOWN,
    "top_down": ALG_TOP_DOWN,
    "bottom_up": ALG_BOTTOM_UP,
    "learned": ALG_LEARNED,
}


class BeedrillError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = _lib_status_string(status)
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)} ({msg})")


class BfsOpts(Structure):
    _fields_ = [
        ("alg", c_int32), ("min_parent", c_int32), ("alpha", c_int64), ("beta", c_int64),
        ("block_size", c_int32), ("large_degree", c_int32), ("chunk_edges", c_int32),
        ("bu_prefix", c_int32), ("spin_limit", c_int64), ("test_extra_ctas", c_int32),
        ("bu_words", c_int32), ("bu_sparse_words", c_int32), ("reserved", c_int32),
    ]


class Step(Structure):
    _fields_ = [
        ("dir", c_int32), ("level", c_int32), ("frontier", c_int64), ("frontier_edges", c_int64),
        ("unexplored_edges", c_int64), ("found", c_int64), ("ns", c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MsBfsOpts(Structure):
    _fields_ = [
        ("alpha", c_int64), ("force_dir", c_int32), ("block_size", c_int32),
        ("large_degree", c_int32), ("chunk_edges", c_int32), ("pull_prefix", c_int32),
        ("use_graph", c_int32), ("spin_limit", c_int64), ("heavy_degree", c_int32),
        ("heavy_chunk", c_int32), ("materialize", c_int32), ("min_parent", c_int32),
    ]


class RunStats(Structure):
    _fields_ = [
        ("ms", c_double), ("num_steps", c_int64), ("reached", c_int64),
        ("traversed_edges", c_int64), ("top_down_steps", c_int64), ("bottom_up_steps", c_int64),
    ]


class ComponentsStats(Structure):
    _fields_ = [("num_components", c_int64), ("num_iters", c_int64), ("ms", c_double)]


_lib = None
TUNING_PATH = os.path.join(HERE, "tuning", "b200.json")


def tuned_options(kind: str, num_vertices: int | None = None) -> dict:
    """Launch parameters picked by beedrill_b200.autotune for `kind`
    ("single" or "batched"): those tuned at the scale nearest to
    log2(num_vertices) when the file holds several, else the default entry;
    {} when no tuning file exists."""
    if not os.path.exists(TUNING_PATH):
        return {}
    import json
    import math
    with open(TUNING_PATH) as f:
        d = json.load(f)
    by_scale = d.get("by_scale") or {}
    if num_vertices and by_scale:
        scale = math.log2(max(num_vertices, 2))
        key = min(by_scale, key=lambda k: (abs(int(k) - scale), -int(k)))
        return dict(by_scale[key].get(kind, {}))
    return dict(d.get(kind, {}))


def lib() -> ctypes.CDLL:
    """Load libbeedrill_b200.so (built by `make`); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `make` (or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    i64p, u32p, i32p = POINTER(c_int64), POINTER(c_uint32), POINTER(c_int32)
    f32p = POINTER(c_float)
    vpp = POINTER(c_void_p)
    sig = {
        "bd_status_string": (c_char_p, [c_int]),
        "bd_version": (c_char_p, []),
        "bd_set_device": (c_int, [c_int]),
        "bd_graph_from_el64": (c_int, [c_char_p, c_int32, vpp]),
        "bd_graph_from_edges": (c_int, [c_int64, c_int64, i64p, i64p, c_int32, vpp]),
        "bd_graph_from_csr": (c_int, [c_int64, c_int64, i64p, u32p, vpp]),
        "bd_graph_rmat": (c_int, [c_int32, c_int64, c_double, c_double, c_double, c_double,
                                  c_uint64, c_int32, vpp]),
        "bd_graph_rmat_stream": (c_int, [c_int32, c_int64, c_double, c_double, c_double, c_double,
                                         ctypes.c_uint32, c_int32, c_uint64, c_int32, vpp]),
        "bd_graph_concat": (c_int, [vpp, c_int64, vpp, i64p]),
        "bd_graph_grid": (c_int, [c_int64, c_int64, c_double, c_uint64, c_int32, vpp]),
        "bd_graph_info": (c_int, [c_void_p, i64p, i64p]),
        "bd_graph_copy_csr": (c_int, [c_void_p, i64p, u32p]),
        "bd_graph_copy_edges": (c_int, [c_void_p, i64p, i64p]),
        "bd_graph_write_el64": (c_int, [c_void_p, c_char_p]),
        "bd_graph_check": (c_int, [c_void_p, i32p]),
        "bd_graph_check_parents": (c_int, [c_void_p, c_int64, i64p, i32p, i64p]),
        "bd_graph_check_components": (c_int, [c_void_p, i64p, i32p, i64p]),
        "bd_components_create": (c_int, [c_void_p, vpp]),
        "bd_components_clear": (c_int, [c_void_p]),
        "bd_components_run": (c_int, [c_void_p, POINTER(ComponentsStats)]),
        "bd_components_get_labels": (c_int, [c_void_p, i64p]),
        "bd_components_get_sizes": (c_int, [c_void_p, i64p]),
        "bd_components_device_labels": (c_int, [c_void_p, vpp]),
        "bd_components_check": (c_int, [c_void_p, i32p]),
        "bd_components_destroy": (c_int, [c_void_p]),
        "bd_graph_pick_roots": (c_int, [c_void_p, c_uint64, c_int64, i64p]),
        "bd_graph_device_csr": (c_int, [c_void_p, vpp, vpp]),
        "bd_graph_destroy": (c_int, [c_void_p]),
        "bd_bfs_default_opts": (None, [POINTER(BfsOpts)]),
        "bd_bfs_create": (c_int, [c_void_p, POINTER(BfsOpts), vpp]),
        "bd_bfs_clear": (c_int, [c_void_p]),
        "bd_bfs_run": (c_int, [c_void_p, c_int64, POINTER(RunStats)]),
        "bd_bfs_run_beamer": (c_int, [c_void_p, c_int64, c_int64, c_int64, POINTER(RunStats)]),
        "bd_bfs_run_top_down": (c_int, [c_void_p, c_int64, POINTER(RunStats)]),
        "bd_bfs_run_bottom_up": (c_int, [c_void_p, c_int64, POINTER(RunStats)]),
        "bd_bfs_run_multi": (c_int, [c_void_p, i64p, c_int64, POINTER(RunStats)]),
        "bd_bfs_run_many": (c_int, [c_void_p, i64p, c_int64, POINTER(c_double), i64p, i64p,
                                    POINTER(c_double)]),
        "bd_bfs_run_many_into": (c_int, [c_void_p, i64p, c_int64, c_void_p, c_void_p,
                                         POINTER(c_double), i64p, i64p, POINTER(c_double)]),
        "bd_bfs_get_depths": (c_int, [c_void_p, i32p]),
        "bd_bfs_get_parents": (c_int, [c_void_p, i64p]),
        "bd_bfs_device_ptrs": (c_int, [c_void_p, vpp, vpp]),
        "bd_bfs_count_traversed_edges": (c_int, [c_void_p, i64p]),
        "bd_bfs_check": (c_int, [c_void_p, c_int64, i32p]),
        "bd_bfs_get_steps": (c_int, [c_void_p, POINTER(Step), c_int64, i64p]),
        "bd_bfs_destroy": (c_int, [c_void_p]),
        "bd_bfs_set_policy": (c_int, [c_void_p, f32p, f32p, f32p, f32p, f32p, c_float]),
        "bd_msbfs_default_opts": (None, [POINTER(MsBfsOpts)]),
        "bd_msbfs_create": (c_int, [c_void_p, c_int32, POINTER(MsBfsOpts), vpp]),
        "bd_msbfs_run": (c_int, [c_void_p, i64p, c_int32, POINTER(RunStats)]),
        "bd_msbfs_get_depths": (c_int, [c_void_p, c_int32, i32p]),
        "bd_msbfs_get_parents": (c_int, [c_void_p, c_int32, i64p]),
        "bd_msbfs_count_traversed_edges": (c_int, [c_void_p, c_int32, i64p, i64p]),
        "bd_msbfs_get_steps": (c_int, [c_void_p, POINTER(Step), c_int64, i64p]),
        "bd_msbfs_check": (c_int, [c_void_p, c_int32, POINTER(c_int32)]),
        "bd_msbfs_device_results": (c_int, [c_void_p, c_int32, vpp, vpp]),
        "bd_msbfs_destroy": (c_int, [c_void_p]),
        "bd_msbfs_set_policy": (c_int, [c_void_p, f32p, f32p, f32p, f32p, f32p, c_float]),
        "bd_policy_forward": (c_int, [f32p, f32p, c_int64, f32p]),
        "bd_policy_loss_grad": (c_int, [f32p, f32p, i32p, f32p, c_int64, f32p, f32p]),
        "bd_policy_train": (c_int, [f32p, f32p, i32p, f32p, c_int64, c_int32, c_float, c_float,
                                    f32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _lib_status_string(status: int) -> str:
    try:
        return lib().bd_status_string(status).decode()
    except Exception:  # library not loadable: the caller's message says why
        return "?"


def _check(status: int, what: str) -> None:
    if status != BD_OK:
        raise BeedrillError(status, what)


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(POINTER(ct))


def _set_policy(fn, handle, params, mean, inv_std, margin, lo, hi) -> None:
    if params is None:
        _check(fn(handle, None, None, None, None, None, 0.0), "set_policy")
        return
    lo_p = hi_p = None
    if lo is not None:
        lo_a = np.ascontiguousarray(lo, np.float32)
        hi_a = np.ascontiguousarray(hi, np.float32)
        lo_p, hi_p = _ptr(lo_a, c_float), _ptr(hi_a, c_float)
    p = np.ascontiguousarray(params, np.float32)
    mu = np.ascontiguousarray(mean, np.float32)
    isd = np.ascontiguousarray(inv_std, np.float32)
    if p.size != 1410 or mu.size != 8 or isd.size != 8:
        raise ValueError("policy shapes: 1410 params, 8 means, 8 inverse std devs")
    _check(fn(handle, _ptr(p, c_float), _ptr(mu, c_float), _ptr(isd, c_float), lo_p, hi_p,
              margin), "set_policy")


class Graph:
    """A graph resident in HBM (CSR: int64 offsets, uint32 neighbour ids)."""

    def __init__(self, handle: c_void_p):
        self._h = handle

    # -- construction -------------------------------------------------------
    @classmethod
    def from_el64(cls, path: str, order: int = ORDER_INSERTION) -> "Graph":
        h = c_void_p()
        _check(lib().bd_graph_from_el64(os.fsencode(path), order, byref(h)), f"load {path}")
        return cls(h)

    @classmethod
    def from_edges(cls, num_vertices: int, src, dst, order: int = ORDER_INSERTION) -> "Graph":
        src = np.ascontiguousarray(src, np.int64)
        dst = np.ascontiguousarray(dst, np.int64)
        if src.shape != dst.shape:
            raise ValueError("src and dst differ in length")
        h = c_void_p()
        _check(lib().bd_graph_from_edges(num_vertices, len(src), _ptr(src, c_int64),
                                         _ptr(dst, c_int64), order, byref(h)), "from_edges")
        return cls(h)

    @classmethod
    def from_csr(cls, offsets, adjacency) -> "Graph":
        off = np.ascontiguousarray(offsets, np.int64)
        adj = np.ascontiguousarray(adjacency, np.uint32)
        h = c_void_p()
        _check(lib().bd_graph_from_csr(len(off) - 1, len(adj), _ptr(off, c_int64),
                                       _ptr(adj, c_uint32), byref(h)), "from_csr")
        return cls(h)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, d: float = 0.05, seed: int = 0,
             order: int = ORDER_INSERTION) -> "Graph":
        h = c_void_p()
        _check(lib().bd_graph_rmat(scale, edge_factor, a, b, c, d, seed, order, byref(h)),
               f"rmat(scale={scale})")
        return cls(h)

    @classmethod
    def rmat_stream(cls, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
                    c: float = 0.19, d: float = 0.05, stream_seed: int = 0, permute: bool = False,
                    permute_seed: int = 0, order: int = ORDER_INSERTION) -> "Graph":
        """RMAT edges drawn exactly as the reference's generator draws them
        (its sitmo stream, rmat_generator.h:70-193), flipped, sorted and
        deduplicated; permute=False keeps the generator's ids and the sorted
        order, permute=True applies the seeded relabel and shuffle of rmat()."""
        h = c_void_p()
        _check(lib().bd_graph_rmat_stream(scale, edge_factor, a, b, c, d, stream_seed,
                                          int(bool(permute)), permute_seed, order, byref(h)),
               f"rmat_stream(scale={scale})")
        return cls(h)

    @classmethod
    def grid(cls, rows: int, cols: int, delete_frac: float = 0.01, seed: int = 0,
             order: int = ORDER_INSERTION) -> "Graph":
        h = c_void_p()
        _check(lib().bd_graph_grid(rows, cols, delete_frac, seed, order, byref(h)),
               f"grid({rows}x{cols})")
        return cls(h)

    @classmethod
    def concat(cls, graphs) -> tuple["Graph", np.ndarray]:
        arr = (c_void_p * len(graphs))(*[g._h.value for g in graphs])
        base = np.zeros(len(graphs) + 1, np.int64)
        h = c_void_p()
        _check(lib().bd_graph_concat(ctypes.cast(arr, POINTER(c_void_p)), len(graphs), byref(h),
                                     _ptr(base, c_int64)), "concat")
        return cls(h), base

    # -- queries ------------------------------------------------------------
    def num_vertices(self) -> int:
        n = c_int64()
        _check(lib().bd_graph_info(self._h, byref(n), None), "info")
        return n.value

    def num_edges(self) -> int:
        m = c_int64()
        _check(lib().bd_graph_info(self._h, None, byref(m)), "info")
        return m.value

    def csr(self):
        n = self.num_vertices()
        off = np.empty(n + 1, np.int64)
        lib().bd_graph_copy_csr(self._h, _ptr(off, c_int64), None)
        adj = np.empty(int(off[-1]), np.uint32)
        _check(lib().bd_graph_copy_csr(self._h, _ptr(off, c_int64), _ptr(adj, c_uint32)), "csr")
        return off, adj

    def edges(self):
        m = self.num_edges()
        src = np.empty(m, np.int64)
        dst = np.empty(m, np.int64)
        _check(lib().bd_graph_copy_edges(self._h, _ptr(src, c_int64), _ptr(dst, c_int64)), "edges")
        return src, dst

    def write_el64(self, path: str) -> None:
        _check(lib().bd_graph_write_el64(self._h, os.fsencode(path)), f"write {path}")

    def check(self) -> bool:
        ok = c_int32()
        _check(lib().bd_graph_check(self._h, byref(ok)), "graph check")
        return bool(ok.value)

    # hybrid_bfs::check (hybrid_bfs.cc:281-379) of any parent array, on the device
    def check_parents(self, source: int, parent: np.ndarray) -> tuple[bool, int]:
        """(passes, lowest failing vertex or -1) for a parent array of n
        entries in the reference's encoding (source -> source, unreached
        vertices negative)."""
        par = np.ascontiguousarray(parent, dtype=np.int64)
        n = self.num_vertices()
        if par.shape != (n,):
            raise ValueError(f"parent array of shape {par.shape} for {n} vertices")
        ok, bad = c_int32(), c_int64()
        _check(lib().bd_graph_check_parents(self._h, source, _ptr(par, c_int64), byref(ok),
                                            byref(bad)), "check_parents")
        return bool(ok.value), int(bad.value)

    # components::check (components.cc:155-200) of any labelling, on the device
    def check_components(self, labels: np.ndarray) -> tuple[bool, int]:
        """(passes, lowest vertex breaking the rule or -1) for int64 labels of
        every vertex."""
        lab = np.ascontiguousarray(labels, dtype=np.int64)
        n = self.num_vertices()
        if lab.shape != (n,):
            raise ValueError(f"label array of shape {lab.shape} for {n} vertices")
        ok, bad = c_int32(), c_int64()
        _check(lib().bd_graph_check_components(self._h, _ptr(lab, c_int64), byref(ok), byref(bad)),
               "check_components")
        return bool(ok.value), int(bad.value)

    def pick_roots(self, seed: int, k: int) -> np.ndarray:
        roots = np.empty(k, np.int64)
        _check(lib().bd_graph_pick_roots(self._h, seed, k, _ptr(roots, c_int64)), "pick_roots")
        return roots

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().bd_graph_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HybridBFS:
    """Mirror of the reference's hybrid_bfs class on the GPU."""

    def __init__(self, graph: Graph, alg: str = "beamer_hybrid", alpha: int = 15,
                 beta: int = 18, min_parent: bool = False, block_size: int = 0,
                 large_degree: int = 0, chunk_edges: int = 0, bu_prefix: int = 0,
                 spin_limit: int = 0, test_extra_ctas: int = 0, bu_words: int = 0,
                 bu_sparse_words: int = 0, tuned: bool = True):
        if alg not in ALGORITHMS:
            raise ValueError(f"Algorithm '{alg}' not implemented!")
        if tuned:
            t = tuned_options("single", graph.num_vertices())
            block_size = block_size or t.get("block_size", 0)
            large_degree = large_degree or t.get("large_degree", 0)
            chunk_edges = chunk_edges or t.get("chunk_edges", 0)
            bu_prefix = bu_prefix or t.get("bu_prefix", 0)
            bu_words = bu_words or t.get("bu_words", 0)
            bu_sparse_words = bu_sparse_words or t.get("bu_sparse_words", 0)
        self.graph = graph  # keeps the graph alive
        o = BfsOpts()
        lib().bd_bfs_default_opts(byref(o))
        o.alg = ALGORITHMS[alg]
        o.alpha, o.beta = alpha, beta
        o.min_parent = int(bool(min_parent))
        o.block_size, o.large_degree, o.chunk_edges = block_size, large_degree, chunk_edges
        o.bu_prefix, o.spin_limit, o.test_extra_ctas = bu_prefix, spin_limit, test_extra_ctas
        o.bu_words = bu_words
        o.bu_sparse_words = bu_sparse_words
        self.alg = alg
        self.alpha, self.beta = alpha, beta
        self._h = c_void_p()
        _check(lib().bd_bfs_create(graph._h, byref(o), byref(self._h)), "hybrid_bfs")
        self.last_stats = RunStats()

    # hybrid_bfs::clear (hybrid_bfs.cc:433-443)
    def clear(self) -> None:
        _check(lib().bd_bfs_clear(self._h), "clear")

    def run(self, source: int) -> RunStats:
        """Run with the policy chosen at construction (the --alg dispatch of
        hybrid_bfs_main.cc:268-281)."""
        _check(lib().bd_bfs_run(self._h, source, byref(self.last_stats)), "run")
        return self.last_stats

    # hybrid_bfs::run_beamer (hybrid_bfs.cc:152-191)
    def run_beamer(self, source: int, alpha: int = 15, beta: int = 18) -> RunStats:
        _check(lib().bd_bfs_run_beamer(self._h, source, alpha, beta, byref(self.last_stats)),
               "run_beamer")
        return self.last_stats

    # hybrid_bfs::run_with_remote_writes_hybrid (hybrid_bfs.cc:243-277): the
    # same Beamer switch; its top-down flavour is an Emu artefact.
    def run_with_remote_writes_hybrid(self, source: int, alpha: int = 15, beta: int = 18):
        return self.run_beamer(source, alpha, beta)

    def run_top_down(self, source: int) -> RunStats:
        _check(lib().bd_bfs_run_top_down(self._h, source, byref(self.last_stats)), "top_down")
        return self.last_stats

    # hybrid_bfs::run_with_migrating_threads / run_with_remote_writes
    # (hybrid_bfs.cc:196-235): top-down only.
    run_with_migrating_threads = run_top_down
    run_with_remote_writes = run_top_down

    def run_bottom_up(self, source: int) -> RunStats:
        _check(lib().bd_bfs_run_bottom_up(self._h, source, byref(self.last_stats)), "bottom_up")
        return self.last_stats

    def run_multi(self, sources) -> RunStats:
        src = np.ascontiguousarray(sources, np.int64)
        _check(lib().bd_bfs_run_multi(self._h, _ptr(src, c_int64), len(src),
                                      byref(self.last_stats)), "run_multi")
        return self.last_stats

    def run_many(self, sources, with_reached: bool = False):
        """k BFSs back to back (clear() before each); returns per-root ms,
        per-root m_c, [per-root n_c,] and the device time of the whole call
        including the root upload and the result download."""
        src = np.ascontiguousarray(sources, np.int64)
        ms = np.empty(len(src), np.float64)
        edges = np.empty(len(src), np.int64)
        reached = np.empty(len(src), np.int64)
        e2e = c_double()
        _check(lib().bd_bfs_run_many(self._h, _ptr(src, c_int64), len(src), _ptr(ms, c_double),
                                     _ptr(edges, c_int64), _ptr(reached, c_int64), byref(e2e)),
               "run_many")
        if with_reached:
            return ms, edges, reached, e2e.value
        return ms, edges, e2e.value

    def run_many_into(self, sources, d_depth: int, d_parent: int):
        """run_many, and root i's depths and parents (caller ids, the
        reference's encoding) written inside its timed region to the device
        arrays at d_depth + i*n (int32) and d_parent + i*n (int64), each of
        len(sources) x n entries.  Returns per-root ms, m_c, n_c and the
        device time of the whole call."""
        src = np.ascontiguousarray(sources, np.int64)
        ms = np.empty(len(src), np.float64)
        edges = np.empty(len(src), np.int64)
        reached = np.empty(len(src), np.int64)
        e2e = c_double()
        _check(lib().bd_bfs_run_many_into(self._h, _ptr(src, c_int64), len(src), c_void_p(d_depth),
                                          c_void_p(d_parent), _ptr(ms, c_double),
                                          _ptr(edges, c_int64), _ptr(reached, c_int64), byref(e2e)),
               "run_many_into")
        return ms, edges, reached, e2e.value

    # hybrid_bfs::check (hybrid_bfs.cc:281-379)
    def check(self, source: int) -> bool:
        ok = c_int32()
        _check(lib().bd_bfs_check(self._h, source, byref(ok)), "check")
        return bool(ok.value)

    # hybrid_bfs::count_num_traversed_edges (hybrid_bfs.cc:401-414)
    def count_num_traversed_edges(self) -> int:
        out = c_int64()
        _check(lib().bd_bfs_count_traversed_edges(self._h, byref(out)), "count")
        return out.value

    def depths(self) -> np.ndarray:
        d = np.empty(self.graph.num_vertices(), np.int32)
        _check(lib().bd_bfs_get_depths(self._h, _ptr(d, c_int32)), "depths")
        return d

    def parents(self) -> np.ndarray:
        p = np.empty(self.graph.num_vertices(), np.int64)
        _check(lib().bd_bfs_get_parents(self._h, _ptr(p, c_int64)), "parents")
        return p

    def steps(self) -> list[dict]:
        count = c_int64()
        _check(lib().bd_bfs_get_steps(self._h, None, 0, byref(count)), "steps")
        buf = (Step * max(count.value, 1))()
        _check(lib().bd_bfs_get_steps(self._h, buf, count.value, byref(count)), "steps")
        return [buf[i].as_dict() for i in range(count.value)]

    def directions(self) -> str:
        return "".join("B" if s["dir"] else "T" for s in self.steps())

    # hybrid_bfs::print_tree (hybrid_bfs.cc:381-399)
    def print_tree(self) -> None:
        print(format_tree(self.parents()), end="")

    def set_policy(self, params, mean, inv_std, margin: float = 0.0, lo=None, hi=None) -> None:
        """Install the learned direction policy used by alg="learned"
        (params=None removes it; Beamer then decides).  lo / hi bound the raw
        features the policy is trusted on (None: no bound)."""
        _set_policy(lib().bd_bfs_set_policy, self._h, params, mean, inv_std, margin, lo, hi)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().bd_bfs_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchedBFS:
    """Many BFSs per pass over the graph: groups of up to 64 roots, one bit
    lane per root, all groups of a call replayed as one captured CUDA graph.
    Per root the results equal HybridBFS's (depths, parents, m_c)."""

    def __init__(self, graph: Graph, max_roots: int = 64, alpha: int = 0, force_dir: int = -1,
                 use_graph: bool = True, block_size: int = 0, large_degree: int = 0,
                 chunk_edges: int = 0, pull_prefix: int = 0, spin_limit: int = 0,
                 heavy_degree: int = 0, heavy_chunk: int = 0, tuned: bool = True,
                 materialize: bool = False, min_parent: bool = False):
        if tuned:
            t = tuned_options("batched", graph.num_vertices())
            alpha = alpha or t.get("alpha", 0)
            block_size = block_size or t.get("block_size", 0)
            large_degree = large_degree or t.get("large_degree", 0)
            chunk_edges = chunk_edges or t.get("chunk_edges", 0)
            pull_prefix = pull_prefix or t.get("pull_prefix", 0)
            heavy_degree = heavy_degree or t.get("heavy_degree", 0)
            heavy_chunk = heavy_chunk or t.get("heavy_chunk", 0)
        self.graph = graph
        o = MsBfsOpts()
        lib().bd_msbfs_default_opts(byref(o))
        if alpha:
            o.alpha = alpha
        o.force_dir = force_dir
        o.use_graph = int(bool(use_graph))
        o.block_size, o.large_degree, o.chunk_edges = block_size, large_degree, chunk_edges
        o.pull_prefix, o.spin_limit = pull_prefix, spin_limit
        o.heavy_degree, o.heavy_chunk = heavy_degree, heavy_chunk
        o.materialize, o.min_parent = int(bool(materialize)), int(bool(min_parent))
        self.max_roots = max_roots
        self._h = c_void_p()
        _check(lib().bd_msbfs_create(graph._h, max_roots, byref(o), byref(self._h)), "msbfs")
        self.last_stats = RunStats()

    def run(self, sources) -> RunStats:
        src = np.ascontiguousarray(sources, np.int64)
        _check(lib().bd_msbfs_run(self._h, _ptr(src, c_int64), len(src), byref(self.last_stats)),
               "msbfs run")
        self.count = len(src)
        return self.last_stats

    def depths(self, i: int) -> np.ndarray:
        d = np.empty(self.graph.num_vertices(), np.int32)
        _check(lib().bd_msbfs_get_depths(self._h, i, _ptr(d, c_int32)), "msbfs depths")
        return d

    def parents(self, i: int) -> np.ndarray:
        p = np.empty(self.graph.num_vertices(), np.int64)
        _check(lib().bd_msbfs_get_parents(self._h, i, _ptr(p, c_int64)), "msbfs parents")
        return p

    def parents_to(self, i: int, host_addr: int) -> None:
        """Root i's parents into caller-owned host memory at host_addr (n
        int64 entries; pinned memory copies fastest)."""
        _check(lib().bd_msbfs_get_parents(self._h, i, ctypes.cast(host_addr, POINTER(c_int64))),
               "msbfs parents")

    def count_num_traversed_edges(self, i: int) -> int:
        e = c_int64()
        _check(lib().bd_msbfs_count_traversed_edges(self._h, i, byref(e), None), "msbfs count")
        return e.value

    def reached(self, i: int) -> int:
        r = c_int64()
        _check(lib().bd_msbfs_count_traversed_edges(self._h, i, None, byref(r)), "msbfs count")
        return r.value

    # hybrid_bfs::check (hybrid_bfs.cc:281-379) of root i's parents
    def check(self, i: int) -> bool:
        ok = c_int32()
        _check(lib().bd_msbfs_check(self._h, i, byref(ok)), "msbfs check")
        return bool(ok.value)

    def device_results(self, i: int) -> tuple[int, int]:
        """Device addresses of root i's materialized depths (int32[n]) and
        parents (int64[n]); the handle must be made with materialize=True."""
        d, p = c_void_p(), c_void_p()
        _check(lib().bd_msbfs_device_results(self._h, i, byref(d), byref(p)), "msbfs results")
        return d.value, p.value

    def counts(self):
        """(m_c, n_c) arrays over the roots of the last run."""
        m = np.empty(self.count, np.int64)
        n = np.empty(self.count, np.int64)
        for i in range(self.count):
            e, r = c_int64(), c_int64()
            _check(lib().bd_msbfs_count_traversed_edges(self._h, i, byref(e), byref(r)), "count")
            m[i], n[i] = e.value, r.value
        return m, n

    def steps(self) -> list[dict]:
        count = c_int64()
        _check(lib().bd_msbfs_get_steps(self._h, None, 0, byref(count)), "steps")
        buf = (Step * max(count.value, 1))()
        _check(lib().bd_msbfs_get_steps(self._h, buf, count.value, byref(count)), "steps")
        return [buf[i].as_dict() for i in range(count.value)]

    def directions(self) -> str:
        return "".join("B" if s["dir"] else "T" for s in self.steps())

    def set_policy(self, params, mean, inv_std, margin: float = 0.0, lo=None, hi=None) -> None:
        """Install the learned push/pull policy (params=None: the rule)."""
        _set_policy(lib().bd_msbfs_set_policy, self._h, params, mean, inv_std, margin, lo, hi)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().bd_msbfs_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def format_tree(parent) -> str:
    """hybrid_bfs::print_tree's text (hybrid_bfs.cc:381-399) for a parent
    array in the reference's encoding: each vertex with a parent and its
    ancestors up to the root, "%4li <- %4li <- ..." per line.  A chain that
    meets a negative or out-of-range entry stops there (the reference would
    index with it); a chain that climbs n times without reaching a root is
    a cycle (the reference would loop forever) and its line ends with
    " <- (cycle)"."""
    n = len(parent)
    lines = []
    for v in range(n):
        p = int(parent[v])
        if p < 0:
            continue
        parts = [f"{v:4d}"]
        for _ in range(n + 1):
            parts.append(f" <- {p:4d}")
            if p < 0 or p >= n or p == parent[p]:
                break
            p = int(parent[p])
        else:
            parts.append(" <- (cycle)")
        lines.append("".join(parts) + "\n")
    return "".join(lines)


class Components:
    """Connected components (components.h): every vertex labelled with the
    smallest vertex id of its component, as the reference's run() leaves
    component_; sizes per label as component_size_."""

    def __init__(self, graph: Graph):
        self.graph = graph
        self._h = c_void_p()
        self.last_stats = ComponentsStats()
        _check(lib().bd_components_create(graph._h, byref(self._h)), "components")

    def clear(self) -> None:
        _check(lib().bd_components_clear(self._h), "clear")

    def run(self) -> ComponentsStats:
        _check(lib().bd_components_run(self._h, byref(self.last_stats)), "components run")
        return self.last_stats

    def labels(self) -> np.ndarray:
        out = np.empty(self.graph.num_vertices(), np.int64)
        _check(lib().bd_components_get_labels(self._h, _ptr(out, c_int64)), "labels")
        return out

    def sizes(self) -> np.ndarray:
        out = np.empty(self.graph.num_vertices(), np.int64)
        _check(lib().bd_components_get_sizes(self._h, _ptr(out, c_int64)), "sizes")
        return out

    def check(self) -> bool:
        ok = c_int32()
        _check(lib().bd_components_check(self._h, byref(ok)), "components check")
        return bool(ok.value)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().bd_components_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Learned-policy kernels (beedrill_b200/csrc/bd_policy.cu)
# ---------------------------------------------------------------------------

def policy_forward(params, x) -> np.ndarray:
    """Device forward pass: logits (n, 2) of standardised features (n, 8)."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 8)
    out = np.empty((len(x), 2), np.float32)
    _check(lib().bd_policy_forward(_ptr(p, c_float), _ptr(x, c_float), len(x), _ptr(out, c_float)),
           "policy_forward")
    return out


def policy_loss_grad(params, x, label, weight):
    """Device weighted cross-entropy and its gradient (1410 floats)."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 8)
    y = np.ascontiguousarray(label, np.int32)
    w = np.ascontiguousarray(weight, np.float32)
    loss = c_float()
    grad = np.empty(1410, np.float32)
    _check(lib().bd_policy_loss_grad(_ptr(p, c_float), _ptr(x, c_float), _ptr(y, c_int32),
                                     _ptr(w, c_float), len(y), byref(loss), _ptr(grad, c_float)),
           "policy_loss_grad")
    return float(loss.value), grad


def policy_train(params, x, label, weight, epochs: int, lr: float, weight_decay: float = 0.0):
    """Full-batch Adam on the device; updates params in place and returns
    the loss history."""
    if not (isinstance(params, np.ndarray) and params.dtype == np.float32 and params.flags.c_contiguous):
        raise TypeError("params must be a C-contiguous float32 array (updated in place)")
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 8)
    y = np.ascontiguousarray(label, np.int32)
    w = np.ascontiguousarray(weight, np.float32)
    hist = np.empty(epochs, np.float32)
    _check(lib().bd_policy_train(_ptr(params, c_float), _ptr(x, c_float), _ptr(y, c_int32),
                                 _ptr(w, c_float), len(y), epochs, lr, weight_decay,
                                 _ptr(hist, c_float)), "policy_train")
    return hist
