"""Autotuner for the traversal kernels.

Picks, by measurement on the GPU it runs on:

* single-source BFS (bd_bfs): threads per CTA (256 / 512 / 1024), bitmap
  words a warp keeps in flight in a bottom-up step (1, 2, 4: 32-, 64- or
  128-bit of visited bits per warp step), the degree at which a top-down
  frontier vertex is split into chunks, the chunk size, and the arcs a lane
  scans alone before the warp takes over a long bottom-up list;
* batched BFS (bd_msbfs): threads per CTA, push split degree, chunk size,
  pull prefix and the push/pull alpha.

Search is coordinate descent over those axes (each axis swept with the
others held), repeated until nothing improves, scored by the harmonic mean
of per-root GTEPS over a fixed root set of an RMAT graph whose seed differs
from the benchmark graph's.  Results go to a JSON file that
beedrill_b200.tuned_options() reads:

    python -m beedrill_b200.autotune --scale 24 --seed 1024 --out beedrill_b200/tuning/b200.json
    python -m beedrill_b200.autotune --scale 20 --merge --out beedrill_b200/tuning/b200.json
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

import beedrill_b200 as bd

DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200.json")

SINGLE_SPACE = {
    "block_size": [256, 512, 1024],
    "bu_words": [1, 2, 4, 32],
    "bu_sparse_words": [4, 32],
    "large_degree": [16, 32, 64, 256, 1024],
    "chunk_edges": [128, 256, 512, 1024],
    "bu_prefix": [4, 8, 16, 32],
}
BATCHED_SPACE = {
    "block_size": [256, 512, 1024],
    "alpha": [1, 2, 4, 8, 16],
    "large_degree": [16, 32, 64, 128, 1024],
    "chunk_edges": [128, 256, 512, 1024],
    "pull_prefix": [8, 16, 32, 64],
    "heavy_degree": [1024, 4096, 16384],
    "heavy_chunk": [512, 2048, 8192],
}


def hmean(x):
    x = np.asarray(x, np.float64)
    return float(len(x) / np.sum(1.0 / x))


def score_single(graph, roots, params, repeats=2):
    try:
        bfs = bd.HybridBFS(graph, alg="beamer_hybrid", **params)
    except bd.BeedrillError:
        return 0.0  # a combination the library was not built with
    try:
        best = None
        for _ in range(repeats):
            ms, edges, _ = bfs.run_many(roots)
            g = hmean(edges / (ms * 1e-3) / 1e9)
            best = g if best is None else max(best, g)
        return best
    finally:
        bfs.close()


def score_batched(graph, roots, params, repeats=2):
    ms_bfs = bd.BatchedBFS(graph, len(roots), **params)
    try:
        best = None
        for _ in range(repeats):
            st = ms_bfs.run(roots)
            m_c, _ = ms_bfs.counts()
            g = hmean(m_c / (st.ms / len(roots) * 1e-3) / 1e9)
            best = g if best is None else max(best, g)
        return best
    finally:
        ms_bfs.close()


def coordinate_descent(space, start, score, log=None, rounds=3):
    cur = dict(start)
    cur_score = score(cur)
    table = [{"params": dict(cur), "gteps": cur_score}]
    for _ in range(rounds):
        improved = False
        for axis, values in space.items():
            for val in values:
                if val == cur[axis]:
                    continue
                cand = dict(cur)
                cand[axis] = val
                s = score(cand)
                table.append({"params": dict(cand), "gteps": s})
                if log:
                    log(f"{axis}={val}: {s:.2f} GTEPS (best {cur_score:.2f})")
                if s > cur_score * 1.01:
                    cur, cur_score, improved = cand, s, True
        if not improved:
            break
    return cur, cur_score, table


def tune(scale=24, roots=64, seed=1024, order=bd.ORDER_HUB, log=None):
    g = bd.Graph.rmat(scale, 16, seed=seed, order=order)
    rs = g.pick_roots(0, roots)
    start_single = {"block_size": 1024, "bu_words": 4, "bu_sparse_words": 32, "large_degree": 256,
                    "chunk_edges": 128, "bu_prefix": 8}
    single, s_score, s_table = coordinate_descent(
        SINGLE_SPACE, start_single, lambda p: score_single(g, rs, p), log)
    start_batched = {"block_size": 512, "alpha": 4, "large_degree": 32, "chunk_edges": 256,
                     "pull_prefix": 16, "heavy_degree": 4096, "heavy_chunk": 2048}
    batched, b_score, b_table = coordinate_descent(
        BATCHED_SPACE, start_batched, lambda p: score_batched(g, rs[:64], p), log)
    g.close()
    return {
        "graph": {"kind": "rmat", "scale": scale, "edge_factor": 16, "seed": seed, "roots": roots,
                  "adjacency_order": order},
        "single": single, "single_gteps": s_score,
        "batched": batched, "batched_gteps": b_score,
        "tables": {"single": s_table, "batched": b_table},
        "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description="tune the BFS kernels on this GPU")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--roots", type=int, default=64)
    ap.add_argument("--seed", type=int, default=1024,
                    help="graph seed (the benchmark's graph uses another)")
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--order", type=int, default=bd.ORDER_HUB)
    ap.add_argument("--merge", action="store_true",
                    help="add this scale's entry to an existing tuning file")
    args = ap.parse_args(argv)
    log = lambda s: print(f"[autotune] {s}", flush=True)  # noqa: E731
    res = tune(args.scale, args.roots, seed=args.seed, order=args.order, log=log)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    # One entry per tuned scale (handles use the one nearest their graph);
    # the top-level entry is the largest scale tuned so far.
    data = {}
    if args.merge and os.path.exists(args.out):
        with open(args.out) as f:
            data = json.load(f)
    keys = ("single", "batched", "single_gteps", "batched_gteps", "graph", "when")
    by_scale = data.get("by_scale", {})
    if not by_scale and "graph" in data:  # a file with one entry
        by_scale[str(data["graph"]["scale"])] = {k: data[k] for k in keys if k in data}
    by_scale[str(args.scale)] = {k: res[k] for k in keys}
    top = max(by_scale, key=int)
    data.update({k: v for k, v in res.items() if k != "tables"} if args.scale >= int(top) else {})
    data["by_scale"] = by_scale
    data.setdefault("tables", {})[str(args.scale)] = res["tables"]
    with open(args.out, "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")
    log(f"single {res['single']} {res['single_gteps']:.2f} GTEPS; "
        f"batched {res['batched']} {res['batched_gteps']:.2f} GTEPS -> {args.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
