"""Regenerates the golden fixtures in this directory from the reference itself.

Run from the repository root, on a machine where the reference sources are
present (they are compiled by oracle/Makefile into oracle/_ref/):

    python tests/golden/make_golden.py

What it writes, and where each number comes from:

* graph500-scale10.el64 -- written by the reference's own generator
  (oracle/_ref/rmat_dataset_dump graph500-scale10, one OpenMP thread: its
  output depends on the thread count).  Pins the el64 format end to end.
* ref_scale10.npz -- oracle/_ref/ref_dump on that file: the reference's CSR
  (insertion order), the 8 roots of lcg(0), and for each of the four
  reference algorithms the parent array, bottom-up flags, queue level
  boundaries, m_c and the reference's own check() verdict.
* ref_gen12.npz -- the same reference run on the project's seeded generator
  output at scale 12 (seed 12), so parents/levels can be compared at full
  detail on a graph the device generator must reproduce byte for byte.
* ref_components.npz -- oracle/_ref/components (the reference's
  connected-components CLI) with --check_results --dump_results on five
  graphs: graph500-scale10.el64, a sparse project-generated RMAT graph
  (scale 12, edge factor 2, seed 5), a 48 x 48 grid with 30 % of its
  edges deleted (seed 3), and two graphs whose last component is one run
  of vertices ending at n-1 (a scale-10 RMAT graph plus one isolated
  vertex; graph500-scale10 plus a 3-vertex path), where the reference's
  dump ends without a newline.  Per graph: the CSR, the labels parsed from
  the reference's dump, its component count, iteration count and check()
  verdict, the raw text of its --dump_results; and a set of planted labellings (a vertex relabelled, two
  components merged under one label, arbitrary distinct labels, two labels
  swapped, one label for all, an isolated vertex given a used label) with
  the verdict of the reference's own components::check on each
  (oracle/_ref/ref_components_check).  `python tests/golden/make_golden.py
  --components` rewrites only this file.
* ref_gen.npz -- oracle/_ref/ref_gen_edges (the reference's own RMAT
  generator, rmat_generator.h, run serially, plus the flip / sort / dedup of
  rmat_dataset_dump.cc:48-53) on six cases (scales 8-14, several A-D,
  seeds 0-12345, one where most edges are self loops): edge counts and the
  sha256 of the generated list (after the self-loop re-roll) and of the
  deduplicated sorted list; the scale-10 case keeps both lists.
  `python tests/golden/make_golden.py --generator` rewrites only this file.
* ref_check.npz -- hybrid_bfs::check run by the reference itself
  (oracle/_ref/ref_check) on parent arrays of graph500-scale10.el64: the
  reference's beamer_hybrid tree of each of its 8 roots, and for each root
  the same tree with planted mistakes (a parent that is no neighbour, a
  neighbour on the same level or one level down, a reached vertex without a
  parent, a vertex its own parent, parent ids past n, an unreached vertex
  with a parent, a source that is not its own parent, two mistakes at
  once).  Per record: source, parents, the reference's verdict and the
  vertex its LOG lines name (where its loop stops; -1 on PASS); and the
  text of the reference's print_tree() for each of the 8 trees.
  `python tests/golden/make_golden.py --check` rewrites only this file.
* golden.json -- hashes and per-root summaries: sha256 of the generator's
  el64 files (scale 12 and 16), and for scale 16 (seed 16, 8 roots of lcg(0))
  the reference's m_c, per-step discovered counts, per-level directions and
  the sha256 of the depth array derived from the reference's parent tree.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ALGS = ["beamer_hybrid", "migrating_threads", "remote_writes", "remote_writes_hybrid"]


def sha256_file(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def ref_dump(graph, out, alg="beamer_hybrid", roots=8, dump_graph=False):
    cmd = [os.path.join(O.REF_DIR, "ref_dump"), "--graph_filename", graph, "--out", out,
           "--algorithm", alg, "--num_trials", str(roots)]
    if dump_graph:
        cmd.append("--dump_graph")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    return O.read_ref_dump(out)


def level_dirs(parent, flags, root):
    """Direction that produced each non-empty level, from the reference's
    new_parent_ marks (>= 0 exactly for bottom-up discoveries)."""
    depth = O.depth_from_parents(parent, root)
    out = []
    for lv in range(1, int(depth.max()) + 1):
        f = flags[depth == lv]
        assert f.min() == f.max(), "mixed directions within one level"
        out.append("B" if f[0] else "T")
    return "".join(out), depth


def pack_roots(d):
    k = len(d["roots"])
    n = d["n"]
    heads_len = max(len(r["heads"]) for r in d["roots"])
    heads = np.full((k, heads_len), -1, np.int64)
    for i, r in enumerate(d["roots"]):
        heads[i, : len(r["heads"])] = r["heads"]
    return {
        "roots": np.array([r["root"] for r in d["roots"]], np.int64),
        "parent": np.stack([r["parent"] for r in d["roots"]]).reshape(k, n),
        "bottom_up": np.stack([r["bottom_up"] for r in d["roots"]]).reshape(k, n),
        "heads": heads,
        "m_c": np.array([r["m_c"] for r in d["roots"]], np.int64),
        "check": np.array([r["check"] for r in d["roots"]], np.bool_),
    }


def ref_components(el64, n):
    """Labels, component count, iteration count and check() verdict printed
    by the reference's components CLI (components_main.cc:164-196)."""
    out = subprocess.run([os.path.join(O.REF_DIR, "components"), "--graph_filename", el64,
                          "--check_results", "--dump_results"], check=True,
                         stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True).stdout
    labels = np.full(n, -1, np.int64)
    count = iters = None
    passed = None
    for line in out.splitlines():
        m = re.match(r"Found (\d+) components in (\d+) iterations", line)
        if m:
            count, iters = int(m.group(1)), int(m.group(2))
        if line.startswith("Checking results..."):
            passed = line.endswith("PASS")
        m = re.match(r"Component (\d+): (.*)$", line)
        if m:
            c = int(m.group(1))
            for part in m.group(2).split(", "):
                lo, _, hi = part.partition("-")
                labels[int(lo): int(hi or lo) + 1] = c
    assert (labels >= 0).all() and count is not None and passed is not None
    # the dump is the last thing the CLI prints, right after the check's
    # verdict; kept byte for byte (a line may lack its newline)
    verdict = "Checking results...PASS\n" if passed else "Checking results...FAIL\n"
    dump = out[out.rindex(verdict) + len(verdict):]
    return labels, count, iters, passed, dump


def planted_parents(off, adj, root, good, rng):
    """The reference tree of one root and copies with mistakes planted."""
    n = len(off) - 1
    depth = O.bfs_depth(off, adj, root)
    reached = np.flatnonzero(depth > 1)
    v = int(rng.choice(reached))
    nbrs = adj[off[v]:off[v + 1]].astype(np.int64)
    out = [good.copy()]

    def plant(changes):
        bad = good.copy()
        for u, p in changes:
            bad[u] = p
        out.append(bad)

    non = np.setdiff1d(np.arange(n), nbrs)
    plant([(v, int(non[non != v][0]))])
    for d in (depth[v], depth[v] + 1):
        cand = nbrs[depth[nbrs] == d]
        if len(cand):
            plant([(v, int(cand[0]))])
    plant([(v, -1)])
    plant([(v, v)])
    plant([(v, n + 5)])
    unreached = np.flatnonzero(depth < 0)
    if len(unreached):
        plant([(int(unreached[-1]), root)])
    plant([(root, int(adj[off[root]]))])
    w = int(rng.choice(reached[reached != v]))
    plant([(v, -1), (w, -1)])
    return out


def write_parents(path, sources, parents):
    with open(path, "wb") as f:
        f.write(np.array([len(sources), parents.shape[1]], np.int64).tobytes())
        for s, p in zip(sources, parents):
            f.write(np.int64(s).tobytes())
            f.write(np.ascontiguousarray(p, np.int64).tobytes())


def ref_print_tree(el64, sources, parents, tmp):
    """The text of the reference's own print_tree() for each parent array."""
    path = os.path.join(tmp, "trees.bin")
    write_parents(path, sources, parents)
    out = subprocess.run([os.path.join(O.REF_DIR, "ref_check"), "--graph_filename", el64,
                          "--parents", path, "--print_tree"], check=True, stdout=subprocess.PIPE,
                         stderr=subprocess.DEVNULL, text=True).stdout
    texts = []
    for i in range(len(sources)):
        head, tail = f"BEGIN {i}\n", f"END {i}\n"
        texts.append(out[out.index(head) + len(head): out.index(tail)])
    return texts


def ref_check(el64, sources, parents, tmp):
    """Verdict and stopping vertex of the reference's own check() per record."""
    path = os.path.join(tmp, "parents.bin")
    write_parents(path, sources, parents)
    out = subprocess.run([os.path.join(O.REF_DIR, "ref_check"), "--graph_filename", el64,
                          "--parents", path], check=True, stdout=subprocess.PIPE,
                         stderr=subprocess.DEVNULL, text=True).stdout
    verdict, stop = [], []
    for i, block in enumerate(out.split("BEGIN ")[1:]):
        m = re.search(r"VERDICT (\d+) (\d)", block)
        assert m and int(m.group(1)) == i
        ok = int(m.group(2))
        where = -1
        if not ok:
            if "Source wrong" in block:
                where = int(sources[i])
            else:
                e = re.search(r"Couldn't find edge from -?\d+ to (\d+)", block)
                r = re.search(r"Reachability mismatch: depth\[(\d+)\]", block)
                where = int((e or r).group(1))
        verdict.append(ok)
        stop.append(where)
    assert len(verdict) == len(sources)
    return np.array(verdict, np.int64), np.array(stop, np.int64)


def check_fixture(tmp):
    el10 = os.path.join(HERE, "graph500-scale10.el64")
    ref = np.load(os.path.join(HERE, "ref_scale10.npz"))
    off, adj = ref["offsets"], ref["adj"].astype(np.uint32)
    rng = np.random.default_rng(281)
    sources, parents = [], []
    for root, good in zip(ref["beamer_hybrid.roots"], ref["beamer_hybrid.parent"]):
        for p in planted_parents(off, adj, int(root), good, rng):
            sources.append(int(root))
            parents.append(p)
    sources = np.array(sources, np.int64)
    parents = np.stack(parents)
    verdict, stop = ref_check(el10, sources, parents, tmp)
    trees = ref_print_tree(el10, ref["beamer_hybrid.roots"], ref["beamer_hybrid.parent"], tmp)
    tree_bytes = [t.encode() for t in trees]
    np.savez_compressed(os.path.join(HERE, "ref_check.npz"), sources=sources, parents=parents,
                        verdict=verdict, stop=stop,
                        tree_text=np.frombuffer(b"".join(tree_bytes), np.uint8),
                        tree_offsets=np.cumsum([0] + [len(b) for b in tree_bytes]).astype(np.int64))


def planted_labellings(off, good):
    """Correct and wrong labellings of one graph, made from its labels."""
    uniq, counts = np.unique(good, return_counts=True)
    big = int(uniq[np.argmax(counts)])
    other = int(uniq[uniq != big][0])
    members = np.flatnonzero(good == big)
    out = [good.copy()]
    bad = good.copy()
    bad[members[len(members) // 2]] = -7
    out.append(bad)
    bad = good.copy()
    bad[good == other] = big
    out.append(bad)
    out.append(good * 3 + (1 << 40))
    bad = good.copy()
    bad[good == big], bad[good == other] = other, big
    out.append(bad)
    out.append(np.zeros_like(good))
    isolated = np.flatnonzero(np.diff(off) == 0)
    if len(isolated):
        bad = good.copy()
        bad[isolated[-1]] = big
        out.append(bad)
    return np.stack(out)


def ref_components_check(el64, planted, tmp):
    path = os.path.join(tmp, "planted.bin")
    with open(path, "wb") as f:
        f.write(np.array(planted.shape, np.int64).tobytes())
        f.write(np.ascontiguousarray(planted, np.int64).tobytes())
    out = subprocess.run([os.path.join(O.REF_DIR, "ref_components_check"), "--graph_filename",
                          el64, "--labels", path], check=True, stdout=subprocess.PIPE,
                         stderr=subprocess.DEVNULL, text=True).stdout
    verdicts = [int(v) for v in re.findall(r"VERDICT (\d)", out)]
    assert len(verdicts) == len(planted)
    return np.array(verdicts, np.int64)


def with_tail(graph, k):
    """The graph with k new vertices at the end joined as a path (k = 1: one
    isolated vertex), so the last component is one run ending at vertex
    n-1: the reference's dump prints no newline after that line."""
    n, src, dst = graph
    extra = np.arange(n, n + k - 1, dtype=np.int64)
    return n + k, np.concatenate([src, extra]), np.concatenate([dst, extra + 1])


def components_fixture(tmp):
    graphs = {"scale10": O.el64_load(os.path.join(HERE, "graph500-scale10.el64")),
              "rmat12_ef2": O.rmat_graph(12, edge_factor=2, seed=5),
              "grid48": O.grid_graph(48, 48, 0.3, seed=3),
              "tail_isolated": with_tail(O.rmat_graph(10, edge_factor=4, seed=9), 1),
              "tail_path": with_tail(O.el64_load(os.path.join(HERE, "graph500-scale10.el64")), 3)}
    arrays = {}
    for name, (n, src, dst) in graphs.items():
        el = os.path.join(tmp, name + ".el64")
        O.el64_write(el, n, src, dst)
        off, adj = O.csr_build(n, src, dst)
        labels, count, iters, passed, dump = ref_components(el, n)
        planted = planted_labellings(off, labels)
        arrays.update({f"{name}.offsets": off, f"{name}.adj": adj, f"{name}.labels": labels,
                       f"{name}.summary": np.array([count, iters, int(passed)], np.int64),
                       f"{name}.dump": np.frombuffer(dump.encode(), np.uint8),
                       f"{name}.planted": planted,
                       f"{name}.planted_verdict": ref_components_check(el, planted, tmp)})
    np.savez_compressed(os.path.join(HERE, "ref_components.npz"), **arrays)


# (scale, edge factor, a, b, c, d, seed) of the generator fixture; the first
# case keeps its full edge lists, the others their sha256.  The last one
# makes most edges self loops, so the serial re-roll runs long.
GEN_CASES = [
    (10, 16, 0.57, 0.19, 0.19, 0.05, 0),
    (12, 16, 0.57, 0.19, 0.19, 0.05, 0),
    (11, 4, 0.45, 0.25, 0.25, 0.05, 7),
    (14, 16, 0.57, 0.19, 0.19, 0.05, 12345),
    (9, 32, 0.7, 0.1, 0.1, 0.1, 3),
    (8, 8, 0.9, 0.03, 0.03, 0.04, 11),
]


def ref_gen_edges(case, tmp):
    """The reference generator's edges for one case (oracle/_ref/ref_gen_edges):
    generation order after the self-loop re-roll, and the deduplicated,
    sorted list of rmat_dataset_dump.cc:48-53."""
    path = os.path.join(tmp, "gen.bin")
    subprocess.run([os.path.join(O.REF_DIR, "ref_gen_edges")] + [str(x) for x in case] + [path],
                   check=True)
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:8] == b"BDGEN001"
    nv, e = np.frombuffer(raw[8:24], np.int64)
    gen = np.frombuffer(raw[24:24 + 16 * e], np.int64).reshape(e, 2)
    m = int(np.frombuffer(raw[24 + 16 * e:32 + 16 * e], np.int64)[0])
    ded = np.frombuffer(raw[32 + 16 * e:], np.int64).reshape(m, 2)
    return int(nv), gen, ded


def generator_fixture(tmp):
    """ref_gen.npz: per case, the parameters, the generated and deduplicated
    edge counts and the sha256 of both lists (int64 src, dst pairs, in
    order); the first case also keeps both lists whole."""
    arrays = {"cases": np.array([(c[0], c[1], c[6]) for c in GEN_CASES], np.int64),
              "params": np.array([c[2:6] for c in GEN_CASES], np.float64)}
    for i, case in enumerate(GEN_CASES):
        nv, gen, ded = ref_gen_edges(case, tmp)
        arrays[f"{i}.counts"] = np.array([nv, len(gen), len(ded),
                                          int((gen[:, 0] == gen[:, 1]).sum())], np.int64)
        arrays[f"{i}.gen_sha"] = np.frombuffer(hashlib.sha256(gen.tobytes()).digest(), np.uint8)
        arrays[f"{i}.ded_sha"] = np.frombuffer(hashlib.sha256(ded.tobytes()).digest(), np.uint8)
        if i == 0:
            arrays["0.gen"] = gen
            arrays["0.ded"] = ded
    np.savez_compressed(os.path.join(HERE, "ref_gen.npz"), **arrays)


def main():
    O.build()
    flags = ("--components", "--check", "--generator")
    if any(f in sys.argv[1:] for f in flags):
        with tempfile.TemporaryDirectory() as tmp:
            if "--components" in sys.argv[1:]:
                components_fixture(tmp)
            if "--check" in sys.argv[1:]:
                check_fixture(tmp)
            if "--generator" in sys.argv[1:]:
                generator_fixture(tmp)
        return
    if not os.path.exists(os.path.join(O.REF_DIR, "ref_dump")):
        sys.exit("reference builds missing: the reference sources are needed")
    golden = {"generator": {"a": 0.57, "b": 0.19, "c": 0.19, "d": 0.05, "edge_factor": 16}}

    # 1. reference generator output, scale 10
    el10 = os.path.join(HERE, "graph500-scale10.el64")
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, OMP_NUM_THREADS="1")
        subprocess.run([os.path.join(O.REF_DIR, "rmat_dataset_dump"), "graph500-scale10"],
                       cwd=tmp, env=env, check=True, stderr=subprocess.DEVNULL)
        os.replace(os.path.join(tmp, "graph500-scale10"), el10)
        arrays = {}
        for i, alg in enumerate(REF_ALGS):
            d = ref_dump(el10, os.path.join(tmp, "s10.bin"), alg, 8, dump_graph=(i == 0))
            if i == 0:
                arrays["offsets"] = d["offsets"]
                arrays["adj"] = d["adj"]
            for key, val in pack_roots(d).items():
                arrays[f"{alg}.{key}"] = val
        np.savez_compressed(os.path.join(HERE, "ref_scale10.npz"), **arrays)
        golden["graph500-scale10.el64"] = {"sha256": sha256_file(el10)}

        # 2. project generator, scale 12, full detail
        n, src, dst = O.rmat_graph(12, seed=12)
        el12 = os.path.join(tmp, "gen12.el64")
        O.el64_write(el12, n, src, dst)
        d = ref_dump(el12, os.path.join(tmp, "g12.bin"), "beamer_hybrid", 8)
        arrays = pack_roots(d)
        arrays["num_edges"] = np.array([len(src)], np.int64)
        np.savez_compressed(os.path.join(HERE, "ref_gen12.npz"), **arrays)
        golden["gen12"] = {"scale": 12, "seed": 12, "num_edges": int(len(src)),
                           "el64_sha256": sha256_file(el12)}

        # 3. project generator, scale 16: hashes and per-root summaries
        n, src, dst = O.rmat_graph(16, seed=16)
        el16 = os.path.join(tmp, "gen16.el64")
        O.el64_write(el16, n, src, dst)
        off, adj = O.csr_build(n, src, dst)
        d = ref_dump(el16, os.path.join(tmp, "g16.bin"), "beamer_hybrid", 8)
        roots = []
        for r in d["roots"]:
            dirs, depth = level_dirs(r["parent"], r["bottom_up"], r["root"])
            roots.append({
                "root": r["root"],
                "check": r["check"],
                "m_c": r["m_c"],
                "found": np.diff(r["heads"]).tolist(),
                "level_dirs": dirs,
                "depth_sha256": hashlib.sha256(depth.astype("<i4").tobytes()).hexdigest(),
                "reference_ms": round(r["ms"], 3),
            })
        golden["gen16"] = {
            "scale": 16, "seed": 16, "num_edges": int(len(src)),
            "el64_sha256": sha256_file(el16),
            "csr_sha256": hashlib.sha256(off.astype("<i8").tobytes()
                                         + adj.astype("<u4").tobytes()).hexdigest(),
            "alpha": 15, "beta": 18, "roots": roots,
        }
        components_fixture(tmp)
        check_fixture(tmp)
        generator_fixture(tmp)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
