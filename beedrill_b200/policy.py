"""The learned direction policy: data collection, training and evaluation.

The policy is an fp32 MLP (8 -> 32 -> 32 -> 2) that the persistent BFS kernel
evaluates on the device before every level, in place of run_beamer's
alpha/beta rule (hybrid_bfs.cc:166-188).  Beamer's rule stays the fallback
(no policy installed, or a logit gap below the margin) and the yardstick of
the policy's regret.

Training data come from the plain BFS itself.  A top-down step and a
bottom-up step from the same state discover the same next level, so the
state before level L does not depend on the directions taken before it.
One forced top-down run and one forced bottom-up run per root therefore give
the cost of BOTH directions at EVERY level:  t_td[L], t_bu[L].  The label of
level L is the faster direction, its weight the time difference, and the
best achievable total is sum_L min(t_td[L], t_bu[L]).

Forward, backward and Adam run in the hand-written kernels of
beedrill_b200/csrc/bd_policy.cu (bd_policy_train).

    python -m beedrill_b200.policy train --out beedrill_b200/policy/learned_policy.json
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time
from dataclasses import dataclass, field

import numpy as np

import beedrill_b200 as bd

NUM_PARAMS = 1410
NUM_FEATURES = 8
DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "policy",
                            "learned_policy.json")
# push/pull policy of the batched (64-root) traversal
BATCHED_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "policy",
                            "learned_policy_batched.json")


def raw_features(frontier, frontier_edges, unexplored, level, n, m, prev_dir, prev_ns):
    """The features the traversal kernels compute on the device
    (policy_feature in bd_policy.cuh), in the same order, units and float32
    arithmetic: differences of log2(1 + x) terms, so that one range covers
    graphs of every size --
      0 m_f vs m_u, 1 frontier vs n, 2 m_u vs 2m, 3 level (alone),
      4 m vs n, 5 previous direction, 6 previous step us vs m / 2^20,
      7 m_f vs frontier."""
    one = np.float32(1.0)

    def lg(x):
        return np.log2(one + np.maximum(np.float32(x), np.float32(0)), dtype=np.float32)

    def f32(x):
        return np.float32(max(int(x), 0))

    f = np.empty(NUM_FEATURES, np.float32)
    f[0] = lg(f32(frontier_edges)) - lg(f32(unexplored))
    f[1] = lg(f32(frontier)) - lg(f32(n))
    f[2] = lg(f32(unexplored)) - lg(f32(2 * m))
    f[3] = lg(f32(level))
    f[4] = lg(f32(m)) - lg(f32(n))
    f[5] = prev_dir
    f[6] = lg(f32(prev_ns) * np.float32(1e-3)) - lg(f32(m) * np.float32(1.0 / 1048576.0))
    f[7] = lg(f32(frontier_edges)) - lg(f32(frontier))
    return f


@dataclass
class LevelTable:
    """Per-level costs of both directions for one (graph, root)."""
    n: int
    m: int
    frontier: np.ndarray
    frontier_edges: np.ndarray
    unexplored: np.ndarray
    found: np.ndarray
    t_td: np.ndarray  # ns
    t_bu: np.ndarray  # ns
    beamer_dirs: str = ""
    beamer_ns: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def levels(self) -> int:
        return len(self.t_td)

    def optimal_ns(self) -> float:
        return float(np.minimum(self.t_td, self.t_bu).sum())

    def cost_ns(self, dirs: str) -> float:
        t = 0.0
        for lv, d in enumerate(dirs[: self.levels]):
            t += self.t_bu[lv] if d == "B" else self.t_td[lv]
        return float(t)

    def features(self, lv: int, prev_dir: int, prev_ns: float) -> np.ndarray:
        return raw_features(self.frontier[lv], self.frontier_edges[lv], self.unexplored[lv], lv,
                            self.n, self.m, prev_dir, prev_ns)


def measure_tables(graph: "bd.Graph", roots, repeats: int = 1, with_beamer: bool = True):
    """Forced top-down and forced bottom-up runs from each root; returns one
    LevelTable per root (per-level times are the minimum over `repeats`)."""
    n, m = graph.num_vertices(), graph.num_edges()
    td = bd.HybridBFS(graph, alg="top_down")
    bu = bd.HybridBFS(graph, alg="bottom_up")
    bm = bd.HybridBFS(graph, alg="beamer_hybrid") if with_beamer else None
    tables = []
    for root in roots:
        root = int(root)
        runs = {}
        for name, h in (("td", td), ("bu", bu)):
            best = None
            for _ in range(repeats):
                h.clear()
                h.run(root)
                st = h.steps()
                t = np.array([s["ns"] for s in st], np.float64)
                best = t if best is None else np.minimum(best, t)
                runs[name] = st
            runs[name + "_t"] = best
        a, b = runs["td"], runs["bu"]
        if len(a) != len(b) or any(x["found"] != y["found"] for x, y in zip(a, b)):
            raise RuntimeError("forced runs disagree on the level structure")
        tab = LevelTable(
            n=n, m=m,
            frontier=np.array([s["frontier"] for s in a], np.int64),
            frontier_edges=np.array([s["frontier_edges"] for s in a], np.int64),
            unexplored=np.array([s["unexplored_edges"] for s in a], np.int64),
            found=np.array([s["found"] for s in a], np.int64),
            t_td=runs["td_t"], t_bu=runs["bu_t"], meta={"root": root})
        if bm is not None:
            bm.clear()
            stats = bm.run(root)
            tab.beamer_dirs = bm.directions()
            tab.beamer_ns = stats.ms * 1e6
        tables.append(tab)
    for h in (td, bu, bm):
        if h is not None:
            h.close()
    return tables


def measure_tables_batched(graph: "bd.Graph", roots, repeats: int = 1, alpha: int | None = None):
    """Forced push and forced pull runs of one batch of up to 64 roots; one
    LevelTable whose top-down / bottom-up columns hold push / pull times,
    `found` counts new (vertex, root) pairs and `unexplored` is the degree
    sum of vertices some root has not reached."""
    n, m = graph.num_vertices(), graph.num_edges()
    runs = {}
    for name, fd in (("push", 0), ("pull", 1)):
        h = bd.BatchedBFS(graph, len(roots), force_dir=fd)
        best = None
        for _ in range(repeats):
            h.run(roots)
            st = h.steps()
            t = np.array([s["ns"] for s in st], np.float64)
            best = t if best is None else np.minimum(best, t)
        runs[name], runs[name + "_t"] = st, best
        h.close()
    a, b = runs["push"], runs["pull"]
    if len(a) != len(b) or any(x["found"] != y["found"] for x, y in zip(a, b)):
        raise RuntimeError("forced batched runs disagree on the level structure")
    if alpha is None:  # the rule a batched handle on this graph uses
        alpha = bd.tuned_options("batched", n).get("alpha", 4)
    rule = bd.BatchedBFS(graph, len(roots), alpha=alpha)
    st = rule.run(roots)
    tab = LevelTable(
        n=n, m=m,
        frontier=np.array([s["frontier"] for s in a], np.int64),
        frontier_edges=np.array([s["frontier_edges"] for s in a], np.int64),
        unexplored=np.array([s["unexplored_edges"] for s in a], np.int64),
        found=np.array([s["found"] for s in a], np.int64),
        t_td=runs["push_t"], t_bu=runs["pull_t"], beamer_dirs=rule.directions(),
        beamer_ns=st.ms * 1e6, meta={"roots": len(roots), "alpha": alpha})
    rule.close()
    return tab


def alpha_dirs(tab: LevelTable, alpha=None) -> str:
    """The batched traversal's rule over a level table (ms_rule in
    bd_msbfs.cu): pull when the frontier's degree sum times alpha exceeds
    the unexplored degree sum and the frontier holds at least n / 1024
    vertices.  alpha defaults to the tuned value a batched handle on a
    graph of that size uses."""
    if alpha is None:
        alpha = bd.tuned_options("batched", tab.n).get("alpha", 4)
    out = []
    for lv in range(tab.levels):
        pull = (tab.frontier_edges[lv] * alpha > tab.unexplored[lv]
                and tab.frontier[lv] * 1024 >= tab.n)
        out.append("B" if pull else "T")
    return "".join(out)


def dataset(tables):
    """Samples (raw features, label, weight).  Level 0 has no previous step;
    later levels appear once per possible previous direction."""
    X, y, w = [], [], []
    for tab in tables:
        for lv in range(tab.levels):
            label = 1 if tab.t_bu[lv] < tab.t_td[lv] else 0
            weight = abs(tab.t_bu[lv] - tab.t_td[lv]) * 1e-3  # microseconds
            prevs = [(0, 0.0)] if lv == 0 else [(0, tab.t_td[lv - 1]), (1, tab.t_bu[lv - 1])]
            for pd, pns in prevs:
                X.append(tab.features(lv, pd, pns))
                y.append(label)
                w.append(weight)
    return np.array(X, np.float32), np.array(y, np.int32), np.array(w, np.float32)


@dataclass
class Policy:
    params: np.ndarray
    mean: np.ndarray
    inv_std: np.ndarray
    margin: float = 0.0
    info: dict = field(default_factory=dict)
    lo: np.ndarray | None = None  # trusted raw-feature range (None: unbounded)
    hi: np.ndarray | None = None
    extremes: tuple | None = None  # training (min, max, std) per feature
    band: tuple | None = None  # feature-0 range the network decides in

    def trusts(self, raw: np.ndarray) -> bool:
        if self.lo is None:
            return True
        return bool(np.all(raw >= self.lo) and np.all(raw <= self.hi))

    def logits(self, raw: np.ndarray) -> np.ndarray:
        """Host float32 forward pass (for simulation only; the BFS uses the
        device copy)."""
        p = self.params.astype(np.float32)
        x = (np.atleast_2d(raw).astype(np.float32) - self.mean) * self.inv_std
        w1 = p[0:256].reshape(32, 8); b1 = p[256:288]
        w2 = p[288:1312].reshape(32, 32); b2 = p[1312:1344]
        w3 = p[1344:1408].reshape(2, 32); b3 = p[1408:1410]
        h1 = np.maximum(x @ w1.T + b1, 0)
        h2 = np.maximum(h1 @ w2.T + b2, 0)
        return h2 @ w3.T + b3

    def save(self, path: str) -> None:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        with open(path, "w") as f:
            d = {"params": [float(v) for v in self.params],
                 "mean": [float(v) for v in self.mean],
                 "inv_std": [float(v) for v in self.inv_std],
                 "margin": float(self.margin), "info": self.info}
            if self.lo is not None:
                d["lo"] = [float(v) for v in self.lo]
                d["hi"] = [float(v) for v in self.hi]
            json.dump(d, f)
            f.write("\n")

    @classmethod
    def load(cls, path: str = DEFAULT_PATH) -> "Policy":
        with open(path) as f:
            d = json.load(f)
        lo = np.array(d["lo"], np.float32) if "lo" in d else None
        hi = np.array(d["hi"], np.float32) if "hi" in d else None
        return cls(np.array(d["params"], np.float32), np.array(d["mean"], np.float32),
                   np.array(d["inv_std"], np.float32), float(d["margin"]), d.get("info", {}),
                   lo, hi)

    def install(self, bfs: "bd.HybridBFS") -> None:
        bfs.set_policy(self.params, self.mean, self.inv_std, self.margin, self.lo, self.hi)


def decisions_policy(policy: Policy) -> Policy | None:
    """The trained network with the trusted range and margin that its
    decisions alone favour (before its inference cost is counted), or None
    if the trainer found none better than the rule."""
    d = policy.info.get("decisions_only", {})
    if d.get("lo") is None:
        return None
    return Policy(policy.params, policy.mean, policy.inv_std, float(d["margin"]), policy.info,
                  np.array(d["lo"], np.float32), np.array(d["hi"], np.float32))


def beamer_dirs(tab: LevelTable, alpha=15, beta=18) -> str:
    """run_beamer's decisions over a level table (hybrid_bfs.cc:152-191)."""
    etc, scout = 2 * tab.m, int(tab.frontier_edges[0])
    in_bu, awake = False, 0
    out = []
    for lv in range(tab.levels):
        if in_bu:
            d = "B"
        elif scout > etc // alpha:
            in_bu, awake, d = True, int(tab.frontier[lv]), "B"
        else:
            etc -= scout
            d = "T"
        out.append(d)
        found = int(tab.found[lv])
        if d == "T":
            scout = int(tab.frontier_edges[lv + 1]) if lv + 1 < tab.levels else 0
        elif in_bu:
            old, awake = awake, found
            if not (awake >= old or awake > tab.n // beta):
                in_bu, scout = False, 1
    return "".join(out)


def policy_dirs(policy: Policy, tab: LevelTable, alpha=15, beta=18, rule=None) -> str:
    """Decisions the policy makes along a level table (the rule -- Beamer by
    default -- where the logit gap is below the margin or a feature is out
    of the trusted range)."""
    rule = rule if rule is not None else beamer_dirs(tab, alpha, beta)
    out = []
    prev_dir, prev_ns = 0, 0.0
    for lv in range(tab.levels):
        raw = tab.features(lv, prev_dir, prev_ns)
        z = policy.logits(raw)[0]
        gap = float(z[1] - z[0])
        trusted = policy.trusts(raw) and abs(gap) >= policy.margin
        d = ("B" if gap > 0 else "T") if trusted else rule[lv]
        out.append(d)
        prev_dir = 1 if d == "B" else 0
        prev_ns = tab.t_bu[lv] if d == "B" else tab.t_td[lv]
    return "".join(out)


def regret(tables, dirs_fn) -> dict:
    cost = sum(t.cost_ns(dirs_fn(t)) for t in tables)
    best = sum(t.optimal_ns() for t in tables)
    return {"cost_ms": cost * 1e-6, "optimal_ms": best * 1e-6,
            "regret_ms": (cost - best) * 1e-6, "regret_frac": (cost - best) / best}


def he_init(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, np.sqrt(2.0 / 8), (32, 8))
    w2 = rng.normal(0, np.sqrt(2.0 / 32), (32, 32))
    w3 = rng.normal(0, np.sqrt(1.0 / 32), (2, 32))
    return np.concatenate([w1.ravel(), np.zeros(32), w2.ravel(), np.zeros(32), w3.ravel(),
                           np.zeros(2)]).astype(np.float32)


def fit(X, y, w, epochs=3000, lr=3e-3, weight_decay=1e-4, seed=0, widen=3.0, band=None):
    """Standardises the features and trains on the device; returns a Policy
    (margin 0) whose trusted range is the training extremes widened by
    `widen` standard deviations, and the loss history."""
    mean = X.mean(0).astype(np.float32)
    std = X.std(0).astype(np.float32)
    inv_std = np.where(std > 1e-6, 1.0 / np.maximum(std, 1e-6), 0.0).astype(np.float32)
    Xs = ((X - mean) * inv_std).astype(np.float32)
    params = he_init(seed)
    hist = bd.policy_train(params, Xs, y, w, epochs, lr, weight_decay)
    pol = Policy(params, mean, inv_std, 0.0, {}, None, None)
    pol.extremes = (X.min(0).astype(np.float32), X.max(0).astype(np.float32), std)
    pol.band = band
    set_widen(pol, widen)
    return pol, hist


def set_widen(pol: Policy, widen: float) -> None:
    """Trusted range: the training extremes widened by `widen` standard
    deviations, feature 0 cut to the policy's band (the kernels test
    feature 0 first and run the network only inside it)."""
    xmin, xmax, std = pol.extremes
    pol.lo = (xmin - widen * std).astype(np.float32)
    pol.hi = (xmax + widen * std).astype(np.float32)
    if pol.band is not None:
        pol.lo[0] = max(pol.lo[0], np.float32(pol.band[0]))
        pol.hi[0] = min(pol.hi[0], np.float32(pol.band[1]))


# the band extends this far (log2 units) past the feature-0 values at which
# the best direction differed from the rule's
BAND_PAD = 1.0


def network_band(policy: Policy, tables, rule_fn):
    """The feature-0 range (padded by BAND_PAD) of the levels at which the
    policy, trusted and confident, picks another direction than the rule,
    along its own path over `tables`; None when it never does."""
    f0 = []
    for t in tables:
        rule = rule_fn(t)
        dirs = policy_dirs(policy, t, rule=rule)
        prev_dir, prev_ns = 0, 0.0
        for lv, d in enumerate(dirs):
            if d != rule[lv]:
                f0.append(t.features(lv, prev_dir, prev_ns)[0])
            prev_dir = 1 if d == "B" else 0
            prev_ns = t.t_bu[lv] if d == "B" else t.t_td[lv]
    if not f0:
        return None
    return float(min(f0) - BAND_PAD), float(max(f0) + BAND_PAD)


def disagreement_band(tables, rule_fn):
    """The range of feature 0 (log2 of frontier edges over unexplored edges)
    over the levels of `tables` at which the faster direction is not the
    rule's, padded by BAND_PAD; None when the rule is right at every level.
    Outside it the rule decides without the network."""
    f0 = []
    for t in tables:
        dirs = rule_fn(t)
        for lv in range(t.levels):
            best = "B" if t.t_bu[lv] < t.t_td[lv] else "T"
            if best != dirs[lv]:
                f0.append(t.features(lv, 0, 0.0)[0])
    if not f0:
        return None
    return float(min(f0) - BAND_PAD), float(max(f0) + BAND_PAD)


WIDEN_CANDIDATES = (0.0, 0.5, 1.0, 2.0, 3.0)
MARGIN_CANDIDATES = (0.0, 0.25, 0.5, 1.0, 2.0)
OFF = float("inf")  # margin of a policy that leaves every step to the rule


# the graph the inference cost is measured on: thousands of small levels, so
# a per-level cost of a few hundred ns stands out of the run-to-run noise
OVERHEAD_SPEC = {"kind": "grid", "rows": 1024, "cols": 1024, "delete": 0.01, "scale": 20,
                 "seed": 31_337}


def inference_overhead(spec, policy, batched: bool, roots=4, repeats=5):
    """Measured cost of the policy inside the traversal kernel, in ns per
    level: (outside its band, inside it).  Three handles run the same
    roots: no policy, a policy trusted nowhere (the kernel tests feature 0
    against the band and stops), and one trusted everywhere whose margin
    never lets it override (the network runs, the rule still decides).
    `spec` None: OVERHEAD_SPEC."""
    spec = OVERHEAD_SPEC if spec is None else spec
    g = spec_graph(spec)
    rs = g.pick_roots(spec["seed"] + 1, 64 if batched else roots)
    big = np.full(NUM_FEATURES, 1e30, np.float32)
    make = (lambda: bd.BatchedBFS(g, len(rs))) if batched else \
        (lambda: bd.HybridBFS(g, alg="learned"))
    variants = {"none": None, "features": (big, -big, 1.0), "network": (-big, big, 1e30)}
    out = {}
    for name, v in variants.items():
        h = make()
        if v is not None:
            h.set_policy(policy.params, policy.mean, policy.inv_std, v[2], v[0], v[1])
        ms, levels = [], []
        for _ in range(repeats + 1):
            if batched:
                st = h.run(rs)
                ms.append(st.ms)
                levels.append(len(h.steps()))
            else:
                t, lv = 0.0, 0
                for r in rs:
                    h.clear()
                    st = h.run(int(r))
                    t += st.ms
                    lv += len(h.steps())
                ms.append(t)
                levels.append(lv)
        out[name] = (min(ms[1:]), float(np.mean(levels[1:])))
        h.close()
    g.close()
    per_level = lambda a: max(0.0, (out[a][0] - out["none"][0]) * 1e6 / out["none"][1])  # noqa: E731
    return per_level("features"), per_level("network")


def priced_cost_ns(policy: Policy, tables, rule_fn, overhead) -> float:
    """Cost of the policy's decisions plus its own inference cost: the
    features at every level it is installed for, the network at the levels
    its features are trusted."""
    if policy.margin == OFF:
        return sum(t.cost_ns(rule_fn(t)) for t in tables)
    total = 0.0
    for t in tables:
        dirs = policy_dirs(policy, t, rule=rule_fn(t))
        total += t.cost_ns(dirs)
        prev_dir, prev_ns = 0, 0.0
        for lv, d in enumerate(dirs):
            raw = t.features(lv, prev_dir, prev_ns)
            total += overhead[1] if policy.trusts(raw) else overhead[0]
            prev_dir = 1 if d == "B" else 0
            prev_ns = t.t_bu[lv] if d == "B" else t.t_td[lv]
    return total


def train_policy(tables, rule_fn, args, log, batched=False):
    """Training with its two choices made on graphs it did not train on.

    * How far past the training extremes the network may decide (its
      trusted range) is chosen for extrapolation: a probe network trained
      on the smaller training scales is scored, decisions alone, on the
      largest one.
    * Whether the network decides at all, and with what margin, is chosen
      on validation graphs of every training scale, priced with the
      network's measured inference cost inside the traversal kernel: the
      network is kept only where its decisions save more than it costs.

    Graphs split by seed: every 5th (seed % 5 == 0) for the report, the
    next (seed % 5 == 1) for the margin, the rest for training."""
    report = [t for t in tables if t.meta["seed"] % 5 == 0]
    val = [t for t in tables if t.meta["seed"] % 5 == 1]
    train = [t for t in tables if t.meta["seed"] % 5 > 1]
    top = max(t.meta["scale"] for t in train)
    lower = [t for t in train if t.meta["scale"] < top]
    upper = [t for t in train if t.meta["scale"] == top]
    band = disagreement_band(train, rule_fn)
    log(f"feature-0 band where the rule's choice is not the faster one: {band}")
    if band is None:  # the rule is right everywhere: an empty band keeps the network out
        band = (1.0, -1.0)
    X, y, w = dataset(lower)
    probe, _ = fit(X, y, w, epochs=args.epochs, lr=args.lr, band=band)
    widen_cost = []
    for widen in WIDEN_CANDIDATES:
        set_widen(probe, widen)
        widen_cost.append((regret(upper, lambda t: policy_dirs(probe, t, rule=rule_fn(t)))["cost_ms"],
                           widen))
    widen = min(widen_cost)[1]
    log(f"trusted range for extrapolation to scale {top}: training extremes +{widen} sd")
    X, y, w = dataset(train)
    policy, hist = fit(X, y, w, epochs=args.epochs, lr=args.lr, widen=widen, band=band)
    # the network is needed only where it disagrees with the rule: cut the
    # band to the feature-0 range of those levels (training tables, along
    # the network's own path), so elsewhere the kernels skip it
    tight = network_band(policy, train, rule_fn)
    log(f"feature-0 band where the network overrides the rule: {tight}")
    policy.band = tight if tight is not None else (1.0, -1.0)
    set_widen(policy, widen)
    overhead = inference_overhead(None, policy, batched)
    log(f"inference cost per level: features {overhead[0]:.0f} ns, network {overhead[1]:.0f} ns")
    policy.margin = OFF
    rule_cost = priced_cost_ns(policy, val, rule_fn, overhead)
    best, best_d = (rule_cost, OFF), (rule_cost, OFF)
    for mgn in MARGIN_CANDIDATES:
        policy.margin = mgn
        cost = priced_cost_ns(policy, val, rule_fn, overhead)
        cost_d = priced_cost_ns(policy, val, rule_fn, (0.0, 0.0))
        if cost < best[0] - 1e-6:
            best = (cost, mgn)
        if cost_d < best_d[0] - 1e-6:
            best_d = (cost_d, mgn)
    log(f"margin {best[1]} ({best[0] * 1e-6:.3f} ms with inference vs rule {rule_cost * 1e-6:.3f} ms "
        f"on {len(val)} validation tables); decisions alone favour margin {best_d[1]}")
    rb = regret(report, rule_fn)
    decisions = {"trust_widen_sd": widen, "margin": best_d[1]}
    if best_d[1] != OFF:
        policy.margin = best_d[1]
        decisions.update(lo=[float(v) for v in policy.lo], hi=[float(v) for v in policy.hi],
                         validation={"rule": rb, "learned": regret(
                             report, lambda t: policy_dirs(policy, t, rule=rule_fn(t)))})
    policy.margin = best[1]
    rl = regret(report, lambda t: policy_dirs(policy, t, rule=rule_fn(t)))
    policy.info = {"samples": int(len(y)), "epochs": args.epochs, "lr": args.lr,
                   "loss_first": float(hist[0]), "loss_last": float(hist[-1]),
                   "margin": best[1], "trust_widen_sd": widen,
                   "inference_ns_per_level": {"features": overhead[0], "network": overhead[1]},
                   "selection": f"trusted range: train on scales < {top}, score on {top}; margin: "
                                "validation graphs of every scale, priced with the measured "
                                "inference cost",
                   "validation": {"rule": rb, "learned": rl},
                   "decisions_only": decisions}
    return policy, rb, rl


def training_graph_specs(count=200, seed=2024, large=True, grids=True):
    """The training distribution: RMAT scales 16-22, A ~ U[0.45, 0.65],
    D = 0.05, B = C = (1 - A - D) / 2, edge factor 16; with `large`, five
    more at scales 23-24 (A = 0.57); with `grids`, six rows x cols grids
    (512^2 to 2048^2, 1 % of the edges deleted), whose thousands of small
    levels are the high-diameter case.  Graph seeds decide the split
    (seed % 5: 0 report, 1 validation, else training)."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(count):
        a = float(rng.uniform(0.45, 0.65))
        d = 0.05
        b = c = (1.0 - a - d) / 2
        specs.append({"kind": "rmat", "scale": int(16 + k % 7), "edge_factor": 16, "a": a, "b": b,
                      "c": c, "d": d, "seed": 10_000 + k})
    if large:
        for scale, s in ((23, 20_002), (23, 20_003), (23, 20_001), (24, 20_012), (24, 20_014)):
            specs.append({"kind": "rmat", "scale": scale, "edge_factor": 16, "a": 0.57,
                          "b": 0.19, "c": 0.19, "d": 0.05, "seed": s})
    if grids:
        for side, s in ((512, 30_002), (1024, 30_003), (1024, 30_001), (2048, 30_004),
                        (2048, 30_007), (2048, 30_005)):
            specs.append({"kind": "grid", "rows": side, "cols": side, "delete": 0.01,
                          "scale": int(np.log2(side * side)), "seed": s})
    return specs


def spec_graph(s, order=None):
    """The graph of a training spec, in the layout the policy runs on."""
    order = bd.ORDER_HUB if order is None else order
    if s.get("kind", "rmat") == "grid":
        return bd.Graph.grid(s["rows"], s["cols"], s["delete"], s["seed"], order=order)
    return bd.Graph.rmat(s["scale"], s["edge_factor"], s["a"], s["b"], s["c"], s["d"], s["seed"],
                         order=order)


def collect(specs, roots_per_graph=8, repeats=2, log=None, order=None):
    """Level tables of the training graphs, built with the layout the
    policy will run on (the hub numbering by default, as the benchmark's
    graphs are; the layout changes step costs)."""
    tables = []
    for i, s in enumerate(specs):
        g = spec_graph(s, order)
        roots = g.pick_roots(s["seed"], roots_per_graph if s.get("kind") != "grid" else 2)
        for t in measure_tables(g, roots, repeats=repeats, with_beamer=False):
            t.meta.update(s)
            tables.append(t)
        g.close()
        if log and (i + 1) % 20 == 0:
            log(f"collected {i + 1}/{len(specs)} graphs")
    return tables


def train_batched(args, log):
    """The push/pull policy of the batched traversal, trained the same way
    on one 64-root batch per training graph."""
    specs = training_graph_specs(args.graphs)
    tables = []
    t0 = time.time()
    for i, s in enumerate(specs):
        g = spec_graph(s)
        tab = measure_tables_batched(g, g.pick_roots(s["seed"], 64), repeats=2)
        tab.meta.update(s)
        tables.append(tab)
        g.close()
        if (i + 1) % 20 == 0:
            log(f"collected {i + 1}/{len(specs)} graphs")
    log(f"{len(tables)} batched level tables in {time.time() - t0:.1f} s")
    policy, rb, rl = train_policy(tables, alpha_dirs, args, log, batched=True)
    policy.info.update({"kind": "batched", "graphs": args.graphs,
                        "distribution": "RMAT scales 16-22, A~U[0.45,0.65], D=0.05, "
                                        "B=C=(1-A-D)/2, ef 16; 5 RMAT graphs at scales 23-24; "
                                        "6 grids 512^2-2048^2 (1% of edges deleted); 64 roots per "
                                        "graph, hub numbering"})
    policy.save(args.out)
    log(f"saved {args.out}: rule regret {rb['regret_frac']:.3%}, learned {rl['regret_frac']:.3%}")
    return 0


def headroom(args, log):
    """How much any direction policy could gain on one graph: per level, the
    measured cost of both directions (forced runs; a level discovers the
    same vertices either way), the rule's choices, and the sum of the
    per-level minima against the rule's cost on the same table."""
    g = bd.Graph.rmat(args.scale, 16, seed=args.seed, order=bd.ORDER_HUB)
    out = {"graph": {"scale": args.scale, "seed": args.seed, "n": g.num_vertices(),
                     "m": g.num_edges()}}
    if args.batched:
        tab = measure_tables_batched(g, g.pick_roots(args.root_seed, 64), repeats=args.repeats)
        rule = alpha_dirs(tab)
        tables, names = [tab], ("push", "pull")
    else:
        tables = measure_tables(g, g.pick_roots(args.root_seed, args.roots), repeats=args.repeats,
                                with_beamer=False)
        rule, names = None, ("top-down", "bottom-up")
    rows = []
    for t in tables:
        dirs = rule if rule is not None else beamer_dirs(t)
        rows.append({"frontier": [int(x) for x in t.frontier],
                     names[0] + "_us": [round(x * 1e-3, 1) for x in t.t_td],
                     names[1] + "_us": [round(x * 1e-3, 1) for x in t.t_bu],
                     "rule": dirs, "rule_us": round(t.cost_ns(dirs) * 1e-3, 1),
                     "best_us": round(t.optimal_ns() * 1e-3, 1)})
    r = regret(tables, (lambda t: rule) if rule is not None else beamer_dirs)
    out.update({"kind": "batched (64 roots)" if args.batched else f"single-source ({args.roots} roots)",
                "tables": rows if args.batched else rows[:4], "rule_regret": r})
    print(json.dumps(out))
    g.close()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    h = sub.add_parser("headroom", help="per-level costs of both directions against the rule")
    h.add_argument("--scale", type=int, default=24)
    h.add_argument("--seed", type=int, default=24)
    h.add_argument("--root-seed", type=int, default=0)
    h.add_argument("--roots", type=int, default=16)
    h.add_argument("--repeats", type=int, default=3)
    h.add_argument("--batched", action="store_true")
    t = sub.add_parser("train")
    t.add_argument("--graphs", type=int, default=200)
    t.add_argument("--roots", type=int, default=8)
    t.add_argument("--epochs", type=int, default=3000)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--out", default=None)
    t.add_argument("--tables-out", default=None)
    t.add_argument("--batched", action="store_true",
                   help="train the push/pull policy of the 64-root batched traversal")
    args = ap.parse_args(argv)
    log = lambda s: print(f"[policy {time.strftime('%H:%M:%S')}] {s}", flush=True)  # noqa: E731
    if args.cmd == "headroom":
        return headroom(args, log)
    if args.batched:
        args.out = args.out or BATCHED_PATH
        return train_batched(args, log)
    args.out = args.out or DEFAULT_PATH
    specs = training_graph_specs(args.graphs)
    t0 = time.time()
    tables = collect(specs, args.roots, log=log)
    log(f"{len(tables)} level tables in {time.time() - t0:.1f} s")
    policy, rb, rl = train_policy(tables, beamer_dirs, args, log)
    policy.info.update({"kind": "single-source", "graphs": args.graphs,
                        "roots_per_graph": args.roots,
                        "distribution": "RMAT scales 16-22, A~U[0.45,0.65], D=0.05, "
                                        "B=C=(1-A-D)/2, ef 16; 5 RMAT graphs at scales 23-24; "
                                        "6 grids 512^2-2048^2 (1% of edges deleted, 2 roots "
                                        "each); hub numbering"})
    policy.save(args.out)
    log(f"saved {args.out}: beamer regret {rb['regret_frac']:.3%}, learned {rl['regret_frac']:.3%}")
    if args.tables_out:
        np.savez_compressed(args.tables_out, **{
            f"{i}.{k}": getattr(tb, k) for i, tb in enumerate(tables)
            for k in ("frontier", "frontier_edges", "unexplored", "found", "t_td", "t_bu")})
    return 0


if __name__ == "__main__":
    sys.exit(main())
