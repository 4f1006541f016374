"""The learned direction policy.

CPU: the float64 oracle's analytic gradient agrees with finite differences
(this pins the oracle; the reference has no learned component to compare
with).  GPU: the hand-written forward / backward / Adam kernels agree with the
oracle; a BFS under the learned policy returns exactly the plain BFS's
depths; and the trained network's regret on held-out graphs is below the
Beamer rule's.
"""
import os

import numpy as np
import pytest

from oracle import policy_oracle as PO

# fp32 device arithmetic against the float64 oracle
RTOL = 2e-3
ATOL = 2e-5


def _problem(n=700, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, 8))
    y = (x[:, 0] + 0.5 * x[:, 2] - x[:, 6] > 0).astype(np.int64)
    w = rng.uniform(0.1, 3.0, n)
    theta = PO.init_params(seed + 1)
    return theta, x, y, w


def test_oracle_gradient_matches_finite_differences():
    theta, x, y, w = _problem(60, 3)
    _, g = PO.loss_grad(theta, x, y, w)
    idx = list(range(0, PO.NUM_PARAMS, 37)) + [PO.NUM_PARAMS - 1, PO.NUM_PARAMS - 2]
    fd = PO.finite_difference(theta, x, y, w, 1e-6, idx)
    for i in idx:
        assert abs(fd[i] - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), i


def test_oracle_adam_decreases_loss():
    theta, x, y, w = _problem(200, 4)
    _, losses = PO.adam(theta, lambda t: PO.loss_grad(t, x, y, w), 200, lr=1e-2)
    assert losses[-1] < 0.5 * losses[0]


@pytest.mark.gpu
def test_device_forward_matches_oracle():
    bd = pytest.importorskip("beedrill_b200")
    theta, x, y, w = _problem()
    z_ref, _ = PO.forward(theta, x)
    z = bd.policy_forward(theta.astype(np.float32), x.astype(np.float32))
    np.testing.assert_allclose(z, z_ref, rtol=RTOL, atol=1e-4)


@pytest.mark.gpu
def test_device_gradient_matches_oracle():
    bd = pytest.importorskip("beedrill_b200")
    theta, x, y, w = _problem()
    loss_ref, g_ref = PO.loss_grad(theta, x, y, w)
    loss, g = bd.policy_loss_grad(theta.astype(np.float32), x.astype(np.float32), y, w)
    assert abs(loss - loss_ref) <= RTOL * abs(loss_ref)
    scale = np.abs(g_ref).max()
    np.testing.assert_allclose(g, g_ref, rtol=RTOL, atol=ATOL * max(scale, 1.0))


@pytest.mark.gpu
def test_device_adam_tracks_oracle():
    bd = pytest.importorskip("beedrill_b200")
    theta, x, y, w = _problem(300, 5)
    steps, lr = 40, 5e-3
    ref_theta, ref_losses = PO.adam(theta, lambda t: PO.loss_grad(t, x, y, w), steps, lr=lr)
    p = theta.astype(np.float32).copy()
    hist = bd.policy_train(p, x.astype(np.float32), y, w, steps, lr, 0.0)
    np.testing.assert_allclose(hist, ref_losses, rtol=1e-2, atol=1e-4)
    np.testing.assert_allclose(p, ref_theta, rtol=5e-2, atol=5e-3)


@pytest.mark.gpu
def test_learned_policy_does_not_change_results():
    bd = pytest.importorskip("beedrill_b200")
    from oracle import oracle as O
    g = bd.Graph.rmat(15, seed=31)
    off, adj = g.csr()
    bfs = bd.HybridBFS(g, alg="learned")
    # an arbitrary (untrained) network: decisions change, results must not
    theta = PO.init_params(9).astype(np.float32)
    bfs.set_policy(theta, np.zeros(8, np.float32), np.full(8, 0.3, np.float32), 0.0)
    for root in g.pick_roots(2, 4):
        root = int(root)
        bfs.clear()
        bfs.run(root)
        assert np.array_equal(bfs.depths(), O.bfs_depth(off, adj, root))
        assert O.check(off, adj, root, bfs.parents())


def _held_out_specs(count, seed):
    """Graphs from the training distribution (scales 16-20, A in
    [0.45, 0.65]) with seeds the trainer never used."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        a = float(rng.uniform(0.45, 0.65))
        d = 0.05
        out.append((16 + k % 5, a, (1 - a - d) / 2, d, 900_000 + seed * 100 + k))
    return out


@pytest.mark.gpu
def test_trained_policy_vs_beamer_on_held_out_graphs():
    """What the trained network gains over the rule it replaces, on graphs
    it was not trained on: the total time of its decisions, priced with the
    measured per-level costs of both directions, against Beamer's -- for the
    network's own decisions (with the trusted range and margin they favour)
    and for the policy as shipped, which the trainer may have switched off
    when the network's inference cost inside the kernel outweighs what its
    decisions save."""
    bd = pytest.importorskip("beedrill_b200")
    from beedrill_b200 import policy as P
    if not os.path.exists(P.DEFAULT_PATH):
        pytest.skip("no trained policy committed")
    pol = P.Policy.load()
    tables = []
    for scale, a, b, d, seed in _held_out_specs(10, 1):
        g = bd.Graph.rmat(scale, 16, a, b, b, d, seed, order=bd.ORDER_HUB)
        tables += P.measure_tables(g, g.pick_roots(seed, 2), repeats=2, with_beamer=False)
        g.close()
    rb = P.regret(tables, P.beamer_dirs)
    rl = P.regret(tables, lambda t: P.policy_dirs(pol, t))
    print(f"held-out regret: Beamer {rb['regret_frac']:.2%}, shipped policy {rl['regret_frac']:.2%}")
    assert rl["cost_ms"] <= rb["cost_ms"] * 1.005, (rl, rb)
    net = P.decisions_policy(pol)
    if net is not None:
        rn = P.regret(tables, lambda t: P.policy_dirs(net, t))
        print(f"held-out regret of the network's decisions: {rn['regret_frac']:.2%}")
        assert rn["cost_ms"] <= rb["cost_ms"] * 1.005, (rn, rb)


@pytest.mark.gpu
def test_trained_policies_at_scale24_held_out():
    """The evaluation case: RMAT scale 24 (A=.57 B=C=.19 D=.05) with a seed
    no training graph used, beyond the training scales (16-22); the
    single-source policy against Beamer's alpha=15/beta=18 switch over 16
    roots, the batched policy against its rule over one 64-root batch."""
    bd = pytest.importorskip("beedrill_b200")
    from beedrill_b200 import policy as P
    if not (os.path.exists(P.DEFAULT_PATH) and os.path.exists(P.BATCHED_PATH)):
        pytest.skip("no trained policies committed")
    g = bd.Graph.rmat(24, 16, seed=2424, order=bd.ORDER_HUB)
    tables = P.measure_tables(g, g.pick_roots(7, 16), repeats=2, with_beamer=False)
    pol = P.Policy.load()
    rb = P.regret(tables, P.beamer_dirs)
    rl = P.regret(tables, lambda t: P.policy_dirs(pol, t))
    print(f"scale 24 regret: Beamer {rb['regret_frac']:.2%}, learned {rl['regret_frac']:.2%}, "
          f"consulted at {_consulted(pol, tables, P.beamer_dirs)} of "
          f"{sum(t.levels for t in tables)} levels")
    assert rl["cost_ms"] <= rb["cost_ms"] * 1.005, (rl, rb)
    tab = P.measure_tables_batched(g, g.pick_roots(8, 64), repeats=2)
    bpol = P.Policy.load(P.BATCHED_PATH)
    rule = P.regret([tab], P.alpha_dirs)
    rl = P.regret([tab], lambda t: P.policy_dirs(bpol, t, rule=P.alpha_dirs(t)))
    print(f"scale 24 batched regret: rule {rule['regret_frac']:.2%}, learned {rl['regret_frac']:.2%}, "
          f"consulted at {_consulted(bpol, [tab], P.alpha_dirs)} of {tab.levels} levels")
    assert rl["cost_ms"] <= rule["cost_ms"] * 1.005, (rl, rule)


def _consulted(pol, tables, rule_fn):
    """Levels at which the policy's trusted range (the band on feature 0
    included) lets the network decide, over the rule's path."""
    from beedrill_b200 import policy as P
    count = 0
    for t in tables:
        prev_dir, prev_ns = 0, 0.0
        for lv, d in enumerate(P.policy_dirs(pol, t, rule=rule_fn(t))):
            if pol.trusts(t.features(lv, prev_dir, prev_ns)):
                count += 1
            prev_dir = 1 if d == "B" else 0
            prev_ns = t.t_bu[lv] if d == "B" else t.t_td[lv]
    return count


@pytest.mark.gpu
def test_trained_policies_on_a_held_out_grid():
    """The high-diameter contrast: a 1024 x 1024 grid with 1 % of its edges
    deleted (a seed no training grid used).  Grids are in the training set,
    and the features are scale-free, so the network's range covers their
    thousands of small levels; its decisions must cost no more than the
    rule's (single-source against Beamer, batched against its rule)."""
    bd = pytest.importorskip("beedrill_b200")
    from beedrill_b200 import policy as P
    if not (os.path.exists(P.DEFAULT_PATH) and os.path.exists(P.BATCHED_PATH)):
        pytest.skip("no trained policies committed")
    g = bd.Graph.grid(1024, 1024, 0.01, 4242, order=bd.ORDER_HUB)
    tables = P.measure_tables(g, g.pick_roots(3, 2), repeats=2, with_beamer=False)
    pol = P.Policy.load()
    net = P.decisions_policy(pol) or pol
    rb = P.regret(tables, P.beamer_dirs)
    rn = P.regret(tables, lambda t: P.policy_dirs(net, t))
    print(f"grid regret: Beamer {rb['regret_frac']:.2%}, network {rn['regret_frac']:.2%}, "
          f"consulted at {_consulted(net, tables, P.beamer_dirs)} of "
          f"{sum(t.levels for t in tables)} levels")
    assert rn["cost_ms"] <= rb["cost_ms"] * 1.005, (rn, rb)
    tab = P.measure_tables_batched(g, g.pick_roots(4, 64), repeats=2)
    bpol = P.Policy.load(P.BATCHED_PATH)
    rule = P.regret([tab], P.alpha_dirs)
    rl = P.regret([tab], lambda t: P.policy_dirs(bpol, t, rule=P.alpha_dirs(t)))
    print(f"grid batched regret: rule {rule['regret_frac']:.2%}, learned {rl['regret_frac']:.2%}, "
          f"consulted at {_consulted(bpol, [tab], P.alpha_dirs)} of {tab.levels} levels")
    assert rl["cost_ms"] <= rule["cost_ms"] * 1.005, (rl, rule)
    g.close()


@pytest.mark.gpu
def test_trained_batched_policy_vs_rule_on_held_out_graphs():
    bd = pytest.importorskip("beedrill_b200")
    from beedrill_b200 import policy as P
    if not os.path.exists(P.BATCHED_PATH):
        pytest.skip("no trained batched policy committed")
    pol = P.Policy.load(P.BATCHED_PATH)
    tables = []
    for scale, a, b, d, seed in _held_out_specs(5, 2):
        g = bd.Graph.rmat(scale, 16, a, b, b, d, seed, order=bd.ORDER_HUB)
        tables.append(P.measure_tables_batched(g, g.pick_roots(seed, 64), repeats=2))
        g.close()
    rule = P.regret(tables, P.alpha_dirs)
    rl = P.regret(tables, lambda t: P.policy_dirs(pol, t, rule=P.alpha_dirs(t)))
    print(f"held-out regret: rule {rule['regret_frac']:.2%}, learned {rl['regret_frac']:.2%}")
    assert rl["cost_ms"] <= rule["cost_ms"] * 1.005, (rl, rule)


def _decisions_agree(pol, steps, m2):
    """Rebuilds the features each step's decision saw from the run's own
    step records and checks every confident, trusted decision against the
    host float32 forward pass."""
    from beedrill_b200 import policy as P
    checked = 0
    for s, st in enumerate(steps):
        prev_dir = steps[s - 1]["dir"] if s else 0
        prev_ns = steps[s - 1]["ns"] if s else 0
        raw = P.raw_features(st["frontier"], st["frontier_edges"], st["unexplored_edges"],
                             st["level"], m2[0], m2[1], prev_dir, prev_ns)
        gap = float(np.diff(pol.logits(raw)[0])[0])
        if not pol.trusts(raw) or abs(abs(gap) - pol.margin) < 1e-3 or abs(gap) < pol.margin:
            continue
        assert st["dir"] == (1 if gap > 0 else 0), (s, gap, st)
        checked += 1
    return checked


@pytest.mark.gpu
def test_in_kernel_decisions_follow_the_network():
    """The traversal kernels' own evaluation of the network (transposed
    weights in shared memory, shuffles) decides as the host forward pass
    does, single-source and batched."""
    bd = pytest.importorskip("beedrill_b200")
    from beedrill_b200 import policy as P
    rng = np.random.default_rng(11)
    pol = P.Policy(PO.init_params(21).astype(np.float32), np.array(
        [-5, -8, -1, 1.5, 4, 0.5, 3, 5], np.float32), np.full(8, 0.25, np.float32), 0.05)
    checked = 0
    for scale in (14, 16, 17):
        g = bd.Graph.rmat(scale, 16, seed=int(rng.integers(1 << 30)), order=bd.ORDER_DEGREE)
        n, m = g.num_vertices(), g.num_edges()
        bfs = bd.HybridBFS(g, alg="learned")
        pol.install(bfs)
        for root in g.pick_roots(3, 4):
            bfs.clear()
            bfs.run(int(root))
            checked += _decisions_agree(pol, bfs.steps(), (n, m))
        ms = bd.BatchedBFS(g, 64)
        pol.install(ms)
        ms.run(g.pick_roots(4, 64))
        checked += _decisions_agree(pol, ms.steps(), (n, m))
        g.close()
    assert checked > 20
