"""Host-side logic of the learned policy and the tuning file, on CPU: the
per-scale tuning lookup, the batched rule's mirror of the kernel's, the
trusted range that never extends past the largest training graph, and the
trainer's choices (trusted range by extrapolation, margin or no network at
all priced with the inference cost) on synthetic level tables, with a CPU
stand-in for the device trainer."""
import json
import types

import numpy as np
import pytest

import beedrill_b200 as bd
from beedrill_b200 import policy as P
from oracle import policy_oracle as PO


def test_tuned_options_pick_the_nearest_scale(tmp_path, monkeypatch):
    f = tmp_path / "t.json"
    f.write_text(json.dumps({
        "single": {"block_size": 999}, "batched": {"alpha": 9},
        "by_scale": {"20": {"single": {"block_size": 256}, "batched": {"alpha": 4}},
                     "24": {"single": {"block_size": 512}, "batched": {"alpha": 2}}}}))
    monkeypatch.setattr(bd, "TUNING_PATH", str(f))
    assert bd.tuned_options("batched", 1 << 20)["alpha"] == 4
    assert bd.tuned_options("batched", 1 << 23)["alpha"] == 2   # 23 is nearer 24
    assert bd.tuned_options("batched", 1 << 22)["alpha"] == 2   # a tie goes to the larger
    assert bd.tuned_options("single", 1 << 30)["block_size"] == 512
    assert bd.tuned_options("batched")["alpha"] == 9            # no size: the default entry
    monkeypatch.setattr(bd, "TUNING_PATH", str(tmp_path / "missing.json"))
    assert bd.tuned_options("batched", 1 << 20) == {}


def _table(n, m, frontier, fedges, unexplored, t_td, t_bu, scale=16, seed=0):
    k = len(frontier)
    return P.LevelTable(n=n, m=m, frontier=np.array(frontier, np.int64),
                        frontier_edges=np.array(fedges, np.int64),
                        unexplored=np.array(unexplored, np.int64),
                        found=np.zeros(k, np.int64), t_td=np.array(t_td, np.float64),
                        t_bu=np.array(t_bu, np.float64), meta={"scale": scale, "seed": seed})


def test_batched_rule_mirror():
    n = 1 << 16
    t = _table(n, 10 * n, [10, 5000, 50, 40], [100, 900000, 400, 300],
               [2000000, 1000000, 100, 100], [1] * 4, [1] * 4)
    # pull needs frontier degree sum x alpha > unexplored AND frontier >= n/1024
    dirs = P.alpha_dirs(t, alpha=4)
    assert dirs[0] == "T"          # 100 * 4 < 2e6
    assert dirs[1] == "B"          # 9e5 * 4 > 1e6, 5000 >= 64
    assert dirs[2] == "T"          # 400 * 4 > 100 but 50 < n / 1024
    assert dirs[3] == "T"


def test_trusted_range_is_the_band_on_feature_0_and_scale_free():
    """The features are differences of logarithms, so a graph larger than
    any training graph is not outside the trusted range by its size; the
    range of feature 0 is cut to the band where the rule's choice was not
    the faster one, and outside it the network is never consulted."""
    rng = np.random.default_rng(0)
    X = rng.normal(0, 1, (200, 8)).astype(np.float32)
    pol = P.Policy(np.zeros(1410, np.float32), np.zeros(8, np.float32), np.ones(8, np.float32))
    pol.extremes = (X.min(0), X.max(0), X.std(0))
    pol.band = (-0.5, 0.25)
    P.set_widen(pol, 3.0)
    assert pol.lo[0] == np.float32(-0.5) and pol.hi[0] == np.float32(0.25)
    assert pol.hi[4] > X[:, 4].max() and pol.lo[4] < X[:, 4].min()
    raw = np.zeros(8, np.float32)
    assert pol.trusts(raw)
    raw[0] = 0.5
    assert not pol.trusts(raw)
    # the same frontier shares at scale 16 and at scale 26 give the same
    # size-free features (0, 1, 2, 7) and the same average-degree feature
    a = P.raw_features(1 << 10, 1 << 14, 1 << 20, 3, 1 << 16, 1 << 20, 0, 0)
    b = P.raw_features(1 << 20, 1 << 24, 1 << 30, 3, 1 << 26, 1 << 30, 0, 0)
    assert np.allclose(a[[0, 1, 2, 4, 7]], b[[0, 1, 2, 4, 7]], atol=2e-3)


def test_disagreement_band():
    """The band is the feature-0 range of the levels where the faster
    direction is not the rule's, padded; None when the rule is always
    right."""
    t = _table(1 << 16, 1 << 20, np.array([1, 100, 5000, 200]), np.array([16, 2000, 80000, 3000]),
               np.array([2 << 20, 2 << 20, 2 << 20, 2 << 19]), np.array([1.0, 5.0, 90.0, 2.0]),
               np.array([50.0, 50.0, 10.0, 1.0]))
    assert P.disagreement_band([t], lambda tab: "TTBB") is None
    lo, hi = P.disagreement_band([t], lambda tab: "TTTB")
    f0 = t.features(2, 0, 0.0)[0]
    assert lo == pytest.approx(f0 - P.BAND_PAD) and hi == pytest.approx(f0 + P.BAND_PAD)


def _fake_train(params, Xs, y, w, epochs, lr, wd):
    th = params.astype(np.float64)
    m = np.zeros_like(th)
    v = np.zeros_like(th)
    hist = []
    for t in range(1, epochs + 1):
        loss, g = PO.loss_grad(th, Xs, y, w)
        hist.append(loss)
        g = g + wd * th
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        th = th - lr * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    params[:] = th.astype(np.float32)
    return np.array(hist, np.float32)


def _synthetic_tables():
    """Levels where bottom-up wins when the frontier holds over 5 % of the
    edges and top-down otherwise; the rule (Beamer) switches too late."""
    rng = np.random.default_rng(3)
    tables = []
    for k in range(60):
        scale = 16 + k % 4
        n = 1 << scale
        m = 16 * n
        fe = np.array([10, 2000, int(0.08 * 2 * m), int(0.2 * 2 * m), 3000, 20]) * \
            rng.uniform(0.8, 1.2)
        fr = fe / 16
        un = 2 * m - np.cumsum(fe)
        td = fe * 1.0 + 50
        bu = np.full(6, 0.06 * 2 * m) + 50
        tables.append(_table(n, m, fr.astype(np.int64), fe.astype(np.int64),
                             np.maximum(un, 1).astype(np.int64), td, bu, scale=scale,
                             seed=10_000 + k))
    return tables


@pytest.mark.parametrize("overhead, expect_off", [((0.0, 0.0), False), ((1e9, 1e9), True)])
def test_trainer_prices_the_network_inference(monkeypatch, overhead, expect_off):
    monkeypatch.setattr(bd, "policy_train", _fake_train)
    monkeypatch.setattr(P, "inference_overhead", lambda spec, pol, batched: overhead)
    args = types.SimpleNamespace(epochs=300, lr=1e-2)
    pol, rb, rl = P.train_policy(_synthetic_tables(), P.beamer_dirs, args, lambda s: None)
    if expect_off:
        # inference dearer than any saving: no network, the rule decides
        assert pol.margin == P.OFF and rl["cost_ms"] == rb["cost_ms"]
    else:
        assert pol.margin != P.OFF
        assert rl["cost_ms"] <= rb["cost_ms"]
    assert "decisions_only" in pol.info
