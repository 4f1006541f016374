"""CPU float64 restatement of the direction-policy MLP (8-32-32-2, ReLU,
softmax cross-entropy weighted per sample).

TEST INFRASTRUCTURE ONLY: the checker for the device forward / backward /
training kernels in beedrill_b200/csrc/bd_policy.cu.  The reference has no
learned component; this oracle is pinned by finite differences instead
(tests/test_policy_oracle.py).

Parameter vector layout (fp32 on the device, 1410 values):
    w1[32][8], b1[32], w2[32][32], b2[32], w3[2][32], b3[2]
"""
from __future__ import annotations

import numpy as np

IN, H, OUT = 8, 32, 2
SHAPES = [("w1", (H, IN)), ("b1", (H,)), ("w2", (H, H)), ("b2", (H,)), ("w3", (OUT, H)),
          ("b3", (OUT,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    theta = np.asarray(theta, np.float64)
    out, pos = {}, 0
    for name, shape in SHAPES:
        size = int(np.prod(shape))
        out[name] = theta[pos:pos + size].reshape(shape)
        pos += size
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.asarray(parts[name], np.float64).ravel() for name, _ in SHAPES])


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation (used by the trainer's host side as well)."""
    rng = np.random.default_rng(seed)
    parts = {
        "w1": rng.normal(0, np.sqrt(2.0 / IN), (H, IN)),
        "b1": np.zeros(H),
        "w2": rng.normal(0, np.sqrt(2.0 / H), (H, H)),
        "b2": np.zeros(H),
        "w3": rng.normal(0, np.sqrt(1.0 / H), (OUT, H)),
        "b3": np.zeros(OUT),
    }
    return pack(parts)


def forward(theta, x):
    p = unpack(theta)
    x = np.asarray(x, np.float64)
    a1 = x @ p["w1"].T + p["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ p["w2"].T + p["b2"]
    h2 = np.maximum(a2, 0)
    z = h2 @ p["w3"].T + p["b3"]
    return z, (x, h1, h2)


def loss_grad(theta, x, label, weight):
    """Weighted mean cross-entropy sum_i w_i CE_i / sum_i w_i and its
    gradient with respect to theta."""
    p = unpack(theta)
    label = np.asarray(label, np.int64)
    w = np.asarray(weight, np.float64)
    z, (x, h1, h2) = forward(theta, x)
    zmax = z.max(axis=1, keepdims=True)
    e = np.exp(z - zmax)
    prob = e / e.sum(axis=1, keepdims=True)
    n = len(label)
    wsum = w.sum()
    ce = -np.log(prob[np.arange(n), label])
    loss = float((w * ce).sum() / wsum)
    dz = prob.copy()
    dz[np.arange(n), label] -= 1.0
    dz *= (w / wsum)[:, None]
    g = {}
    g["w3"] = dz.T @ h2
    g["b3"] = dz.sum(0)
    dh2 = (dz @ p["w3"]) * (h2 > 0)
    g["w2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ p["w2"]) * (h1 > 0)
    g["w1"] = dh1.T @ x
    g["b1"] = dh1.sum(0)
    return loss, pack(g)


def finite_difference(theta, x, label, weight, eps=1e-6, indices=None):
    theta = np.asarray(theta, np.float64)
    idx = range(len(theta)) if indices is None else indices
    out = {}
    for i in idx:
        tp = theta.copy()
        tm = theta.copy()
        tp[i] += eps
        tm[i] -= eps
        out[i] = (loss_grad(tp, x, label, weight)[0] - loss_grad(tm, x, label, weight)[0]) / (2 * eps)
    return out


def adam(theta, grads_fn, steps, lr=1e-2, b1=0.9, b2=0.999, eps=1e-8, weight_decay=0.0):
    """Reference Adam loop (Kingma & Ba 2015) for checking the device
    trainer over a few steps."""
    theta = np.asarray(theta, np.float64).copy()
    m = np.zeros_like(theta)
    v = np.zeros_like(theta)
    losses = []
    for t in range(1, steps + 1):
        loss, g = grads_fn(theta)
        g = g + weight_decay * theta
        losses.append(loss)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        mh = m / (1 - b1 ** t)
        vh = v / (1 - b2 ** t)
        theta -= lr * mh / (np.sqrt(vh) + eps)
    return theta, losses
