"""Oracle for the learned insertion scheduler's network: a NumPy restatement.

Test infrastructure only (imported by tests/); the wtet_b200 product never
uses it.  The reference has no learned scheduler (its vote is the circumsphere
determinant, src/shaders/vote.wgsl:401-494), so this oracle restates the
network the B200 build adds: 12 -> 64 -> 64 -> 64 -> 1 with ReLU, mean binary
cross-entropy on the logit, flat FP32 parameter layout
W1[64][12] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4.

* ``loss_grad``: forward + backward in float64 (the checker for the device
  training kernels' gradients); pinned here by central finite differences in
  the tests.
* ``score_bf16``: the inference the vote kernel runs -- weights and
  activations rounded to BF16 (round to nearest even), sums in float32.
"""
from __future__ import annotations

import numpy as np

IN = 12
H = 64
SIZES = (("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
         ("W4", (H,)), ("b4", (1,)))
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(params):
    p = np.asarray(params)
    assert p.shape == (NUM_PARAMS,), p.shape
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SIZES])


def forward(X, params):
    """Logits of the FP32 network, evaluated in float64."""
    P = {k: v.astype(np.float64) for k, v in unpack(params).items()}
    h = np.asarray(X, np.float64)
    for W, b in (("W1", "b1"), ("W2", "b2"), ("W3", "b3")):
        h = np.maximum(h @ P[W].T + P[b], 0)
    return h @ P["W4"] + P["b4"][0]


def loss_grad(X, y, params):
    """Mean BCE-with-logits and its gradient (flat, float64)."""
    P = {k: v.astype(np.float64) for k, v in unpack(params).items()}
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    n = X.shape[0]
    z1 = X @ P["W1"].T + P["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ P["W2"].T + P["b2"]
    h2 = np.maximum(z2, 0)
    z3 = h2 @ P["W3"].T + P["b3"]
    h3 = np.maximum(z3, 0)
    logit = h3 @ P["W4"] + P["b4"][0]
    loss = np.mean(np.maximum(logit, 0) - logit * y + np.log1p(np.exp(-np.abs(logit))))
    dl = (1.0 / (1.0 + np.exp(-logit)) - y) / n
    g = {}
    g["W4"] = h3.T @ dl
    g["b4"] = np.array([dl.sum()])
    d3 = np.outer(dl, P["W4"]) * (z3 > 0)
    g["W3"] = d3.T @ h2
    g["b3"] = d3.sum(0)
    d2 = (d3 @ P["W3"]) * (z2 > 0)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ P["W2"]) * (z1 > 0)
    g["W1"] = d1.T @ X
    g["b1"] = d1.sum(0)
    return float(loss), pack(g)


def bf16(x):
    """Rounds float32 values to the nearest BF16 value (ties to even)."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def score_bf16(X, params):
    """Logits as the fused BF16 inference computes them (up to summation order)."""
    P = {k: v.astype(np.float32) for k, v in unpack(np.asarray(params, np.float32)).items()}
    h = bf16(np.asarray(X, np.float32))
    for W, b in (("W1", "b1"), ("W2", "b2"), ("W3", "b3")):
        h = bf16(np.maximum(h @ bf16(P[W]).T + P[b], 0).astype(np.float32))
    return (h @ bf16(P["W4"]) + P["b4"][0]).astype(np.float32)
