"""CPU oracle of the learned chemistry seed's network (NumPy, FP64).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the library's tensor-core
forward, backward and prediction kernels; the product never imports it.

The network (no counterpart in the reference): input x[8] (normalised
log T, log p, Y[5], log dt), three hidden layers of 64 units with the
tanh-form GELU (Hendrycks & Gimpel 2016), output z[6].  Parameters are one
FP32 vector in the layout W1[64][8] b1[64] W2[64][64] b2 W3[64][64] b3
W4[6][64] b4[6].

``mirror=True`` rounds to BF16 (round to nearest even) exactly where the
library's kernels feed the tensor cores -- the inputs, the weights, every
hidden activation and every back-propagated output gradient -- and keeps
everything else in FP64; the library accumulates in FP32, so the two agree
to FP32 rounding plus the rare BF16 tie that falls the other way.
``mirror=False`` is the plain FP64 network, whose gradient is checked against
finite differences.
"""
from __future__ import annotations

import numpy as np

NPARAM = 9286
NNORM = 30
_SHAPES = [("W1", (64, 8)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
           ("W3", (64, 64)), ("b3", (64,)), ("W4", (6, 64)), ("b4", (6,))]


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    assert p.size == NPARAM
    out, o = {}, 0
    for name, shp in _SHAPES:
        n = int(np.prod(shp))
        out[name] = p[o:o + n].reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in _SHAPES])


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    r = ((u + rounding) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    c = np.sqrt(2.0 / np.pi)
    return 0.5 * x * (1.0 + np.tanh(c * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    c = np.sqrt(2.0 / np.pi)
    th = np.tanh(c * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * c * (1.0 + 3.0 * 0.044715 * x * x)


def forward(params, X, mirror=True):
    """Network output z[n][6] and the cached intermediates."""
    r = bf16 if mirror else (lambda a: np.asarray(a, dtype=np.float64))
    P = unpack(params)
    W = {k: r(P[k]) for k in ("W1", "W2", "W3", "W4")}
    h0 = r(np.asarray(X, dtype=np.float32) if mirror else X)
    z1 = h0 @ W["W1"].T + P["b1"]
    h1 = r(gelu(z1))
    z2 = h1 @ W["W2"].T + P["b2"]
    h2 = r(gelu(z2))
    z3 = h2 @ W["W3"].T + P["b3"]
    h3 = r(gelu(z3))
    z4 = h3 @ W["W4"].T + P["b4"]
    return z4, (W, h0, z1, h1, z2, h2, z3, h3)


def loss_grad(params, X, Y, mirror=True):
    """Mean squared error over the n x 6 outputs and its gradient (packed)."""
    r = bf16 if mirror else (lambda a: np.asarray(a, dtype=np.float64))
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    n = X.shape[0]
    z4, (W, h0, z1, h1, z2, h2, z3, h3) = forward(params, X, mirror)
    diff = z4 - Y
    loss = float(np.sum(diff * diff) / (n * 6))
    d4 = r(2.0 * diff / (n * 6))
    d3 = r((d4 @ W["W4"]) * gelu_grad(z3))
    d2 = r((d3 @ W["W3"]) * gelu_grad(z2))
    d1 = r((d2 @ W["W2"]) * gelu_grad(z1))
    g = {"W4": d4.T @ h3, "b4": d4.sum(0), "W3": d3.T @ h2, "b3": d3.sum(0),
         "W2": d2.T @ h1, "b2": d2.sum(0), "W1": d1.T @ h0, "b1": d1.sum(0)}
    return loss, pack(g)


def init_params(seed):
    """Uniform +-1/sqrt(fan_in) weights and biases (as the library's trainer)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shp in _SHAPES:
        fan_in = {"1": 8}.get(name[1], 64)
        d[name] = rng.uniform(-1.0, 1.0, shp) / np.sqrt(fan_in)
    return pack(d).astype(np.float32)


def predict(params, norm, rows, mirror=True):
    """(dY[5], dT) for rows (T, p, Y[5], dt), as the library's predict kernel."""
    norm = np.asarray(norm, dtype=np.float64)
    rows = np.asarray(rows, dtype=np.float64)
    f = np.column_stack([np.log(rows[:, 0]), np.log(rows[:, 1]), rows[:, 2:7],
                         np.log(rows[:, 7])])
    x = ((f - norm[0:8]) / norm[8:16]).astype(np.float32)
    z, _ = forward(params, x, mirror)
    z = z.astype(np.float32).astype(np.float64) * norm[22:28] + norm[16:22]
    s = np.concatenate([np.full(5, norm[28]), [norm[29]]])
    return s * np.sinh(z)
