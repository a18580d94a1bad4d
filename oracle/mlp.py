"""CPU oracle of the learned Newton predictor's network (test infrastructure only).

The reference has no learned part: it starts each implicit stage from a linear extrapolation
(core/solver.py:420, :432, :435).  The network this library adds is new, so this oracle restates the
library's own definition (dac_vtsa_b200/csrc/dv_mlp.cu) in numpy to check its tensor-core kernels:
the forward pass and the gradient of the mean squared error, with BF16 rounding at the same points as
the device (inputs, weights, every activation and every back-propagated gradient are BF16 values; sums
run in float64 here and in FP32 on the tensor cores).  It is pinned by its own finite-difference check
in float64 (tests/test_mlp_oracle.py), not by any reference output ("parity unpinned" in the sense of
the reference: there is nothing in the reference to compare with).

Parameter vector (fp32): W1 [NH x NIN], b1 [NH], W2 [NH x NH], b2, W3 [NH x NH], b3, W4 [NOUT x NH], b4.
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT, NOUT_USED = 112, 128, 16, 6
SIZES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
         ("W4", (NOUT, NH)), ("b4", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float32 (finite inputs)."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (r.astype(np.uint32) << 16).view(np.float32).reshape(a.shape)


def unpack(P):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(P[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float32).ravel() for name, _ in SIZES])


def forward(P, X, rounding=True):
    """Outputs [rows, NOUT] and the hidden activations (as the device holds them)."""
    w = unpack(P)
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    x = np.asarray(r(X), dtype=np.float64)
    Wb = {k: np.asarray(r(w[k]), dtype=np.float64) for k in ("W1", "W2", "W3", "W4")}
    h1 = np.asarray(r(np.tanh(x @ Wb["W1"].T + w["b1"])), dtype=np.float64)
    h2 = np.asarray(r(np.tanh(h1 @ Wb["W2"].T + w["b2"])), dtype=np.float64)
    h3 = np.asarray(r(np.tanh(h2 @ Wb["W3"].T + w["b3"])), dtype=np.float64)
    o = h3 @ Wb["W4"].T + w["b4"]
    return o, (x, h1, h2, h3, Wb)


def loss(P, X, T, rounding=True):
    o, _ = forward(P, X, rounding)
    d = o[:, :NOUT_USED] - np.asarray(T, dtype=np.float64)[:, :NOUT_USED]
    return float(np.mean(d * d))


def gradient(P, X, T, rounding=True):
    """(gradient vector [NPARAM], loss) of mean((O - T)^2) over the used outputs, back-propagated with
    the device's BF16 rounding of every gradient that feeds a product."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    o, (x, h1, h2, h3, Wb) = forward(P, X, rounding)
    rows = x.shape[0]
    d = np.zeros_like(o)
    d[:, :NOUT_USED] = o[:, :NOUT_USED] - np.asarray(T, dtype=np.float64)[:, :NOUT_USED]
    L = float(np.mean(d[:, :NOUT_USED] ** 2))
    d4 = np.asarray(r((2.0 / (rows * NOUT_USED)) * d), dtype=np.float64)
    d3 = np.asarray(r((d4 @ Wb["W4"]) * (1.0 - h3 * h3)), dtype=np.float64)
    d2 = np.asarray(r((d3 @ Wb["W3"]) * (1.0 - h2 * h2)), dtype=np.float64)
    d1 = np.asarray(r((d2 @ Wb["W2"]) * (1.0 - h1 * h1)), dtype=np.float64)
    g = {"W1": d1.T @ x, "b1": d1.sum(0), "W2": d2.T @ h1, "b2": d2.sum(0), "W3": d3.T @ h2, "b3": d3.sum(0),
         "W4": d4.T @ h3, "b4": d4.sum(0)}
    return np.concatenate([np.asarray(g[name], dtype=np.float64).ravel() for name, _ in SIZES]), L


def init_params(seed=0, scale_out=0.0):
    """Random hidden layers (uniform +-1/sqrt(fan_in)); the output layer scaled by scale_out."""
    rng = np.random.default_rng(seed)
    d = {}
    fan = {"W1": 97, "W2": NH, "W3": NH, "W4": NH}
    for name, shape in SIZES:
        if name.startswith("W"):
            a = 1.0 / np.sqrt(fan[name])
            d[name] = rng.uniform(-a, a, size=shape) * (scale_out if name == "W4" else 1.0)
        else:
            d[name] = rng.uniform(-0.1, 0.1, size=shape)
    return pack(d)
