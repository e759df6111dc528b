"""CPU restatement of the learned SGS closure -- TEST INFRASTRUCTURE ONLY.

Only tests and bench.py's CPU baseline use this module; the product path runs the tensor-core
kernels of fasteddy-model_b200/csrc/engine/fe_mlp.cuh and never calls into here.

The network is the closure's: 11 -> 64 -> 64 -> 64 -> 9, tanh hidden layers, standardised
inputs, outputs tau/rho = out_mu + out_sig * y, loss = mean over samples and the 9 outputs of
the squared standardised error. Parameter layout as fe_mlp_param_count() documents in
include/fasteddy_b200.h (W1[64][16], b1, W2[64][64], b2, W3[64][64], b3, W4[16][64], b4[16]).

Two modes:
  exact=True   FP64 throughout (pinned against central finite differences in the tests);
  exact=False  FP64 arithmetic, but every tensor-core operand rounded to BF16 (round to
               nearest even) exactly where the device rounds it: the standardised inputs, the
               weights, the hidden activations and the backward signals dZ. This is the
               reference the device gradients and predictions are checked against.
"""
from __future__ import annotations

import numpy as np

NIN, NOUT, H, K0, N4 = 11, 9, 64, 16, 16
W1, B1 = 0, 64 * 16
W2 = B1 + 64
B2 = W2 + 64 * 64
W3 = B2 + 64
B3 = W3 + 64 * 64
W4 = B3 + 64
B4 = W4 + 16 * 64
NPARAM = B4 + 16


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even); returned as float64."""
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, np.float64)
    return {
        "W1": p[W1:B1].reshape(64, 16), "b1": p[B1:W2],
        "W2": p[W2:B2].reshape(64, 64), "b2": p[B2:W3],
        "W3": p[W3:B3].reshape(64, 64), "b3": p[B3:W4],
        "W4": p[W4:B4].reshape(16, 64), "b4": p[B4:NPARAM],
    }


def standardise(X: np.ndarray, norm: dict) -> np.ndarray:
    """(x - mu)/sig in float32 as the device computes it, padded to 16 columns."""
    X = np.asarray(X, np.float32)
    z = (X - np.asarray(norm["in_mu"], np.float32)) / np.asarray(norm["in_sig"], np.float32)
    out = np.zeros((X.shape[0], K0), np.float64)
    out[:, :NIN] = z.astype(np.float64)
    return out


def forward(p: np.ndarray, X: np.ndarray, norm: dict, exact: bool = False) -> dict:
    w = unpack(p)
    r = (lambda a: a) if exact else bf16
    x0 = r(standardise(X, norm))
    h1 = r(np.tanh(x0 @ r(w["W1"]).T + w["b1"]))
    h2 = r(np.tanh(h1 @ r(w["W2"]).T + w["b2"]))
    h3 = r(np.tanh(h2 @ r(w["W3"]).T + w["b3"]))
    y = h3 @ r(w["W4"]).T + w["b4"]
    return {"x0": x0, "h1": h1, "h2": h2, "h3": h3, "y": y[:, :NOUT]}


def predict(p: np.ndarray, X: np.ndarray, norm: dict, exact: bool = False) -> np.ndarray:
    """Outputs tau/rho (samples x 9)."""
    y = forward(p, X, norm, exact)["y"]
    return np.asarray(norm["out_mu"], np.float64) + np.asarray(norm["out_sig"], np.float64) * y


def loss_and_grad(p: np.ndarray, X: np.ndarray, T: np.ndarray, norm: dict, exact: bool = False):
    """Loss and gradient (flat, NPARAM) of the mean squared standardised error."""
    w = unpack(p)
    r = (lambda a: a) if exact else bf16
    f = forward(p, X, norm, exact)
    n = X.shape[0]
    t = (np.asarray(T, np.float32) - np.asarray(norm["out_mu"], np.float32)) / np.asarray(norm["out_sig"], np.float32)
    e = f["y"] - t.astype(np.float64)
    loss = float(np.sum(e * e) / (n * NOUT))
    scale = 1.0 / (n * NOUT)
    dz4 = np.zeros((n, N4))
    dz4[:, :NOUT] = r(2.0 * e)
    g = np.zeros(NPARAM)
    g[W4:B4] = (dz4.T @ f["h3"]).ravel() * scale
    g[B4:NPARAM] = dz4.sum(0) * scale
    dz3 = r((dz4 @ r(w["W4"])) * (1.0 - f["h3"] ** 2))
    g[W3:B3] = (dz3.T @ f["h2"]).ravel() * scale
    g[B3:W4] = dz3.sum(0) * scale
    dz2 = r((dz3 @ r(w["W3"])) * (1.0 - f["h2"] ** 2))
    g[W2:B2] = (dz2.T @ f["h1"]).ravel() * scale
    g[B2:W3] = dz2.sum(0) * scale
    dz1 = r((dz2 @ r(w["W2"])) * (1.0 - f["h1"] ** 2))
    gw1 = dz1.T @ f["x0"]
    gw1[:, NIN:] = 0.0
    g[W1:B1] = gw1.ravel() * scale
    g[B1:W2] = dz1.sum(0) * scale
    g[W4:B4].reshape(16, 64)[NOUT:, :] = 0.0
    g[B4 + NOUT:NPARAM] = 0.0
    return loss, g


def glorot(seed: int) -> np.ndarray:
    """A parameter vector in the device's initial form (Glorot-uniform weights, zero biases)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM)

    def fill(ofs, nout, nin, use_out, use_in):
        a = np.sqrt(6.0 / (use_in + use_out))
        m = np.zeros((nout, nin))
        m[:use_out, :use_in] = rng.uniform(-a, a, (use_out, use_in))
        p[ofs:ofs + nout * nin] = m.ravel()

    fill(W1, 64, 16, 64, NIN)
    fill(W2, 64, 64, 64, 64)
    fill(W3, 64, 64, 64, 64)
    fill(W4, 16, 64, NOUT, 64)
    return p
