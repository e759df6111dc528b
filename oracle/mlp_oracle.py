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
               weights, the hidden activations (for predictions also the pre-activations,
               the argument of the inference kernel's BF16 tanh, with ties rounded away from
               zero as that kernel does), and the backward signals dZ. This is the
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


def bf16_ta(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties away from zero in magnitude: the inference
    kernel's integer rounding of the tanh argument); returned as float64."""
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    u = (u + 0x8000) & 0xFFFF0000
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
    """(x - mu) * (1/sig) in float32 as the device computes it (the reciprocal rounded to
    float32 once), padded to 16 columns."""
    X = np.asarray(X, np.float32)
    isig = (np.float32(1.0) / np.asarray(norm["in_sig"], np.float32)).astype(np.float32)
    z = (X - np.asarray(norm["in_mu"], np.float32)) * isig
    out = np.zeros((X.shape[0], K0), np.float64)
    out[:, :NIN] = z.astype(np.float64)
    return out


def forward(p: np.ndarray, X: np.ndarray, norm: dict, exact: bool = False, inference: bool = False) -> dict:
    """Forward pass. In bf16 mode the hidden activations are rounded to BF16; the inference
    kernel also rounds the pre-activation (the argument of its BF16 tanh), the training kernel
    does not (FP32 tanh)."""
    w = unpack(p)
    r = (lambda a: a) if exact else bf16
    ra = (lambda a: a) if (exact or not inference) else bf16_ta
    x0 = r(standardise(X, norm))
    h1 = r(np.tanh(ra(x0 @ r(w["W1"]).T + w["b1"])))
    h2 = r(np.tanh(ra(h1 @ r(w["W2"]).T + w["b2"])))
    h3 = r(np.tanh(ra(h2 @ r(w["W3"]).T + w["b3"])))
    y = h3 @ r(w["W4"]).T + w["b4"]
    return {"x0": x0, "h1": h1, "h2": h2, "h3": h3, "y": y[:, :NOUT]}


def predict(p: np.ndarray, X: np.ndarray, norm: dict, exact: bool = False) -> np.ndarray:
    """Outputs tau/rho (samples x 9)."""
    y = forward(p, X, norm, exact, inference=True)["y"]
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


def closure_inputs(hydro: np.ndarray, J31: np.ndarray, J32: np.ndarray, J33: np.ndarray, D: np.ndarray,
                   dX: float, dY: float, dZ: float, g: float, halo: int = 3) -> np.ndarray:
    """FP64 closure inputs of every interior cell (rows in i, j, k order, k fastest).

    hydro is the flux-form state [rho, rho u, rho v, rho w, rho theta][i][j][k] with `halo` cells
    per side; J31/J32/J33/D the grid metrics on the same points. The 9 velocity-gradient halves
    are the staggered strain-rate terms of cuda_sgsTurbDevice.cu:60-197 at the stress point (the
    cell's lower faces and edges); N^2 = g/theta * dtheta/dz with the centred terrain-following
    derivative of cuda_sgstkeDevice.cu:96-151; the grid scale is (dx dy dz D)^(1/3).
    """
    h = hydro.astype(np.float64)
    r = np.maximum(h[0], 1e-6)
    u, v, w, th = h[1] / r, h[2] / r, h[3] / r, h[4] / r
    j1, j2, j3 = (a.astype(np.float64) for a in (J31, J32, J33))
    nx, ny, nz = h.shape[1] - 2 * halo, h.shape[2] - 2 * halo, h.shape[3] - 2 * halo
    dxi, dyi, dzi = 1.0 / dX, 1.0 / dY, 1.0 / dZ

    def at(a, di, dj, dk):
        return a[halo + di:halo + di + nx, halo + dj:halo + dj + ny, halo + dk:halo + dk + nz]

    J1, J2, J3 = at(j1, 0, 0, 0), at(j2, 0, 0, 0), at(j3, 0, 0, 0)

    def dx(a, o1, o2):  # d/dx between points o1 and o2 (o1 - o2 = one cell in x)
        return dxi * (at(a, *o1) - at(a, *o2))

    def dy(a, o1, o2):
        return dyi * (at(a, *o1) - at(a, *o2))

    def dz(a, o1, o2):
        return dzi * (at(a, *o1) - at(a, *o2))

    C, Ai, Bj, Dk = (0, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, -1)
    AB, AD, BD, ABD = (-1, -1, 0), (-1, 0, -1), (0, -1, -1), (-1, -1, -1)
    x = np.empty((11, nx, ny, nz))
    x[0] = dx(u, C, Ai)
    x[1] = 0.5 * (dy(u, C, Bj) + dy(u, Ai, AB))
    x[2] = (0.5 * J1 * (dx(u, C, Ai) + dx(u, Dk, AD))
            + 0.25 * J2 * (dy(u, C, Bj) + dy(u, Ai, AB) + dy(u, Dk, BD) + dy(u, AD, ABD))
            + 0.5 * J3 * (dz(u, C, Dk) + dz(u, Ai, AD)))
    x[3] = 0.5 * (dx(v, C, Ai) + dx(v, Bj, AB))
    x[4] = dy(v, C, Bj)
    x[5] = (0.25 * J1 * (dx(v, C, Ai) + dx(v, Bj, AB) + dx(v, Dk, AD) + dx(v, BD, ABD))
            + 0.5 * J2 * (dy(v, C, Bj) + dy(v, Dk, BD))
            + 0.5 * J3 * (dz(v, C, Dk) + dz(v, Bj, BD)))
    x[6] = 0.5 * (dx(w, C, Ai) + dx(w, Dk, AD))
    x[7] = 0.5 * (dy(w, C, Bj) + dy(w, Dk, BD))
    x[8] = J1 * dx(w, C, Ai) + J2 * dy(w, C, Bj) + J3 * dz(w, C, Dk)
    dthdz = 0.5 * (J1 * dxi * (at(th, 1, 0, 0) - at(th, -1, 0, 0)) + J2 * dyi * (at(th, 0, 1, 0) - at(th, 0, -1, 0))
                   + J3 * dzi * (at(th, 0, 0, 1) - at(th, 0, 0, -1)))
    x[9] = g / at(th, 0, 0, 0) * dthdz
    x[10] = np.cbrt(float(dX) * float(dY) * float(dZ) * at(D.astype(np.float64), 0, 0, 0))
    return x.reshape(11, -1).T
