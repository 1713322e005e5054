"""CPU oracle of the learned troubled-cell indicator.  TEST INFRASTRUCTURE ONLY.

The indicator has no counterpart in the reference; this numpy restatement in
float64 (forward pass, BCE-with-logits loss with a positive-class weight, and
hand-written backpropagation) is the checker of the GPU kernels in
zuikakucfd_b200/csrc/mlp.cu ("parity unpinned": nothing in the reference
pins it).  It is itself checked against central finite differences in the CPU
test suite.  Also restated here: the 40 input features the GPU computes per
cell (zk_mlp.h) from a DG state.

Parameter block (flat, row-major, out x in): w1[32][40] b1[32] w2[32][32]
b2[32] w3[32][32] b3[32] w4[32] b4.
"""
from __future__ import annotations

import math

import numpy as np

IN, H = 40, 32
NPARAM = H * IN + H + 2 * (H * H + H) + H + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = {}
    for name, shape in (("w1", (H, IN)), ("b1", (H,)), ("w2", (H, H)), ("b2", (H,)), ("w3", (H, H)),
                        ("b3", (H,)), ("w4", (H,)), ("b4", ())):
        n = int(np.prod(shape)) if shape else 1
        out[name] = p[o:o + n].reshape(shape) if shape else p[o]
        o += n
    assert o == NPARAM
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation, zero biases."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, math.sqrt(2.0 / IN), (H, IN)), np.zeros(H),
             rng.normal(0, math.sqrt(2.0 / H), (H, H)), np.zeros(H),
             rng.normal(0, math.sqrt(2.0 / H), (H, H)), np.zeros(H),
             rng.normal(0, math.sqrt(1.0 / H), H), np.zeros(1)]
    return np.concatenate([np.ravel(a) for a in parts]).astype(np.float32)


_K, _C = math.sqrt(2.0 / math.pi), 0.044715


def gelu(x):
    """GELU, tanh form (the form the GPU kernels use)."""
    return 0.5 * x * (1.0 + np.tanh(_K * (x + _C * x ** 3)))


def gelu_grad(x):
    t = np.tanh(_K * (x + _C * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _K * (1.0 + 3.0 * _C * x * x)


def forward(p, X):
    """Logits of X[n][40]; also returns the intermediates for backward."""
    W = unpack(p)
    X = np.asarray(X, np.float64)
    z1 = X @ W["w1"].T + W["b1"]
    h1 = gelu(z1)
    z2 = h1 @ W["w2"].T + W["b2"]
    h2 = gelu(z2)
    z3 = h2 @ W["w3"].T + W["b3"]
    h3 = gelu(z3)
    z = h3 @ W["w4"] + W["b4"]
    return z, (X, z1, h1, z2, h2, z3, h3)


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def forward_bf16(p, X):
    """Logits with the arithmetic of the GPU's tensor-core inference: features,
    every parameter and each hidden layer's GELU output rounded to BF16,
    products summed in FP32 (here exactly, in float64, then rounded), GELU in
    FP32 and the output unit in FP32."""
    W = {k: bf16(v) if np.ndim(v) else bf16(np.float32(v))[()] for k, v in unpack(p).items()}
    h = bf16(X).astype(np.float64)
    for l in ("1", "2", "3"):
        z = (h @ W["w" + l].astype(np.float64).T + W["b" + l]).astype(np.float32)
        u = np.float32(_K) * (z + np.float32(_C) * z * z * z)
        g = np.float32(0.5) * z * (np.float32(1.0) + np.tanh(u.astype(np.float64)).astype(np.float32))
        h = bf16(g).astype(np.float64)
    return (h @ W["w4"].astype(np.float64) + W["b4"]).astype(np.float32)


def loss_and_grad(p, X, y, pos_weight):
    """Mean BCE-with-logits loss (positive weight) and its gradient."""
    W = unpack(p)
    z, (X, z1, h1, z2, h2, z3, h3) = forward(p, X)
    y = np.asarray(y, np.float64)
    sp_pos = np.logaddexp(0.0, -z)   # softplus(-z)
    sp_neg = np.logaddexp(0.0, z)    # softplus(z)
    n = X.shape[0]
    loss = float(np.mean(pos_weight * y * sp_pos + (1.0 - y) * sp_neg))
    sig = 1.0 / (1.0 + np.exp(-z))
    dz = (pos_weight * y * (sig - 1.0) + (1.0 - y) * sig) / n
    g = {}
    g["w4"] = h3.T @ dz
    g["b4"] = dz.sum()
    d3 = np.outer(dz, W["w4"]) * gelu_grad(z3)
    g["w3"] = d3.T @ h2
    g["b3"] = d3.sum(0)
    d2 = (d3 @ W["w3"]) * gelu_grad(z2)
    g["w2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ W["w2"]) * gelu_grad(z1)
    g["w1"] = d1.T @ X
    g["b1"] = d1.sum(0)
    flat = np.concatenate([np.ravel(g[k]) for k in ("w1", "b1", "w2", "b2", "w3", "b3", "w4")] + [[g["b4"]]])
    return loss, flat


def features(P: int, dof: np.ndarray, kind: np.ndarray, src: np.ndarray, means: np.ndarray | None = None) -> np.ndarray:
    """The 40 per-cell features of the GPU indicator (zk_mlp.h) for every
    updated cell: the rho and E modes of the DG state dof[4][NM][ny][nx] and
    the means (own and neighbours', gathered through the ghost map: kind/src as
    oracle Restatement.ghost_map returns, with slip) of `means` -- the input
    of the RK stage whose output dof is -- or of dof itself when None.  FP32
    arithmetic on FP32-rounded values, as the GPU computes them.  The two
    scaled means (slots 0 and 16) are centred (minus 1): a constant state's
    features are all 0."""
    NM = (P + 1) ** 2
    ny, nx = dof.shape[2:]
    out = np.zeros((ny * nx, IN), np.float32)
    flat = dof.reshape(4, NM, -1)
    mflat = (dof if means is None else means).reshape(4, NM, -1)

    def mean(k):
        s = int(src.flat[k]) if src.flat[k] >= 0 else k   # slip walls negate momentum only
        return np.float32(mflat[0, 0, s]), np.float32(mflat[3, 0, s])

    for k in range(ny * nx):
        if kind.flat[k] != 0:
            continue
        ms = [mean(k)] if means is not None else [(np.float32(mflat[0, 0, k]), np.float32(mflat[3, 0, k]))]
        ms += [mean(k - 1), mean(k + 1), mean(k - nx), mean(k + nx)]
        sr = np.float32(max(abs(m[0]) for m in ms)) + np.float32(1e-12)
        se = np.float32(max(abs(m[1]) for m in ms)) + np.float32(1e-12)
        ir, ie = np.float32(1.0) / sr, np.float32(1.0) / se
        for m in range(NM):
            slot = (m // (P + 1)) * 4 + m % (P + 1)
            out[k, slot] = np.float32(flat[0, m, k]) * ir
            out[k, 16 + slot] = np.float32(flat[3, m, k]) * ie
        out[k, 0] -= np.float32(1.0)   # the scaled means, centred
        out[k, 16] -= np.float32(1.0)
        for n_ in range(4):
            out[k, 32 + n_] = (ms[1 + n_][0] - ms[0][0]) * ir
            out[k, 36 + n_] = (ms[1 + n_][1] - ms[0][1]) * ie
    return out
