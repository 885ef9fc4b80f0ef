"""FP64 numpy restatement of the learned smoother's network -- test infrastructure.

Checks the GPU forward / backward kernels (dendro_b200/csrc/mlp.cu).  The
network: y = w3 . gelu(W2 gelu(W1 f + b1) + b2) + b3 with exact (erf) GELU;
parameters packed as W1[64][6] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3.
"""
from __future__ import annotations

import math

import numpy as np

IN, H = 6, 64
SIZES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("w3", (H,)), ("b3", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SIZES])


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(p, F):
    w = unpack(p)
    z1 = F @ w["W1"].T + w["b1"]
    a1 = gelu(z1)
    z2 = a1 @ w["W2"].T + w["b2"]
    a2 = gelu(z2)
    return a2 @ w["w3"] + w["b3"][0], (z1, a1, z2, a2)


def loss_and_grad(p, F, T):
    """Mean squared error and its gradient w.r.t. the packed parameters."""
    F = np.asarray(F, np.float64)
    T = np.asarray(T, np.float64)
    n = len(T)
    w = unpack(p)
    y, (z1, a1, z2, a2) = forward(p, F)
    diff = y - T
    dy = 2.0 * diff / n
    g = {"w3": a2.T @ dy, "b3": np.array([dy.sum()])}
    dz2 = (dy[:, None] * w["w3"][None, :]) * gelu_grad(z2)
    g["W2"] = dz2.T @ a1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * gelu_grad(z1)
    g["W1"] = dz1.T @ F
    g["b1"] = dz1.sum(0)
    return float((diff * diff).mean()), pack(g)


def init_params(seed: int = 0):
    """He-style initialisation with a zero output layer bias."""
    rng = np.random.default_rng(seed)
    d = {"W1": rng.normal(0, math.sqrt(2.0 / IN), (H, IN)), "b1": np.zeros(H),
         "W2": rng.normal(0, math.sqrt(2.0 / H), (H, H)), "b2": np.zeros(H),
         "w3": rng.normal(0, math.sqrt(1.0 / H), H), "b3": np.zeros(1)}
    return pack(d)
