"""Learned post-smoother: training data from the plain solver and training
with the library's own GPU kernels (forward, backward, Adam).

Pairs: for a seeded log-normal octree and a random load vector b, one
V-cycle without post-smoothing gives x_pc (the state the post-smoother sees);
its residual r = b - A x_pc and error e = A^-1 r form one residual/error pair.
The part of e that a smoother can remove is its rough part: the target is
(I - S^k) e with S = I - w D^-1 A the damped-Jacobi error propagator (k = 4,
w = 2/3), i.e. what k Jacobi sweeps would take out of the error, computed
from r as k sweeps on A c = r from c = 0 (no solve needed).  The smooth rest
of e is left to the coarse grids; as a target it would be large and not
predictable from local features.  The network input is the per-node feature
vector of r (dg_damg_features) and the target t_i = c_i d_i / s, so that the
update x_i += y_i s / d_i applies the predicted correction.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import inputs as I
from ._lib import check, lib, ptr
from .api import DAMG, Jacobian2, balanceOctree, points2Octree

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "mlp_smoother.npy")


class MLP:
    """Handle of the GPU network (dg_mlp)."""

    def __init__(self, params=None):
        self.n_params = int(lib().dg_mlp_param_count())
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        h = C.c_void_p()
        check(lib().dg_mlp_create(ptr(p), C.byref(h)), "mlp_create")
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                lib().dg_mlp_destroy(h)
            except TypeError:  # interpreter shutdown: module globals already cleared
                pass
            self.h = None

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        check(lib().dg_mlp_get_params(self.h, ptr(out)), "mlp_get_params")
        return out

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(lib().dg_mlp_set_params(self.h, ptr(p)), "mlp_set_params")

    def forward(self, F, exact=False):
        import torch
        out = torch.empty(F.shape[0], dtype=torch.float32, device=F.device)
        check(lib().dg_mlp_forward(self.h, ptr(F), F.shape[0], ptr(out), int(exact), None), "mlp_forward")
        torch.cuda.synchronize()
        return out

    def gradient(self, F, T, exact=True):
        g = np.empty(self.n_params, np.float32)
        loss = C.c_double()
        check(lib().dg_mlp_gradient(self.h, ptr(F), ptr(T), F.shape[0], int(exact), ptr(g), C.byref(loss)),
              "mlp_gradient")
        return loss.value, g

    def train_step(self, F, T, lr):
        loss = C.c_double()
        check(lib().dg_mlp_train_step(self.h, ptr(F), ptr(T), F.shape[0], C.c_float(lr), C.byref(loss)),
              "mlp_train_step")
        return loss.value


def features(m: DAMG, r):
    """Per-node features [N, 6] of a finest-level residual (device tensors) and s."""
    import torch
    F = torch.empty((r.numel(), 6), dtype=torch.float32, device=r.device)
    s = C.c_float()
    check(lib().dg_damg_features(m.h, ptr(r), ptr(F), C.byref(s)), "damg_features")
    return F, s.value


def vcycle(m: DAMG, b):
    import torch
    x = torch.empty_like(b)
    check(lib().dg_damg_vcycle(m.h, ptr(b), ptr(x)), "damg_vcycle")
    return x


def make_pair_source(seed: int, n_points: int, depth: int = 14, coef_sphere: bool = True):
    """Mesh, hierarchies and operator for one seeded log-normal octree."""
    import torch
    pts = I.clamp_unit(I.lognormal_cloud(n_points, seed), depth)
    bal = balanceOctree(points2Octree(pts, depth, 1))
    pre = DAMG(bal, nu_post=0)            # pre-smoothing + coarse correction only
    da = pre.level_da(0)
    coef = I.sphere_coefficients(da.elementCenters()) if coef_sphere else None
    pre.setKSP(coef)
    A = Jacobian2(da, coef)
    d = A.getDiagonal()
    return dict(pre=pre, A=A, d=d, N=da.N, dev=torch.device("cuda"), bal=bal)


SWEEPS, OMEGA = 4, 2.0 / 3.0


def rough_error(A, d, r, sweeps: int = SWEEPS, omega: float = OMEGA):
    """(I - S^k) A^-1 r: k damped-Jacobi sweeps on A c = r from c = 0."""
    c = omega * r / d
    for _ in range(sweeps - 1):
        c = c + omega * (r - A.mult(c)) / d
    return c


def make_pair(src, rng):
    """One residual/error pair: features F [N,6], targets T [N] (device)."""
    import torch
    N = src["N"]
    b = torch.tensor(rng.uniform(-1.0, 1.0, N), device="cuda")
    xpc = vcycle(src["pre"], b)
    r = b - src["A"].mult(xpc)
    c = rough_error(src["A"], src["d"], r)
    F, s = features(src["pre"], r)
    T = (c * src["d"] / s).float()
    return F, T


def train(n_pairs: int = 2000, steps_per_pair: int = 2, batch: int = 65536, lr: float = 2e-3, seed: int = 0,
          mesh_points=(60000, 120000, 240000), time_budget_s=None, log=print):
    """Train on residual/error pairs from seeded log-normal meshes (about
    262K-1M octants for the default point counts) with the GPU kernels;
    returns the MLP and the per-pair loss history."""
    import torch
    mlp = MLP(init_params(seed))
    rng = np.random.default_rng(seed + 1000)
    sources = [make_pair_source(10 + i, npts) for i, npts in enumerate(mesh_points)]
    hist = []
    t0 = time.time()
    gen = torch.Generator(device="cuda").manual_seed(seed)
    for k in range(n_pairs):
        src = sources[k % len(sources)]
        F, T = make_pair(src, rng)
        loss = None
        for _ in range(steps_per_pair):
            idx = torch.randint(0, F.shape[0], (min(batch, F.shape[0]),), device="cuda", generator=gen)
            loss = mlp.train_step(F[idx].contiguous(), T[idx].contiguous(), lr)
        hist.append(loss)
        if log and (k % 100 == 0 or k == n_pairs - 1):
            log(f"pair {k} loss {loss:.4e} ({time.time() - t0:.1f} s)")
        if time_budget_s and time.time() - t0 > time_budget_s:
            break
    return mlp, hist


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation (W1 / W2 scaled by fan-in), zero biases."""
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0, np.sqrt(2.0 / 6), (64, 6))
    W2 = rng.normal(0, np.sqrt(2.0 / 64), (64, 64))
    w3 = rng.normal(0, np.sqrt(1.0 / 64), 64)
    return np.concatenate([W1.ravel(), np.zeros(64), W2.ravel(), np.zeros(64), w3, np.zeros(1)]).astype(np.float32)


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the learned post-smoother on the GPU")
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--steps-per-pair", type=int, default=2)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--budget", type=float, default=None, help="stop after this many seconds")
    a = ap.parse_args()
    mlp, hist = train(a.pairs, a.steps_per_pair, lr=a.lr, time_budget_s=a.budget)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    np.save(a.out, mlp.params)
    print(json.dumps({"pairs": len(hist), "first_loss": hist[0], "last_loss": float(np.mean(hist[-20:])),
                      "out": a.out}))
