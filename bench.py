"""Benchmark of the matrix-free octree FEM hot path on B200.

Matvec leg (the JSON line's value): 1,048,576 log-normal points (seed 2,
maxDepth 14), points2Octree + 2:1 balance on the GPU, the mesh, and the FP64
variable-coefficient operator -div(a grad u) + u with a = 1e4 inside the
sphere of radius 0.25 about the centre and 1 outside.  A step is one operator
application (y = A x) over the whole mesh; the L2 cache is flushed before
every step.  Extra legs (in the same line): the solve leg on 4,194,304
log-normal points (seed 4, maxDepth 16) -- time to FP64 relative residual
1e-8 for the plain FP64 V(2,2)-preconditioned CG with the reference's solver
options (Jacobi damping 2/3) and the chosen mixed-precision methods (FP32
V-cycle; damping 2/3 and 0.9, plus FP64 at 0.9 to separate the two gains) --
a 64-right-hand-side tensor-core leg on 524,288 uniform points (seed 5,
maxDepth 12) and a batched leg of 32 meshes.

    python bench.py --gpus N --steps K --warmup W [--impl reference]

N > 1 runs under torchrun, one rank per GPU: the matvec workload's one mesh
partitioned over the ranks (SFC-weighted element ranges, ghost exchange of x
over NCCL per application: strong scaling, the reference's parallel form);
rank 0 prints one JSON line with the whole mesh's GDoF/s, timed as the max
over ranks.  With one GPU the same partitioned path is reported beside the
plain operator.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to FP64 rel. residual 1e-8 & matvec GDoF/s: chosen vs plain FP64, 1 B200"
WORKLOAD = "lognormal1m_d14"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one operator
# launch on the default workload, per launch shape, each from a one-kernel
# ncu capture of that shape (profiles/lapmass_traffic_lognormal1m_d14.md
# gives the commands); a shape without a capture reports null.
TRAFFIC = {
    "warp-tile 32 elems, 5 CTAs/SM": 313494528 + 19637248,
    "warp-tile 32 elems, 3 CTAs/SM, ids and x of the next tile in flight": 313441024 + 19751680,
    "octet b128, 4 CTAs/SM": 217575168 + 18488576,
    "octet b256, 2 CTAs/SM": 217540864 + 18269184,
    "octet b128, next ids in flight, 4 CTAs/SM": 217420288 + 15001600,
    "octet b128, next ids in flight, two halves, 4 CTAs/SM": 217417472 + 15151104,
    "octet b128, next ids in flight, two halves, 5 CTAs/SM": 217705984 + 17701376,
    "octet b128, next ids in flight, complete-warp fast path, 4 CTAs/SM": 217558784 + 15632640,
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="dendro_b200", choices=["dendro_b200", "reference"])
    p.add_argument("--workload", default=WORKLOAD)
    p.add_argument("--scale", type=float, default=1.0, help="fraction of the workload's points (testing)")
    p.add_argument("--no-solve", action="store_true")
    p.add_argument("--no-multi", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-cfg1", action="store_true")
    p.add_argument("--no-elasticity", action="store_true")
    p.add_argument("--no-partitioned", action="store_true")
    p.add_argument("--no-cmap", action="store_true")
    p.add_argument("--solve-workload", default="lognormal4m_d16")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--vcycle-profile", metavar="WORKLOAD", default=None,
                   help="only: one FP64 and one FP32 V(2,2) cycle on WORKLOAD's hierarchy between "
                        "cudaProfilerStart/Stop (for ncu --profile-from-start off), then exit")
    p.add_argument("--halo-profile", metavar="PARTS", type=int, default=0,
                   help="only: split the matvec workload's mesh into PARTS parts (all on this GPU) and time "
                        "each part's pack, independent and dependent operator launches, then exit")
    p.add_argument("--cmap-profile", metavar="WORKLOAD", default=None,
                   help="only: the element kernel on the compressed and on the raw element map, FP64 and FP32, "
                        "one launch each between cudaProfilerStart/Stop, then exit")
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    return p.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu_index: int):
        import tempfile
        self.proc = None
        self.path = os.path.join(tempfile.mkdtemp(prefix="dg_clocks_"), f"clocks_gpu{gpu_index}.csv")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        med = float(np.median(sm)) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(name, scale):
    from dendro_b200 import inputs as I
    pts, depth = I.workload_points(name, scale)
    return pts, depth


def run_dendro(args, rank, world):
    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    pts, depth = build_workload(args.workload, args.scale)
    t0 = time.time()
    bal = dg.balanceOctree(dg.points2Octree(pts, depth, 1))
    da = dg.DA(bal)
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    coef = I.sphere_coefficients(da.elementCenters())
    A = dg.Jacobian2(da, coef)
    E, N = da.E, da.N
    x = torch.tensor(I.uniform_rhs(N, 3), device=dev)
    y = torch.empty_like(x)
    if world > 1:
        return run_dendro_partitioned(args, dev, bal, depth, coef, x, E, N, world, setup_s)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    stream = torch.cuda.current_stream(dev)

    clocks = ClockSampler(dev.index)
    for _ in range(args.warmup):
        A.mult(x, y, stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.fill_(float(i))  # evict the mesh and vectors from L2 between steps
        ev[i][0].record(stream)
        A.mult(x, y, stream)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    if world > 1:
        from dendro_b200.parallel import max_over_ranks
        total_ms = max_over_ranks(total_ms, dev)
        torch.distributed.barrier()
    ms_per_step = total_ms / args.steps
    gdofs = N * args.steps / (total_ms * 1e-3) / 1e9

    # roofline of the operator kernel: algorithmic bytes per launch
    alg_bytes = 36 * E + 16 * E + 16 * N  # element record + (a, b) FP64 + x read + y written
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms_per_step * 1e-3) / 1e9

    # end to end through the host entry point (pinned host x, y)
    xh = torch.empty(N, dtype=torch.float64, pin_memory=True)
    xh.copy_(x.cpu())
    yh = torch.empty(N, dtype=torch.float64, pin_memory=True)
    A.mult(xh.numpy(), yh.numpy())
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(args.steps):
        A.mult(xh.numpy(), yh.numpy())
    e2e_s = time.perf_counter() - t1
    clk = clocks.stop()  # samples span the device-timed steps and the end-to-end loop
    e2e = {"value": N * args.steps / e2e_s / 1e9, "unit": "GDoF/s", "h2d_bytes_per_step": 8 * N,
           "d2h_bytes_per_step": 8 * N}

    # the partitioned path with one rank: the same mesh through the
    # partitioned operator (what --gpus N > 1 times), for comparison
    part = None
    if not args.no_partitioned:
        part = run_partitioned(args, dev, bal, coef, x, 1, min(args.steps, 50), args.warmup)
        part = {"ms_per_step": round(part["ms_per_step"], 5),
                "gdofs": round(N / (part["ms_per_step"] * 1e-3) / 1e9, 4)}
    kernel = A.kernel_name(0)
    cmap = None if args.no_cmap else run_cmap(A, da, x, y, flush, stream, min(args.steps, 20))
    solve = None if args.no_solve else run_solve(dev, args.solve_workload)
    multi = None if args.no_multi else run_multi(dev, min(args.steps, 50))
    batch = None if args.no_batch else run_batch(dev)
    cfg1 = None if args.no_cfg1 else run_cfg1(dev)
    elastic = None if args.no_elasticity else run_elasticity(dev, bal)
    return dict(cmap=cmap, elasticity=elastic, partitioned_one_rank=part, multi=multi, batch=batch, cfg1=cfg1, kernel=kernel, E=E, N=N, setup_s=setup_s, ms_per_step=ms_per_step, gdofs=gdofs, achieved=achieved, peak=peak,
                peak_kind=peak_kind, alg_bytes=alg_bytes, clocks=clk, e2e=e2e, solve=solve, bal=bal, depth=depth,
                coef=coef, x=x.cpu().numpy(), y=y.cpu().numpy())


def run_cmap(A, da, x, y_default, flush, stream, steps):
    """The compressed element map on the benchmark mesh: its bytes per element, and the element
    kernel reading it against the same kernel reading the raw map (FP64 and FP32, L2 flushed)."""
    import torch
    t0 = time.time()
    nbytes = da.compressMaps()
    torch.cuda.synchronize()
    build_ms = (time.time() - t0) * 1e3
    shape = None
    for v in range(A.kernel_count()):
        A.set_kernel(v, 0)
        if "compressed map" in A.kernel_name(0):
            shape = v
    out = {"bytes_per_element": round(nbytes / da.E, 3), "raw_bytes_per_element": 32,
           "wide_tiles": da.compressedMapBytes()[1], "build_ms": round(build_ms, 2)}
    for prec, name in ((0, "f64"), (1, "f32")):
        xx = x if prec == 0 else x.float()
        yy = torch.empty_like(xx)
        for tag, v in (("compressed", shape), ("raw", 0)):
            A.set_kernel(v, prec)
            for _ in range(3):
                A.mult(xx, yy, stream)
            ts = []
            for i in range(steps):
                flush.fill_(float(i))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                A.mult(xx, yy, stream)
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            out[f"{name}_{tag}_ms"] = round(float(np.median(ts)), 4)
            if prec == 0 and tag == "compressed":
                out["vs_default_rel_err"] = rel_err(yy.cpu().numpy(), y_default.cpu().numpy())
    return out


def run_partitioned(args, dev, bal, coef, x_full, world, steps, warmup):
    """One mesh over the ranks (strong scaling; the reference's only parallel
    strategy, examples/src/backend/omgNeumann.C:505-525): every rank takes
    its SFC-weighted element range (par::partitionW) and owned nodes, and one
    operator application is the ghost exchange of x (one all-to-all over
    NCCL, overlapped with the independent elements) and the independent and
    dependent elements' launches.  Timed like the single-GPU leg (L2 flushed,
    CUDA events, max over ranks); with one rank it is the whole mesh."""
    import torch

    import dendro_b200 as dg
    from dendro_b200.halo import HaloDA, HaloJacobian2
    da = dg.DA(bal)
    h = HaloDA(da)
    op = HaloJacobian2(h, coef)
    xo = x_full[h.first_owned:h.first_owned + h.n_owned]
    xl = h.local_vector(xo)
    yl = torch.zeros_like(xl)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(warmup):
        op.mult(xl, yl)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for i in range(steps):
        flush.fill_(float(i))
        e0[i].record()
        op.mult(xl, yl)
        e1[i].record()
    torch.cuda.synchronize()
    total = float(sum(a.elapsed_time(b) for a, b in zip(e0, e1)))
    # end to end: this rank's owned x from page-locked host memory in, its y out
    xh = torch.empty(h.n_owned, dtype=torch.float64, pin_memory=True)
    xh.copy_(xo.cpu())
    yh = torch.empty(h.n_owned, dtype=torch.float64, pin_memory=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        xl[: h.n_owned].copy_(xh, non_blocking=True)
        op.mult(xl, yl)
        yh.copy_(yl[: h.n_owned], non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        from dendro_b200.parallel import max_over_ranks
        total = max_over_ranks(total, dev)
        e2e_s = max_over_ranks(e2e_s, dev)
    return {"ms_per_step": total / steps, "e2e_s": e2e_s, "n_owned": h.n_owned, "n_ghost": h.n_ghost,
            "independent": len(h.independent), "dependent": len(h.dependent), "h2d_bytes": 8 * h.n_owned,
            "d2h_bytes": 8 * h.n_owned}


def run_dendro_partitioned(args, dev, bal, depth, coef, x, E, N, world, setup_s):
    """--gpus N > 1: the matvec workload's one mesh partitioned over the N
    ranks; value = the whole mesh's DoF per second (strong scaling)."""
    clocks = ClockSampler(dev.index)
    r = run_partitioned(args, dev, bal, coef, x, world, args.steps, args.warmup)
    clk = clocks.stop()
    ms = r["ms_per_step"]
    alg_bytes = 36 * E + 16 * E + 16 * N
    peak, peak_kind = measured_peaks()
    e2e = {"value": N * args.steps / r["e2e_s"] / 1e9, "unit": "GDoF/s", "h2d_bytes_per_step": 8 * N,
           "d2h_bytes_per_step": 8 * N}
    return dict(partitioned=r, multi=None, batch=None, cfg1=None, kernel="partitioned: per-rank tuned operator",
                E=E, N=N, setup_s=setup_s, ms_per_step=ms, gdofs=N / (ms * 1e-3) / 1e9,
                achieved=alg_bytes / world / (ms * 1e-3) / 1e9, peak=peak, peak_kind=peak_kind, alg_bytes=alg_bytes,
                clocks=clk, e2e=e2e, solve=None, bal=bal, depth=depth, coef=coef, x=None, y=None)


def run_solve(dev, workload):
    """Solve leg: -Laplace u + u (constant coefficients) with f = U[-1,1] per
    node (seed 3) on the given point-cloud octree, time to FP64 relative
    residual rtol for the plain FP64 method and the chosen mixed-precision
    ones.  The FP64 reference solution is the plain solver run to 1e-12."""
    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I
    from dendro_b200.learned import MLP, WEIGHTS
    pts, depth = build_workload(workload, 1.0)
    bal = dg.balanceOctree(dg.points2Octree(pts, depth, 1))
    methods = [("plain_fp64", dict(inner_prec=0, use_graph=False), False, (1e-8,)),
               ("plain_fp64_omega09", dict(inner_prec=0, use_graph=False, omega=0.9), False, (1e-8,)),
               ("mixed_fp32", dict(inner_prec=1, use_graph=True), False, (1e-6, 1e-8, 1e-10)),
               ("mixed_fp32_omega09", dict(inner_prec=1, use_graph=True, omega=0.9), False, (1e-6, 1e-8, 1e-10)),
               ("mixed_fp32_learned", dict(inner_prec=1, use_graph=True), True, (1e-6, 1e-8, 1e-10))]
    if not os.path.exists(WEIGHTS):
        methods = methods[:4]
    ref = dg.DAMG(bal, rtol=1e-12, maxit=400)
    N = int(ref.N[0])
    b = torch.tensor(I.uniform_rhs(N, 3), device=dev)
    xref, rref = ref.solve(b, allow_unconverged=True)
    out = {"workload": workload, "elements": int(ref.E[0]), "nodes": N, "levels": int(ref.nlevels),
           "reference_solution": {"rel_residual": rref["rel_residual"], "iterations": rref["iterations"]}}
    del ref
    nx = float(torch.linalg.norm(xref))
    for tag, kw, learned, tols in methods:
        m = dg.DAMG(bal, **kw)
        if learned:
            m.setSmoother(MLP(np.load(WEIGHTS)))
        m.solve(b, allow_unconverged=True)  # warm-up: autotuning and graph capture
        res = {}
        for rtol in tols:
            m.setTolerances(rtol, 400)
            best = None
            for _ in range(2):
                x, rep = m.solve(b, allow_unconverged=True)
                if best is None or rep["solve_ms"] < best[1]["solve_ms"]:
                    best = (x, rep)
            x, rep = best
            res[f"{rtol:.0e}"] = {"ms": round(rep["solve_ms"], 3), "iterations": rep["iterations"],
                                  "rel_residual": rep["rel_residual"], "converged": rep["converged"],
                                  "error_vs_fp64_solution": float(torch.linalg.norm(x - xref)) / nx,
                                  "smoother_fallbacks": rep.get("smoother_fallbacks", 0)}
        out[tag] = res
        del m
    chosen = [t for t, kw, _, _ in methods if kw["inner_prec"] != 0]
    best = min(out[t]["1e-08"]["ms"] for t in chosen)
    out["chosen_at_1e-8"] = min(chosen, key=lambda t: out[t]["1e-08"]["ms"])
    out["speedup_chosen_vs_plain_at_1e-8"] = round(out["plain_fp64"]["1e-08"]["ms"] / best, 3)
    # the mixed-precision gain alone, both at omega 0.9
    out["speedup_mixed_vs_fp64_same_cycle_at_1e-8"] = round(
        out["plain_fp64_omega09"]["1e-08"]["ms"] / out["mixed_fp32_omega09"]["1e-08"]["ms"], 3)
    out["methods"] = {
        "plain_fp64": "FP64 CG + FP64 V(2,2) damped Jacobi, omega 2/3 (the reference's solver options), "
                      "warp-tile operator, dense FP64 coarse solve",
        "plain_fp64_omega09": "plain_fp64 with Jacobi damping omega 0.9",
        "mixed_fp32": "FP64 flexible CG + FP32 V(2,2), omega 2/3 (FP32 operator, smoother, transfers), FP64 coarse "
                      "solve, V-cycle replayed from a CUDA graph",
        "mixed_fp32_omega09": "mixed_fp32 with Jacobi damping omega 0.9",
        "mixed_fp32_learned": "mixed_fp32 with the trained MLP post-smoother on the finest level, Jacobi fallback "
                              "when the FP64 residual stalls"}
    return out


def run_cfg1(dev, matvecs=100):
    """The small configuration in full on the GPU, with the set-up stages of
    examples/src/drivers/tstMatVec.C:165-275 timed one by one: 131,072
    Gaussian points (seed 0), maxDepth 10 -> points2Octree, 2:1 balance, the
    mesh; 100 operator applications (a = b = 1); PCG with the 4-level V(2,2)
    damped-Jacobi cycle (omega 2/3) to 1e-8 with f = U[-1, 1] (seed 1)."""
    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I
    pts, depth = build_workload("gauss131k_d10", 1.0)
    out = {"workload": "gauss131k_d10"}

    def timed(fn):
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t
    lin, out["points2octree_s"] = timed(lambda: dg.points2Octree(pts, depth, 1))
    bal, out["balance_s"] = timed(lambda: dg.balanceOctree(lin))
    da, out["da_build_s"] = timed(lambda: dg.DA(bal))
    out.update({"elements": da.E, "nodes": da.N})
    A = dg.Jacobian2(da)
    x = torch.tensor(I.uniform_rhs(da.N, 1), device=dev)
    y = torch.empty_like(x)
    for _ in range(3):
        A.mult(x, y)
    _, t = timed(lambda: [A.mult(x, y) for _ in range(matvecs)])
    out["matvec_ms"] = round(1e3 * t / matvecs, 4)
    out["matvec_gdofs"] = round(da.N * matvecs / t / 1e9, 3)
    m = dg.DAMG(bal, nlevels=4)
    b = torch.tensor(I.uniform_rhs(da.N, 1), device=dev)
    m.solve(b)
    xs, rep = m.solve(b)
    out["pcg"] = {"levels": m.nlevels, "coarse_nodes": int(m.N[-1]), "iterations": rep["iterations"],
                  "rel_residual": rep["rel_residual"], "solve_ms": round(rep["solve_ms"], 3)}
    for k in ("points2octree_s", "balance_s", "da_build_s"):
        out[k] = round(out[k], 4)
    return out


def run_elasticity(dev, bal, steps=200):
    """Linear elasticity on the matvec workload's mesh (E = 1, nu = 0.3;
    Dirichlet nodes on the domain boundary; f = U[-1, 1] per dof, seed 3):
    200 operator applications (L2 flushed between them) and the FP64 V(2,2)
    PCG solve to 1e-8 with the multigrid hierarchy of examples/src/drivers/
    newElasSolver.C (elasticity on every level, each level's boundary
    nodes Dirichlet)."""
    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I
    mu, lam = 1.0 / (2.0 * 1.3), 0.3 / (1.3 * 0.4)
    da = dg.DA(bal)
    A = dg.Elasticity(da, mu, lam)
    N, E = da.N, da.E
    x = torch.tensor(I.uniform_rhs(3 * N, 3), device=dev)
    y = torch.empty_like(x)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(3):
        A.mult(x, y)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot = 0.0
    for i in range(steps):
        flush.fill_(float(i))
        e0.record()
        A.mult(x, y)
        e1.record()
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    ms = tot / steps
    alg = 36 * E + 49 * N  # element record + 3-dof x read and y written (FP64) + 1 B Dirichlet flag per node
    peak, _ = measured_peaks()
    out = {"workload": "lognormal1m_d14", "elements": E, "nodes": N, "mu": mu, "lambda": lam, "matvecs": steps,
           "matvec_ms": round(ms, 4), "gdofs": round(3 * N / (ms * 1e-3) / 1e9, 3),
           "achieved_gbs": round(alg / (ms * 1e-3) / 1e9, 1), "frac_of_hbm": round(alg / (ms * 1e-3) / 1e9 / peak, 4),
           "algorithmic_bytes": int(alg)}
    m = dg.DAMG(bal, dof=3, mu=mu, lam=lam)
    b = torch.tensor(I.uniform_rhs(3 * N, 3), device=dev)
    m.solve(b, allow_unconverged=True)
    xs, rep = min((m.solve(b, allow_unconverged=True) for _ in range(2)), key=lambda t: t[1]["solve_ms"])
    res = torch.empty_like(b)
    A.mult(xs, res)
    out["solve"] = {"levels": m.nlevels, "iterations": rep["iterations"], "converged": rep["converged"],
                    "rel_residual": rep["rel_residual"], "ms": round(rep["solve_ms"], 3),
                    "true_rel_residual": float(torch.linalg.norm(res - b) / torch.linalg.norm(b))}
    return out


def run_batch(dev):
    """Batched leg: 32 independent Gaussian clouds (seeds 100-131, point counts
    log-uniform in [10K, 500K], maxDepth 12), -Laplace u + u, f = U[-1,1]
    (seed 7); one concatenated hierarchy solved with the FP32 V-cycle replayed
    from a CUDA graph (one launch per kernel for all meshes, per-mesh
    convergence to 1e-8), against the 32 meshes solved one after another."""
    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I
    clouds, depth = I.batch_clouds()
    trees = [dg.balanceOctree(dg.points2Octree(p, depth, 1)) for p in clouds]
    m = dg.DAMG(trees, inner_prec=1, use_graph=True)
    n = int(m.N[0])
    b = torch.tensor(I.uniform_rhs(n, 7), device=dev)
    m.solve(b, allow_unconverged=True)
    reps = [m.solve(b, allow_unconverged=True)[1] for _ in range(2)]
    rep = min(reps, key=lambda r: r["solve_ms"])
    _, no = m.batch_offsets(0)
    seq_ms, seq_its = 0.0, []
    for i, t in enumerate(trees):
        mi = dg.DAMG(t, inner_prec=1, use_graph=True)
        bi = b[int(no[i]):int(no[i + 1])].contiguous()
        mi.solve(bi, allow_unconverged=True)
        ri = min((mi.solve(bi, allow_unconverged=True)[1] for _ in range(2)), key=lambda r: r["solve_ms"])
        seq_ms += ri["solve_ms"]
        seq_its.append(ri["iterations"])
        del mi
    return {"meshes": len(trees), "elements": int(m.E[0]), "nodes": n, "levels": int(m.nlevels),
            "batched_ms": round(rep["solve_ms"], 3), "batched_iterations": rep["iterations"],
            "converged": rep["converged"], "rel_residual_max_over_meshes": rep["rel_residual"],
            "one_by_one_ms": round(seq_ms, 3), "one_by_one_iterations_max": int(max(seq_its)),
            "speedup_batched": round(seq_ms / rep["solve_ms"], 3)}


def run_multi(dev, steps, nrhs=64):
    """Multi-right-hand-side leg: 64 right-hand sides U[-1,1] (seed 6) on the
    uniform-point mesh (524,288 points, seed 5, maxDepth 12): one operator
    application per step in each form (octet on the CUDA cores, tensor cores
    split 3 and split 1), L2 flushed between steps; then the 64 solved
    together to 1e-8."""
    import torch

    import dendro_b200 as dg
    pts, depth = build_workload("uniform512k_d12", 1.0)
    da = dg.DA(dg.balanceOctree(dg.points2Octree(pts, depth, 1)))
    A = dg.Jacobian2(da)
    E, N = da.E, da.N
    X = torch.tensor(np.random.default_rng(6).uniform(-1, 1, (N, nrhs)), dtype=torch.float32, device=dev)
    Y = torch.empty_like(X)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    out = {"workload": "uniform512k_d12", "elements": E, "nodes": N, "nrhs": nrhs, "octets": da.octets}
    for split in (0, 3, 1, 5, 4):
        for _ in range(3):
            A.mult_multi(X, Y, split=split)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))
            ev[i][0].record(stream)
            A.mult_multi(X, Y, split=split)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
        alg = 36 * E + 2 * 4 * nrhs * N  # element record + X read + Y written (FP32)
        tag = {0: "octet_cuda_cores", 5: "tcgen05_split5", 4: "tcgen05_split4"}.get(split, f"split{split}")
        out[tag] = {"ms": round(ms, 4), "gdofs": round(N * nrhs / (ms * 1e-3) / 1e9, 3),
                    "achieved_gbs": round(alg / (ms * 1e-3) / 1e9, 1),
                    "frac_of_hbm": round(alg / (ms * 1e-3) / 1e9 / measured_peaks()[0], 4)}
        if split in (1, 3):  # m16n8k8 per element and 32 right-hand sides: 2 * 64 * nrhs flops per element
            out[tag]["tensor_tflops"] = round(2 * 64 * nrhs * E * split / (ms * 1e-3) / 1e12, 2)
        elif split in (4, 5):  # per pair of octets and 64 right-hand sides: M 128 x N 64 x K 32 per pass
            passes = 1 if split == 4 else 3
            flops = 2 * 128 * 64 * 32 * passes * ((da.octets + 1) // 2) * (nrhs // 64)
            out[tag]["tensor_tflops"] = round(flops / (ms * 1e-3) / 1e12, 2)
    out["algorithmic_bytes"] = int(36 * E + 8 * nrhs * N)
    # the 64 right-hand sides solved together to FP64 relative residual 1e-8
    # (flexible PCG per column, FP64 outer, one FP32 V-cycle for all columns),
    # against the same 64 solved one after another
    m = dg.DAMG(dg.balanceOctree(dg.points2Octree(pts, depth, 1)), inner_prec=1)
    Bd = X.double()
    m.solve_multi(Bd)
    Xs, rep = min((m.solve_multi(Bd) for _ in range(2)), key=lambda t: t[1]["solve_ms"])
    seq = 0.0
    its = []
    for j in range(nrhs):
        bj = Bd[:, j].contiguous()
        if j == 0:
            m.solve(bj)
        _, rj = m.solve(bj)
        seq += rj["solve_ms"]
        its.append(rj["iterations"])
    out["solve"] = {"nrhs": nrhs, "rtol": 1e-8, "together_ms": round(rep["solve_ms"], 3),
                    "iterations": rep["iterations"], "max_rel_residual": rep["rel_residual"],
                    "converged": rep["converged"], "one_by_one_ms": round(seq, 3),
                    "one_by_one_iterations_max": int(max(its)),
                    "speedup_together": round(seq / rep["solve_ms"], 3),
                    "method": "flexible PCG per column in FP64 around one FP32 V(2,2) cycle for all columns "
                              "(octet multi-RHS operator on every level), dense FP64 coarse solve"}
    out["method"] = {"split3/split1": "mma.sync m16n8k8 TF32, 32 right-hand sides per element pass on the warp "
                                       "tiles (split3: hi/lo TF32 split, three products), FP32 accumulation",
                     "tcgen05_split5/split4": "tcgen05.mma kind::tf32, accumulators in tensor memory: per pair of "
                                              "element parents the assembled 27 x 27 lattice matrices times the "
                                              "lattice values of 64 right-hand sides (M 128, N 64, K 32; split5: "
                                              "hi/lo split, three passes)",
                     "octet_cuda_cores": "a warp per (parent octant, 32 right-hand sides), Walsh-form element "
                                         "operators in FP32 registers, coalesced rows of X and Y"}
    return out


def cpu_baseline(octs, depth, coef, x, seconds):
    """Reference-form CPU matvec (the oracle's restatement) on the same mesh,
    timed on this host; also returns its y, the parity check of the GPU's."""
    from oracle import oracle as O
    mesh = O.Mesh(octs, depth)
    t0 = time.perf_counter()
    n = 0
    while True:
        y = mesh.matvec(x, coef)
        n += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": mesh.N * n / dt / 1e9, "unit": "GDoF/s", "cores": 1, "kind": "port",
            "sample": f"{n} full matvecs of the same mesh (E={mesh.E}, N={mesh.N}) in {dt:.1f} s, 1 thread"}, y


def rel_err(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def octree_digest(octs):
    """sha256 of the octants (x, y, z, level) as uint32, in order."""
    import hashlib
    a = np.stack([octs["x"], octs["y"], octs["z"], octs["lf"] & 31], 1).astype(np.uint32)
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def reference_y_path(workload):
    """Where the reference arm leaves one y of the compiled reference for the
    GPU arm run after it on the same host (the two arms run back to back)."""
    import tempfile
    return os.path.join(tempfile.gettempdir(), f"dendro_b200_reference_y_{workload}.f64")


def run_vcycle_profile(workload):
    """One V(2,2) cycle of the FP64 and of the FP32 hierarchy on `workload`,
    after three warm-up cycles each (operator shapes tuned per level and
    precision), bracketed by cudaProfilerStart / cudaProfilerStop; prints
    their times (CUDA events around the synchronising call)."""
    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I
    from dendro_b200.learned import vcycle
    pts, depth = build_workload(workload, 1.0)
    bal = dg.balanceOctree(dg.points2Octree(pts, depth, 1))
    out = {"workload": workload}
    for prec, name in ((0, "fp64"), (1, "fp32")):
        m = dg.DAMG(bal, inner_prec=prec, use_graph=False)
        b = torch.tensor(I.uniform_rhs(int(m.N[0]), 3), device="cuda")
        for _ in range(3):
            vcycle(m, b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.profiler.start()
        e0.record()
        vcycle(m, b)
        e1.record()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        out[name] = {"levels": m.nlevels, "elements": int(m.E[0]), "nodes": int(m.N[0]),
                     "vcycle_ms": round(e0.elapsed_time(e1), 4)}
        del m
    print(json.dumps({"vcycle_profile": out}), flush=True)


def run_cmap_profile(workload):
    """The element kernel on the compressed element map and on the raw map, FP64 then FP32, one
    launch each between cudaProfilerStart / cudaProfilerStop (for ncu --profile-from-start off),
    after a warm-up launch of each; prints their times (CUDA events)."""
    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I
    pts, depth = build_workload(workload, 1.0)
    da = dg.DA(dg.balanceOctree(dg.points2Octree(pts, depth, 1)))
    nbytes = da.compressMaps()
    A = dg.Jacobian2(da, I.sphere_coefficients(da.elementCenters()))
    shape = None
    for v in range(A.kernel_count()):
        A.set_kernel(v, 0)
        if "compressed map" in A.kernel_name(0):
            shape = v
    x64 = torch.tensor(I.uniform_rhs(da.N, 3), device="cuda")
    out = {"workload": workload, "elements": da.E, "nodes": da.N, "map_bytes_per_element": round(nbytes / da.E, 3)}
    x32 = x64.float()
    y64, y32 = torch.empty_like(x64), torch.empty_like(x32)
    runs = [(p, tag, v) for p in (0, 1) for tag, v in (("compressed", shape), ("raw", 0))]
    for prec, tag, v in runs:
        A.set_kernel(v, prec)
        A.mult(x64, y64) if prec == 0 else A.mult(x32, y32)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for prec, tag, v in runs:
        A.set_kernel(v, prec)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        A.mult(x64, y64) if prec == 0 else A.mult(x32, y32)
        e1.record()
        torch.cuda.synchronize()
        out[f"{'f64' if prec == 0 else 'f32'}_{tag}_ms"] = round(e0.elapsed_time(e1), 4)
    torch.cuda.profiler.stop()
    print(json.dumps({"cmap_profile": out}), flush=True)


def run_halo_profile(parts, workload):
    """The matvec workload's mesh split into `parts` parts by the weighted
    partition, every part on this GPU in turn: per part the launches one
    rank makes per operator application (pack of the values its peers read,
    the independent elements, the dependent elements added in place) timed
    with CUDA events after a 256 MB L2 flush (median of 20),
    beside the whole mesh's operator.  The exchange itself needs several GPUs
    and is reported as bytes per rank."""
    import statistics

    import torch

    import dendro_b200 as dg
    from dendro_b200 import inputs as I
    from dendro_b200.halo import HaloDA, HaloJacobian2
    pts, depth = build_workload(workload, 1.0)
    da = dg.DA(dg.balanceOctree(dg.points2Octree(pts, depth, 1)))
    coef = I.sphere_coefficients(da.elementCenters())
    x = torch.tensor(I.uniform_rhs(da.N, 1), device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        ts = []
        for i in range(reps):
            flush.fill_(i & 255)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return round(statistics.median(ts), 4)

    A = dg.Jacobian2(da, coef)
    y = torch.empty_like(x)
    out = {"workload": workload, "elements": da.E, "nodes": da.N, "parts": parts,
           "whole_ms": timed(lambda: A.mult(x, y)), "ranks": []}
    for r in range(parts):
        h = HaloDA(da, rank=r, nranks=parts)
        op = HaloJacobian2(h, coef)
        xl = h.local_vector(x[h.first_owned:h.first_owned + h.n_owned])
        yl = torch.zeros_like(xl)
        send = h.pack(xl)
        out["ranks"].append({
            "rank": r, "independent": len(h.independent), "dependent": len(h.dependent), "owned": h.n_owned,
            "ghosts": h.n_ghost, "send_bytes": 8 * len(h.send_idx), "recv_bytes": 8 * h.n_ghost,
            "pack_ms": timed(lambda: h.pack(xl, send)),
            "independent_ms": timed(lambda: op._independent(xl, yl)),
            "dependent_ms": timed(lambda: op._dependent(xl, yl))})
        del op, h
    print(json.dumps({"halo_profile": out}), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.vcycle_profile:
        return run_vcycle_profile(args.vcycle_profile)
    if args.cmap_profile:
        return run_cmap_profile(args.cmap_profile)
    if args.halo_profile:
        return run_halo_profile(args.halo_profile, args.workload)
    if args.impl == "reference":
        return main_reference(args, rank, world)
    if world > 1:
        import datetime

        import torch
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    r = run_dendro(args, rank, world)
    line = {
        "metric": METRIC, "value": round(r["gdofs"], 4), "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(r["ms_per_step"], 5), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded point cloud)",
        "config": {"workload": args.workload, "points": int(1048576 * args.scale), "maxDepth": r["depth"],
                   "elements": r["E"], "nodes": r["N"], "operator": "FP64 -div(a grad u)+u, a=1e4 in r<0.25",
                   "l2": "flushed between steps (256 MB write)",
                   "parallelism": "one GPU" if world == 1 else
                   f"one mesh partitioned over {world} GPUs (SFC-weighted element ranges, ghost exchange over NCCL)"},
        "roofline": {"bound": "hbm", "achieved": round(r["achieved"], 1), "peak": r["peak"], "unit": "GB/s",
                     "frac": round(r["achieved"] / r["peak"], 4),
                     "traffic": TRAFFIC.get(r["kernel"]) if args.workload == WORKLOAD and args.scale == 1.0 else None,
                     "peak_source": r["peak_kind"], "algorithmic_bytes": int(r["alg_bytes"])},
        "e2e": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r["e2e"].items()},
        "gpu_launches": args.steps,
        "partitioned": r.get("partitioned") or r.get("partitioned_one_rank"),
        "clocks": r["clocks"],
        "solve": r["solve"],
        "matvec_kernel": r["kernel"],
        "multi_rhs": r["multi"],
        "batch": r["batch"],
        "cfg1": r["cfg1"],
        "elasticity": r.get("elasticity"),
        "compressed_map": r.get("cmap"),
        "setup_s": round(r["setup_s"], 3),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        octs = r["bal"].to_numpy()
        line["cpu_baseline"], y_port = cpu_baseline(octs, r["depth"], r["coef"], r["x"], args.cpu_seconds)
        # results check on the benchmark mesh itself: the GPU's y against the
        # oracle's and, when the reference arm ran before on this host, the
        # compiled reference's Jacobian2MatMult on the same mesh and vector
        parity = {"vs_oracle_rel_err": rel_err(r["y"], y_port), "tolerance": 1e-12}
        yp = reference_y_path(args.workload)
        if os.path.exists(yp) and os.path.getsize(yp) == 8 * r["N"]:
            parity["vs_reference_rel_err"] = rel_err(r["y"], np.fromfile(yp))
        # the GPU's balanced octree against the oracle's, built from the same
        # points by the reference arm (its digest, left beside its y)
        if os.path.exists(yp + ".octree"):
            parity["octree_equals_oracle"] = open(yp + ".octree").read().strip() == octree_digest(octs)
        parity["ok"] = all(v <= 1e-12 for k, v in parity.items() if k.endswith("rel_err")) and \
            parity.get("octree_equals_oracle", True)
        line["parity"] = parity
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


REF_BIN = os.path.join(ROOT, "oracle", "_ref", "dendro_ref")
REF_STENCILS = os.path.join(ROOT, "oracle", "_ref", "stencils")


def ref_processes(mem_per_proc_gb: float = 2.0, cap: int = 64) -> int:
    """One reference process per host core, bounded by available memory."""
    cores = os.cpu_count() or 1
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) for l in f if l.startswith("MemAvailable")) / 1e6
    except Exception:
        avail = 8.0
    return max(1, min(cores, cap, int(avail * 0.6 / mem_per_proc_gb)))


def reference_cfg1(matvecs=20):
    """The small configuration on the CPU: the reference's own balance, DA
    construction and Jacobian2MatMult (the compiled reference; its OpenMP
    loops on every host core), and the oracle's restatement of the 4-level
    V(2,2) PCG solve to 1e-8 (PETSc's CG and PCMG are not in the reference
    tree).  The linear octree comes from the oracle: the reference's
    points2Octree does not finish at this size."""
    import tempfile

    from dendro_b200 import inputs as I
    from oracle import oracle as O
    pts, depth = build_workload("gauss131k_d10", 1.0)
    out = {"workload": "gauss131k_d10", "omp_threads": os.cpu_count()}
    t = time.perf_counter()
    lin = O.points2octree(pts, depth, 1)
    out["points2octree_s_port"] = round(time.perf_counter() - t, 4)
    tmp = tempfile.mkdtemp(prefix="dg_cfg1_")
    np.stack([lin["x"], lin["y"], lin["z"], lin["lf"] & 31], 1).astype(np.uint32).tofile(os.path.join(tmp, "lin.u32"))
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
    if os.path.exists(REF_BIN):
        r = subprocess.run([REF_BIN, "timings", os.path.join(tmp, "lin.u32"), str(depth)], cwd=REF_STENCILS,
                           capture_output=True, text=True, env=env, timeout=1800)
        if r.returncode == 0:
            nb, ne, tb, td = r.stderr.strip().splitlines()[-1].split()
            out.update({"balance_s": float(tb), "da_build_s": float(td), "elements": int(ne)})
    bal = O.balance(lin, depth)
    mesh = O.Mesh(bal, depth)
    x = I.uniform_rhs(mesh.N, 1)
    out["nodes"] = mesh.N
    if os.path.exists(REF_BIN):
        np.stack([bal["x"], bal["y"], bal["z"], bal["lf"] & 31], 1).astype(np.uint32).tofile(os.path.join(tmp, "bal.u32"))
        x.tofile(os.path.join(tmp, "x.f64"))
        r = subprocess.run([REF_BIN, "matvec", os.path.join(tmp, "bal.u32"), str(depth), os.path.join(tmp, "x.f64"),
                            "none", os.path.join(tmp, "y.f64"), str(matvecs)], cwd=REF_STENCILS, capture_output=True,
                           text=True, timeout=1800)
        if r.returncode == 0:
            tm = float(r.stderr.strip().splitlines()[-1])
            out["matvec_ms"] = round(1e3 * tm, 3)
            out["matvec_gdofs"] = round(mesh.N / tm / 1e9, 5)
            out["matvec_cores"] = 1
    H = O.DAMG(bal, depth, 4)
    b = I.uniform_rhs(mesh.N, 1)
    t = time.perf_counter()
    _, it, hist = H.pcg(b, 1e-8, 100)
    out["pcg_port"] = {"levels": H.nlevels, "coarse_nodes": int(H.N[-1]), "iterations": int(it),
                       "rel_residual": float(hist[-1]), "solve_s": round(time.perf_counter() - t, 3), "cores": 1}
    return out


def main_reference(args, rank, world):
    """Reference arm: the reference's own CPU operator application
    (Jacobian2MatMult over ot::DA, compiled from the reference sources into
    oracle/_ref/dendro_ref) on this host's cores, one single-threaded process
    per core on the same mesh; the oracle's restatement when that binary is
    absent.  The octree comes from the oracle (the reference's points2Octree
    does not finish on inputs of this size)."""
    if rank != 0:
        return
    import tempfile

    from dendro_b200 import inputs as I
    from oracle import oracle as O
    pts, depth = build_workload(args.workload, args.scale)
    octs = O.balance(O.points2octree(pts, depth, 1), depth)
    mesh = O.Mesh(octs, depth)
    s = 2.0 ** -(mesh.elev.astype(np.float64) - 1)
    xyz = np.stack([mesh.octs["x"][:mesh.E], mesh.octs["y"][:mesh.E], mesh.octs["z"][:mesh.E]], 1).astype(float)
    cen = xyz / 2.0 ** depth + 0.5 * s[:, None]
    coef = I.sphere_coefficients(cen)
    x = I.uniform_rhs(mesh.N, 3)
    E, N = mesh.E, mesh.N
    reps = max(1, min(args.steps, 30))
    line = {"metric": METRIC, "unit": "GDoF/s", "n_gpus": world, "higher_is_better": True, "impl": "reference",
            "dtype": "f64", "data": "synthetic (seeded point cloud)", "warmup": 1,
            "config": {"workload": args.workload, "points": int(1048576 * args.scale), "maxDepth": depth,
                       "elements": E, "nodes": N, "operator": "FP64 -div(a grad u)+u, a=1e4 in r<0.25"}}
    if os.path.exists(REF_BIN):
        procs = ref_processes()
        tmp = tempfile.mkdtemp(prefix="dg_ref_")
        np.stack([octs["x"], octs["y"], octs["z"], octs["lf"] & 31], 1).astype(np.uint32).tofile(
            os.path.join(tmp, "bal.u32"))
        x.tofile(os.path.join(tmp, "x.f64"))
        np.asarray(coef, np.float64).tofile(os.path.join(tmp, "coef.f64"))
        del mesh
        run = [subprocess.Popen([REF_BIN, "matvec", os.path.join(tmp, "bal.u32"), str(depth),
                                 os.path.join(tmp, "x.f64"), os.path.join(tmp, "coef.f64"),
                                 os.path.join(tmp, f"y{p}.f64"), str(reps)], cwd=REF_STENCILS,
                                stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True) for p in range(procs)]
        per, ok = [], []
        for p, pr in enumerate(run):
            _, err = pr.communicate()
            if pr.returncode == 0:
                per.append(float(err.strip().splitlines()[-1]))
                ok.append(p)
        if per:
            # one y of the reference: checked against the oracle here and kept
            # for the GPU arm, which runs next on this host
            y_ref = np.fromfile(os.path.join(tmp, f"y{ok[0]}.f64"))
            y_port = O.Mesh(octs, depth).matvec(x, coef)
            line["parity"] = {"oracle_vs_reference_rel_err": rel_err(y_port, y_ref), "tolerance": 1e-12}
            y_ref.tofile(reference_y_path(args.workload))
            with open(reference_y_path(args.workload) + ".octree", "w") as f:
                f.write(octree_digest(octs))
            v = sum(N / t for t in per) / 1e9
            line.update({"value": round(v, 5), "steps": reps, "ms_per_step": round(1e3 * float(np.mean(per)), 3),
                         "cpu_baseline": {"value": round(v, 5), "unit": "GDoF/s", "cores": len(per),
                                          "kind": "reference",
                                          "sample": f"{len(per)} concurrent single-threaded processes, each "
                                                    f"{reps} full Jacobian2MatMult applications on the mesh "
                                                    f"(E={E}, N={N}) after one untimed"}})
            line["e2e"] = {"value": line["value"], "unit": "GDoF/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
            if not args.no_cfg1:
                line["cfg1"] = reference_cfg1()
            print(json.dumps(line), flush=True)
            return
        mesh = O.Mesh(octs, depth)
    mesh.matvec(x, coef)  # untimed
    t0 = time.perf_counter()
    for _ in range(reps):
        mesh.matvec(x, coef)
    dt = time.perf_counter() - t0
    v = N * reps / dt / 1e9
    line.update({"value": round(v, 5), "steps": reps, "ms_per_step": round(1e3 * dt / reps, 3),
                 "cpu_baseline": {"value": round(v, 5), "unit": "GDoF/s", "cores": 1, "kind": "port",
                                  "sample": f"{reps} full matvecs of the oracle restatement, 1 thread"},
                 "e2e": {"value": round(v, 5), "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
