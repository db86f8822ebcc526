"""Batched stdPFC phase-diagram sweep and its common-tangent feed.

    python -m pfc_models_b200.sweep [--steps 5000] [--precision fp32,fp64] [--out sweep.json]

The workload: r = linspace(-0.6, -0.05, 16) x mean psi = linspace(-0.6, 0, 32), 512
independent simulations (Gamma = beta = q0 = 1, g = 0, epsilon = r, dt = 0.5). Each
point's box holds a whole number of cells of the triangular lattice, a = 4 pi/sqrt 3
by h = 4 pi (the adapter's `_box` at q00 = 1, models/stdpfc_cpu/phase_diagram.py:161-167):
128^2 with (Mx, My) = (14, 8), 256^2 with (28, 16) or 512^2 with (56, 32), chosen per
point by numpy default_rng(2). Even-numbered points start from the one-mode
triangular profile psi + A (cos(qx) cos(qy/sqrt3) - cos(2qy/sqrt3)/2), q = sqrt3/2,
A = 0.5; odd-numbered points from the liquid psi + 0.01 U[-1, 1]. All points step
together through one `Batch` (one launch per box size and pass, CUDA graphs over
blocks of steps); F and mu per site come from the compensated FP64 device
reductions. Where the reference runs these relaxations one at a time through
`adapter.step` (phase_diagram/q0star.py:261-307), this steps them all at once.

Under torchrun the points are dealt round-robin to the ranks (one GPU each, no
collective on the data path) and the per-point results are gathered on rank 0.

`coexistence` feeds the results to the common-tangent construction (tangent.py):
per r, the analytic liquid branch against the tabulated solid branch made of the
crystal-start points that stayed crystalline.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import asdict, dataclass

import numpy as np

R_VALUES = np.linspace(-0.6, -0.05, 16)
PSI_VALUES = np.linspace(-0.6, 0.0, 32)
BOXES = ((128, 14, 8), (256, 28, 16), (512, 56, 32))   # (n, Mx, My)
A_CELL, H_CELL = 4 * math.pi / math.sqrt(3), 4 * math.pi
Q_ONE_MODE, A_ONE_MODE = math.sqrt(3) / 2, 0.5
DT = 0.5


@dataclass
class SweepPoint:
    index: int
    r: float
    psi: float
    n: int          # n x n grid
    mx: int
    my: int
    start: str      # "crystal" or "liquid"

    @property
    def lx(self):
        return self.mx * A_CELL

    @property
    def ly(self):
        return self.my * H_CELL


def sweep_points(r_values=R_VALUES, psi_values=PSI_VALUES, seed=2, boxes=BOXES):
    """The sweep's points, r-major (index = i_r * len(psi) + i_psi)."""
    rng = np.random.default_rng(seed)
    pick = rng.integers(0, len(boxes), size=len(r_values) * len(psi_values))
    out = []
    for ir, r in enumerate(r_values):
        for ip, psi in enumerate(psi_values):
            i = ir * len(psi_values) + ip
            n, mx, my = boxes[int(pick[i])]
            out.append(SweepPoint(i, float(r), float(psi), n, mx, my, "crystal" if i % 2 == 0 else "liquid"))
    return out


def initial_field(p: SweepPoint, noise_seed=0):
    """(n, n) FP64 initial state of a point."""
    x = np.arange(p.n) * (p.lx / p.n)
    y = np.arange(p.n) * (p.ly / p.n)
    X, Y = np.meshgrid(x, y)
    if p.start == "crystal":
        q = Q_ONE_MODE
        return p.psi + A_ONE_MODE * (np.cos(q * X) * np.cos(q * Y / math.sqrt(3)) - 0.5 * np.cos(2 * q * Y / math.sqrt(3)))
    rng = np.random.default_rng([noise_seed, p.index])
    return p.psi + 0.01 * rng.uniform(-1.0, 1.0, size=X.shape)


def shard(points, rank, world):
    return points[rank::world]


def run_points(points, steps, precision="fp32", block=1000, device=None, settle=500, warmup=0, mark=None,
               engine="batch"):
    """Steps the points together on one GPU; returns (per-point results, timing).
    F is also reduced `settle` steps before the end (F_prev), so that states still
    evolving can be told from settled ones. `warmup` untimed steps come first (the
    batch's graphs are recorded there); the results then belong to warmup + steps.
    `mark(True)` / `mark(False)` are called around each timed block (a clock sampler).
    `engine`: "batch" (a `Batch`: one launch per size class and pass, classes on concurrent
    streams, plans with the batch-tuned kernel variants) or "queue" (a `QueueBatch`: one
    persistent launch per block of steps over a device work list, plans with the variants
    of `queue_kernels`)."""
    import torch

    from . import stdpfc
    from .simulation import Batch, QueueBatch, queue_kernels
    from . import _lib, tune
    from .simulation import _PRECISIONS
    sims = []
    for p in points:
        prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=p.r, g=0.0, dt=DT)
        if engine == "queue":
            variant = queue_kernels(p.n, p.n, precision)
        else:
            # the kernel variant measured for batches of this box size, if there is one
            variant = tune.lookup(p.n, p.n, _PRECISIONS[precision], _lib.MODEL_STD, batched=True) or "auto"
        sim = stdpfc.BuildB200_Simulation(prm, stdpfc.Build2DGeometry(p.n, p.n, p.lx, p.ly), precision=precision,
                                          device=device, kernels=variant)
        sim.State.n[...] = initial_field(p)
        sims.append(sim)
    batch = QueueBatch(sims) if engine == "queue" else Batch(sims)
    dev = sims[0].plan.device
    s = torch.cuda.current_stream(dev)
    if warmup:
        batch.step(warmup)
        torch.cuda.synchronize(dev)
    done, ms = 0, 0.0
    settle = min(settle, steps)
    red_prev = None
    while done < steps:
        if done == steps - settle:
            red_prev = batch.reduce()
        k = min(block, steps - done)
        if done < steps - settle:
            k = min(k, steps - settle - done)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if mark:
            mark(True)
        e0.record(s)
        batch.step(k)
        e1.record(s)
        e1.synchronize()
        if mark:
            mark(False)
        ms += e0.elapsed_time(e1)
        done += k
    red = batch.reduce()
    launches = batch.launches()
    classes = batch.classes
    status = batch.status() if engine == "queue" else 0
    batch.close()
    for sim in sims:
        sim.plan.close()
    sites = sum(p.n * p.n for p in points)
    if red_prev is None:
        red_prev = np.full_like(red, np.nan)
    res = [dict(asdict(p), F=float(red[i, 0]), mu=float(red[i, 1]), mean=float(red[i, 2]),
                F_prev=float(red_prev[i, 0]), settle=settle)
           for i, p in enumerate(points)]
    timing = {"steps": steps, "ms": ms, "sites": sites, "site_steps_per_s": sites * steps / (ms / 1e3),
              "launches": launches, "classes": classes, "points": len(points), "engine": engine}
    if status:
        raise RuntimeError(f"work-queue batch status {status}: a bounded wait gave up")
    return res, timing


def run_sweep(steps=5000, precision="fp32", points=None, block=1000, engine="batch"):
    """The sweep on every rank of the process group (or alone); results gathered on
    every rank, sorted by point index; timing is the max over ranks."""
    import torch.distributed as dist
    points = sweep_points() if points is None else points
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    res, timing = run_points(shard(points, rank, world), steps, precision, block, engine=engine)
    if world > 1:
        res, timing = gather_results(res, timing, world)
    return sorted(res, key=lambda d: d["index"]), timing


def gather_results(res, timing, world):
    """All ranks' per-point results and the slowest rank's time (host objects)."""
    import torch.distributed as dist
    allres, alltime = [None] * world, [None] * world
    dist.all_gather_object(allres, res)
    dist.all_gather_object(alltime, timing)
    merged = [d for part in allres for d in part]
    ms = max(t["ms"] for t in alltime)
    sites = sum(t["sites"] for t in alltime)
    steps = alltime[0]["steps"]
    return merged, {"steps": steps, "ms": ms, "sites": sites, "site_steps_per_s": sites * steps / (ms / 1e3),
                    "launches": sum(t["launches"] for t in alltime), "ranks": world,
                    "points": sum(t["points"] for t in alltime)}


def liquid_f(r, psi):
    return 0.5 * (1.0 + r) * psi ** 2 + 0.25 * psi ** 4


def is_crystal(d, tol=1e-6):
    """The relaxed state is not uniform: its F differs from the uniform liquid's."""
    return abs(d["F"] - liquid_f(d["r"], d["mean"])) > tol


def is_settled(d, tol=1e-9):
    """F changed by at most tol per site over the last `settle` steps."""
    return abs(d["F"] - d.get("F_prev", float("nan"))) <= tol


def solid_run(points, tol=5e-3):
    """The crystal branch next to the liquid: from the lowest-density crystalline
    point upwards, the points whose F table is consistent with their measured mu
    (|dF/dpsi - mean of the two mu| <= tol between neighbours). A state that left
    the triangular phase (stripes, defects, still evolving) breaks that consistency;
    one such point is skipped, two in a row end the run."""
    pts = sorted(points, key=lambda d: d["mean"])
    if not pts:
        return []
    run, k, misses = [pts[0]], 1, 0
    while k < len(pts):
        a, b = run[-1], pts[k]
        slope = (b["F"] - a["F"]) / (b["mean"] - a["mean"])
        if abs(slope - 0.5 * (a["mu"] + b["mu"])) <= tol:
            run.append(b)
            misses = 0
        else:
            misses += 1
            if misses == 2:
                break
        k += 1
    return run


def coexistence(results, min_points=3, extend=0.5):
    """Per r: liquid-solid coexistence densities from the common tangent between the
    analytic liquid and the solid run (F and mu per site, cubic Hermite), or NaN.
    The solid branch may be continued `extend` density spacings below its lowest
    point (crystals just below the coexistence density can melt within the run) when
    its first two points are neighbours on the density grid; tangents further out are
    not reported."""
    from . import tangent
    out = []
    for r in sorted({d["r"] for d in results}):
        sol = solid_run([d for d in results
                         if d["r"] == r and d["start"] == "crystal" and is_crystal(d) and is_settled(d)])
        row = {"r": r, "solid_points": len(sol), "psi_l": float("nan"), "psi_s": float("nan"),
               "mu": float("nan")}
        if len(sol) >= min_points:
            try:
                # continue below the lowest point only on a first interval between neighbouring
                # points of the density grid (the Hermite cubic there uses just those two)
                gaps = np.diff([d["mean"] for d in sol])
                h = float(np.min(gaps))
                ext = extend * h if gaps[0] <= 1.5 * h else 0.0
                br = tangent.tabulated_branch("solid", [d["mean"] for d in sol], [d["F"] for d in sol], min_points,
                                              mu=[d["mu"] for d in sol], extend_lo=ext)
                t = tangent.common_tangent(tangent.std_liquid_branch(r, -1.0, 0.5), br)
                # report it only where the solid branch at psi_s rests on two neighbouring
                # grid points (a cubic across a gap is too loose a fit)
                means = np.array([d["mean"] for d in sol])
                j = int(np.clip(np.searchsorted(means, t.phi_b) - 1, 0, len(means) - 2)) if t.ok else 0
                if t.ok and means[j + 1] - means[j] <= 1.5 * h:
                    row.update(psi_l=t.phi_a, psi_s=t.phi_b, mu=t.mu)
            except ValueError:
                pass
        out.append(row)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--block", type=int, default=1000)
    ap.add_argument("--out", default=None)
    ap.add_argument("--engine", default="batch", choices=["batch", "queue"])
    a = ap.parse_args()
    import os

    import torch
    import torch.distributed as dist
    if "RANK" in os.environ and int(os.environ.get("WORLD_SIZE", "1")) > 1:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl")
    rank = dist.get_rank() if dist.is_initialized() else 0
    report = {}
    for precision in a.precision.split(","):
        t0 = time.time()
        res, timing = run_sweep(a.steps, precision, block=a.block, engine=a.engine)
        timing["wall_s"] = time.time() - t0
        coex = coexistence(res)
        report[precision] = {"timing": timing, "coexistence": coex, "points": res}
        if rank == 0:
            print(json.dumps({"precision": precision, **timing}), flush=True)
            for c in coex:
                print(json.dumps(c), flush=True)
    if rank == 0 and len(report) > 1 and "fp32" in report and "fp64" in report:
        d = [abs(x[k] - y[k]) for x, y in zip(report["fp32"]["coexistence"], report["fp64"]["coexistence"])
             for k in ("psi_l", "psi_s") if np.isfinite(x[k]) and np.isfinite(y[k])]
        dF = max(abs(x["F"] - y["F"]) for x, y in zip(report["fp32"]["points"], report["fp64"]["points"]))
        print(json.dumps({"max_coexistence_diff_fp32_vs_fp64": max(d) if d else None,
                          "tangents": len(d) // 2, "max_F_diff": dF}), flush=True)
    if rank == 0 and a.out:
        with open(a.out, "w") as f:
            json.dump(report, f, indent=1)
    if dist.is_initialized():
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
