"""Long single-simulation workloads, FP32-mixed against FP64 plain.

    python -m pfc_models_b200.workloads --config polycrystal2048|logpfc1024|solidify8192 [--steps N]

polycrystal2048  stdPFC 2048^2, dx = pi/4, dt = 0.5, r = -0.3; mean -0.3 + 0.01 U[-1,1]
                 (seed 0) with 64 seeds of radius 12 dx (seed 1), 20000 steps.
logpfc1024       logPFC with beta = 0.5, eps = -0.9, g = -2, Gamma = q0 = 1, dt = 0.1 on
                 1024^2 with Lx = 108 a, Ly = 62 h (a = 4 pi/sqrt3, h = 4 pi); mean 0.55
                 (inside the eps = -0.9 coexistence window 0.2985 .. 0.6326) + 0.01 U[-1,1]
                 (seed 0), 10000 steps.
solidify8192     stdPFC 8192^2, dx = pi/4, dt = 0.5, r = -0.25, mean -0.28 with 256 seeds
                 of radius 12 dx in the noisy liquid, 10000 steps.

Each runs in both precision forms with the compensated FP64 reductions (F, mu, mean per
site) every `reduce_every` steps into a device buffer (no host round trip), and
reports site-steps/s with and without those reductions, mass drift, and the FP32-mixed
error in F against FP64.
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np

CONFIGS = {
    "polycrystal2048": dict(model="std", n=(2048, 2048), steps=20000, reduce_every=1000),
    "logpfc1024": dict(model="log", n=(1024, 1024), steps=10000, reduce_every=500),
    "solidify8192": dict(model="std", n=(8192, 8192), steps=10000, reduce_every=50),
}


def build(name, precision):
    from . import fields, logpfc, stdpfc
    nx, ny = CONFIGS[name]["n"]
    if name == "logpfc1024":
        a, h = 4 * math.pi / math.sqrt(3), 4 * math.pi
        geom = logpfc.Build2DGeometry(nx, ny, 108 * a, 62 * h)
        prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.1)
        return logpfc.BuildB200_Simulation(prm, geom, precision=precision), \
            fields.GenerateNoisyLiquid(geom, 0.55, 0.01, seed=0)
    dx = math.pi / 4
    geom = stdpfc.Build2DGeometry(nx, ny, nx * dx, ny * dx)
    r, mean, seeds = (-0.3, -0.3, 64) if name == "polycrystal2048" else (-0.25, -0.28, 256)
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=r, g=0.0, dt=0.5)
    return stdpfc.BuildB200_Simulation(prm, geom, precision=precision), \
        fields.GeneratePolycrystalInitialConditions(geom, mean, 0.01, nSeeds=seeds, radius=12 * dx, noise_seed=0,
                                                    seed=1)


def run(name, precision, steps=None, reduce_every=None):
    """Steps one workload; returns F/mu/mean every `reduce_every` steps and timings."""
    import torch
    cfg = CONFIGS[name]
    steps = cfg["steps"] if steps is None else steps
    every = min(cfg["reduce_every"] if reduce_every is None else reduce_every, steps)
    sim, ic = build(name, precision)
    plan = sim.plan
    nx, ny = cfg["n"]
    plan.set_state(ic)
    mean0 = float(sim.Reduce()[2])
    nred = steps // every
    hist = torch.empty((nred, 3), dtype=torch.float64, device=plan.device)
    s = torch.cuda.current_stream(plan.device)
    # warm-up: record the 16-step and one-step graphs of both parities outside the timed
    # region, then restart from the IC
    for n in (16, 1, 16, 1):
        plan.step(n)
    plan.set_state(ic)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for i in range(nred):
        plan.step(every)
        plan.reduce(hist[i])
    plan.step(steps - nred * every)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    # the stepping alone, for the same number of steps, from the final state
    k = min(steps, 2000)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(s)
    plan.step(k)
    e3.record(s)
    e3.synchronize()
    ms_step = e2.elapsed_time(e3) / k
    h = hist.cpu().numpy()
    sites = nx * ny
    out = {"config": name, "precision": precision, "steps": steps, "reduce_every": every,
           "site_steps_per_s": sites * steps / (ms / 1e3), "ms_total": ms,
           "site_steps_per_s_stepping_only": sites / (ms_step / 1e3), "us_per_step": 1e3 * ms_step,
           "F": h[:, 0].tolist(), "mu": h[:, 1].tolist(), "mean": h[:, 2].tolist(), "mean0": mean0,
           "mass_drift": float(np.max(np.abs(h[:, 2] - mean0)))}
    plan.close()
    return out


def compare(name, steps=None):
    r32 = run(name, "fp32", steps)
    r64 = run(name, "fp64", steps)
    F32, F64 = np.array(r32["F"]), np.array(r64["F"])
    rep = {"config": name, "steps": r32["steps"],
           "fp32": {k: r32[k] for k in ("site_steps_per_s", "site_steps_per_s_stepping_only", "us_per_step",
                                        "mass_drift")},
           "fp64": {k: r64[k] for k in ("site_steps_per_s", "site_steps_per_s_stepping_only", "us_per_step",
                                        "mass_drift")},
           "F_final": {"fp32": float(F32[-1]), "fp64": float(F64[-1])},
           "max_abs_F_diff": float(np.max(np.abs(F32 - F64))),
           "max_rel_F_diff": float(np.max(np.abs(F32 - F64) / np.maximum(np.abs(F64), 1e-300))),
           "max_abs_mu_diff": float(np.max(np.abs(np.array(r32["mu"]) - np.array(r64["mu"])))),
           "F_history_every": r32["reduce_every"], "F_fp64": r64["F"], "F_fp32": r32["F"]}
    return rep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", required=True, choices=sorted(CONFIGS))
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    rep = compare(a.config, a.steps)
    short = {k: v for k, v in rep.items() if k not in ("F_fp64", "F_fp32")}
    print(json.dumps(short), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
