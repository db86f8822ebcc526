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
error against FP64: F per site, mu per site, and psi in relative L2 (the two forms
stepped in lockstep from the same field, both fields compared on the device).
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


def parameters(name):
    """Model parameters and box of a workload: dict(model, Nx, Ny, Lx, Ly, Gamma, beta, q0,
    epsilon, g, dt)."""
    nx, ny = CONFIGS[name]["n"]
    if name == "logpfc1024":
        a, h = 4 * math.pi / math.sqrt(3), 4 * math.pi
        return dict(model="log", Nx=nx, Ny=ny, Lx=108 * a, Ly=62 * h, Gamma=1.0, beta=0.5, q0=1.0,
                    epsilon=-0.9, g=-2.0, dt=0.1)
    dx = math.pi / 4
    r = -0.3 if name == "polycrystal2048" else -0.25
    return dict(model="std", Nx=nx, Ny=ny, Lx=nx * dx, Ly=ny * dx, Gamma=1.0, beta=1.0, q0=1.0, epsilon=r,
                g=0.0, dt=0.5)


def initial_field(name, geom):
    """The seeded initial field of a workload on `geom` (host FP64)."""
    from . import fields
    if name == "logpfc1024":
        return fields.GenerateNoisyLiquid(geom, 0.55, 0.01, seed=0)
    dx = math.pi / 4
    mean, seeds = (-0.3, 64) if name == "polycrystal2048" else (-0.28, 256)
    return fields.GeneratePolycrystalInitialConditions(geom, mean, 0.01, nSeeds=seeds, radius=12 * dx,
                                                       noise_seed=0, seed=1)


def build(name, precision, field=None):
    """(Simulation, initial field) of a workload in one precision form; `field`, when
    given, is returned in place of generating the initial field again."""
    from . import logpfc, stdpfc
    p = parameters(name)
    mod = logpfc if p["model"] == "log" else stdpfc
    geom = mod.Build2DGeometry(p["Nx"], p["Ny"], p["Lx"], p["Ly"])
    kw = {k: p[k] for k in ("Gamma", "beta", "q0", "epsilon", "g", "dt")}
    prm = (logpfc.BuildLogPFCModelParameters(**kw) if p["model"] == "log"
           else stdpfc.BuildStdPFCModelParameters(**kw))
    return mod.BuildB200_Simulation(prm, geom, precision=precision), \
        (initial_field(name, geom) if field is None else field)


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


def lockstep_error(name, steps=None, every=None):
    """FP32-mixed against FP64 plain on one workload, both stepped in lockstep from the
    same field: at every `every` steps the relative error of F per site and the absolute
    error of mu per site (the compensated reductions), the relative L2 error of psi and of
    the deviation psi - mean (both fields materialised in FP64 on the device), and the
    mass drift of each form. Returns a dict of per-record lists and their maxima."""
    import torch
    cfg = CONFIGS[name]
    steps = cfg["steps"] if steps is None else steps
    every = min(cfg["reduce_every"] if every is None else every, steps)
    s32, ic = build(name, "fp32")
    s64, _ = build(name, "fp64")
    p32, p64 = s32.plan, s64.plan
    p32.set_state(ic)
    p64.set_state(ic)
    mean0 = float(np.mean(ic))
    f32 = torch.empty(p32.shape, dtype=torch.float64, device=p32.device)
    f64 = torch.empty_like(f32)
    rec = {"step": [], "F32": [], "F64": [], "rel_F": [], "abs_mu": [], "psi_rel_l2": [], "dev_rel_l2": [],
           "drift32": [], "drift64": []}
    done = 0
    while done < steps:
        k = min(every, steps - done)
        p32.step(k)
        p64.step(k)
        done += k
        r32 = p32.reduce().cpu().numpy()
        r64 = p64.reduce().cpu().numpy()
        p32.get_state(f32)
        p64.get_state(f64)
        diff = float(torch.linalg.vector_norm(f32 - f64))
        rec["step"].append(done)
        rec["F32"].append(float(r32[0]))
        rec["F64"].append(float(r64[0]))
        rec["rel_F"].append(abs(float(r32[0]) / float(r64[0]) - 1))
        rec["abs_mu"].append(abs(float(r32[1]) - float(r64[1])))
        rec["psi_rel_l2"].append(diff / float(torch.linalg.vector_norm(f64)))
        rec["dev_rel_l2"].append(diff / float(torch.linalg.vector_norm(f64 - float(r64[2]))))
        rec["drift32"].append(abs(float(r32[2]) - mean0))
        rec["drift64"].append(abs(float(r64[2]) - mean0))
    p32.close()
    p64.close()
    out = {"config": name, "steps": steps, "every": every, "records": rec}
    for k in ("rel_F", "abs_mu", "psi_rel_l2", "dev_rel_l2", "drift32", "drift64"):
        out["max_" + k] = float(max(rec[k]))
    return out


def compare(name, steps=None):
    r32 = run(name, "fp32", steps)
    r64 = run(name, "fp64", steps)
    F32, F64 = np.array(r32["F"]), np.array(r64["F"])
    err = lockstep_error(name, steps, r32["reduce_every"] if name != "solidify8192" else 1000)
    rep = {"config": name, "steps": r32["steps"],
           "fp32": {k: r32[k] for k in ("site_steps_per_s", "site_steps_per_s_stepping_only", "us_per_step",
                                        "mass_drift")},
           "fp64": {k: r64[k] for k in ("site_steps_per_s", "site_steps_per_s_stepping_only", "us_per_step",
                                        "mass_drift")},
           "F_final": {"fp32": float(F32[-1]), "fp64": float(F64[-1])},
           "max_abs_F_diff": float(np.max(np.abs(F32 - F64))),
           "max_rel_F_diff": float(np.max(np.abs(F32 - F64) / np.maximum(np.abs(F64), 1e-300))),
           "max_abs_mu_diff": float(np.max(np.abs(np.array(r32["mu"]) - np.array(r64["mu"])))),
           "lockstep": {k: v for k, v in err.items() if k.startswith("max_") or k == "every"},
           "F_history_every": r32["reduce_every"], "F_fp64": r64["F"], "F_fp32": r32["F"],
           "lockstep_records": err["records"]}
    return rep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", required=True, choices=sorted(CONFIGS))
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    rep = compare(a.config, a.steps)
    short = {k: v for k, v in rep.items() if k not in ("F_fp64", "F_fp32", "lockstep_records")}
    print(json.dumps(short), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
