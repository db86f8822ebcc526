"""Run a short, fixed stepper workload for profiling (ncu) or quick timing.

    python -m pfc_models_b200.profile_step --nx 2048 --ny 2048 --precision fp32 --steps 10

Builds a stdPFC plan, loads a seeded noisy-liquid field and runs `--steps` ETD1
steps, then prints the mean per-kernel device time measured with CUDA events.
Keeps the device footprint small (the plan's buffers only) so that a capture
of a few launches ends quickly.

    python -m pfc_models_b200.profile_step --nx 28 --ny 24 --precision fp64 --model log --batch 256 --steps 64

With `--batch K` it builds K plans of the grid (seeds 0 .. K-1), steps them together
through `simulation.Batch` after one warm-up step, and prints the device time per step
of the whole batch (CUDA events around the call) and the plans' step path: small FP64
mixed-radix grids take the one-CTA kernel, one launch per 2048 steps.
"""
from __future__ import annotations

import argparse
import json
import math


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--model", default="std", choices=["std", "log"])
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--batch", type=int, default=0)
    a = ap.parse_args()

    import numpy as np
    import torch

    from . import fields, logpfc, stdpfc
    mod = stdpfc if a.model == "std" else logpfc
    geom = mod.Build2DGeometry(a.nx, a.ny, a.nx * math.pi / 4, a.ny * math.pi / 4)
    if a.model == "std":
        prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
        mean = -0.3
    else:
        prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.1)
        mean = 0.55
    if a.batch > 0:
        from .simulation import Batch
        sims = []
        for k in range(a.batch):
            s = mod.BuildB200_Simulation(prm, geom, precision=a.precision)
            (s.State.n if a.model == "std" else s.State.phi)[...] = fields.GenerateNoisyLiquid(geom, mean, 0.01,
                                                                                                 seed=k)
            sims.append(s)
        b = Batch(sims)
        b.step(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        b.step(a.steps)
        e1.record()
        e1.synchronize()
        F = b.reduce()[:, 0]
        us = 1e3 * e0.elapsed_time(e1) / a.steps
        print(json.dumps({"nx": a.nx, "ny": a.ny, "precision": a.precision, "model": a.model, "steps": a.steps,
                          "batch": a.batch, "path": sims[0].plan.path(), "classes": b.classes,
                          "us_per_step": us, "site_steps_per_s": a.batch * a.nx * a.ny / (us * 1e-6),
                          "finite": bool(np.isfinite(F).all())}))
        b.close()
        return
    sim = mod.BuildB200_Simulation(prm, geom, precision=a.precision)
    field = sim.State.n if a.model == "std" else sim.State.phi
    field[...] = fields.GenerateNoisyLiquid(geom, mean, 0.01, seed=0)
    ms_r, ms_c = sim.plan.step_timed(a.steps)
    torch.cuda.synchronize()
    F = float(sim.CalculateFreeEnergy())
    print(json.dumps({"nx": a.nx, "ny": a.ny, "precision": a.precision, "model": a.model, "steps": a.steps,
                      "row_us": 1e3 * ms_r / a.steps, "col_us": 1e3 * ms_c / a.steps, "F": F,
                      "finite": bool(np.isfinite(F)), "plan": sim.plan.info()}))


if __name__ == "__main__":
    main()
