"""Run a short, fixed stepper workload for profiling (ncu) or quick timing.

    python -m pfc_models_b200.profile_step --nx 2048 --ny 2048 --precision fp32 --steps 10

Builds a stdPFC plan, loads a seeded noisy-liquid field and runs `--steps` ETD1
steps, then prints the mean per-kernel device time measured with CUDA events.
Keeps the device footprint small (the plan's buffers only) so that a capture
of a few launches ends quickly.
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
