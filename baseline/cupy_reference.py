"""The reference's GPU path, timed on this GPU: BASELINE INFRASTRUCTURE, not product code.

    python baseline/cupy_reference.py [--steps K] [--warmup W]

Runs the unmodified reference model `pfc_models.models.stdpfc` (its `BuildCupyGPU_Simulation`
and `TimeStep`, models/stdpfc/simulation.py:225-235 and :270-286), installed under
`baseline/_ref` by `pip install --target baseline/_ref <reference checkout>`, with the
torch-backed `cupy` stand-in of `baseline/cupy_standin` (no CuPy wheel exists here): cuFFT
through torch.fft and one device kernel per array operation, as CuPy issues them, in FP64.
Workload: the 2048^2 stdPFC polycrystal of the bench (dx = pi/4, dt = 0.5, r = -0.3, g = 0;
the same seeded field). Timed with CUDA events on the current stream around `--steps`
TimeStep() calls after `--warmup` untimed ones (cuFFT plans cached). Prints one JSON line:
site-steps/s, ms per step, the free energy after the run and how the stand-in was used.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    a = ap.parse_args()
    ref_dir = os.path.join(HERE, "_ref")
    if not os.path.isdir(os.path.join(ref_dir, "pfc_models")):
        print(json.dumps({"unavailable": "the reference is not installed under baseline/_ref"}))
        return 0
    sys.path[:0] = [os.path.join(HERE, "cupy_standin"), ref_dir, ROOT]
    import cupy as cp
    import torch
    from pfc_models.models.stdpfc import simulation as ref

    from pfc_models_b200 import workloads
    p = workloads.parameters("polycrystal2048")
    geom = ref.Build2DGeometry(p["Nx"], p["Ny"], p["Lx"], p["Ly"])
    prm = ref.BuildStdPFCModelParameters(Gamma=p["Gamma"], beta=p["beta"], q0=p["q0"], epsilon=p["epsilon"],
                                         g=p["g"], dt=p["dt"])
    sim = ref.BuildCupyGPU_Simulation(prm, geom)
    sim.State.n[...] = cp.asarray(workloads.initial_field("polycrystal2048", geom))
    for _ in range(a.warmup):
        sim.TimeStep()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(a.steps):
        sim.TimeStep()
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    F = float(sim.CalculateFreeEnergy())
    sites = p["Nx"] * p["Ny"]
    print(json.dumps({"value": sites * a.steps / (ms / 1e3), "unit": "site-steps/s", "ms_per_step": ms / a.steps,
                      "steps": a.steps, "warmup": a.warmup, "dtype": "f64", "F_after": F,
                      "after_steps": a.steps + a.warmup,
                      "kind": "reference GPU path (models/stdpfc/simulation.py, unmodified) through a torch-backed "
                              "cupy stand-in: cuFFT via torch.fft, one kernel per array operation"}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
