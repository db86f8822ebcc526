"""Parity at the sizes the throughput metric is quoted on.

* The FP64 plain form against the oracle (the reference CPU stepper restated, run
  with every host core through scipy's threaded pocketfft) on the 2048^2 stdPFC
  polycrystal and the 1024^2 logPFC workloads, over their first steps, from the same
  seeded fields: psi within 1e-10 relative L2 and F per site within 1e-10 relative at
  every record (the reference's own regression tolerance,
  stdpfc_cpu/test_regression.py:64-115). These FP64 runs are the yardstick of every
  FP32-mixed statement at these sizes.
* The FP32-mixed form against the FP64 plain form on the 2048^2 polycrystal over 2000
  steps, stepped in lockstep: F per site within 1e-6 relative (observed 9e-8), mu per site
  within 1e-5 (observed 5e-8), mass drift at most 1e-12, and psi within 2e-3 relative L2
  (observed 5.2e-4: the FP32 rounding shifts the moving grain boundaries of the polycrystal
  slightly, while the quantities the phase-diagram tools consume, F and mu, agree to 1e-7).
"""
import os

import numpy as np
import pytest

from oracle import pfc_oracle as orc
from pfc_models_b200 import workloads

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("name,steps,every", [("polycrystal2048", 100, 50), ("logpfc1024", 200, 100)])
def test_fp64_plain_matches_oracle_at_full_size(name, steps, every):
    p = workloads.parameters(name)
    sim, ic = workloads.build(name, "fp64")
    geom = orc.build_geometry(p["Nx"], p["Ny"], p["Lx"], p["Ly"])
    prm = orc.Params(Gamma=p["Gamma"], beta=p["beta"], q0=p["q0"], epsilon=p["epsilon"], g=p["g"], dt=p["dt"])
    ref = orc.OracleSim(p["model"], prm, geom, fft="scipy", workers=os.cpu_count())
    ref.set_field(ic)
    field = sim.State.phi if p["model"] == "log" else sim.State.n
    field[...] = ic
    assert float(sim.CalculateFreeEnergy()) == pytest.approx(ref.free_energy(), rel=1e-12)
    done = 0
    while done < steps:
        for _ in range(every):
            ref.step()
        sim.TimeSteps(every)
        done += every
        got = field.get()
        err = rel_l2(got, ref.n)
        F, Fref = float(sim.CalculateFreeEnergy()), ref.free_energy()
        print(f"{name} step {done}: psi rel L2 {err:.3e}, F {F:.17g} vs {Fref:.17g}")
        assert err < 1e-10, (done, err)
        assert F == pytest.approx(Fref, rel=1e-10), done
        assert float(np.mean(got)) == pytest.approx(float(np.mean(ic)), abs=1e-12)


def test_fp32_mixed_tracks_fp64_on_the_polycrystal():
    r = workloads.lockstep_error("polycrystal2048", steps=2000, every=250)
    print({k: v for k, v in r.items() if k.startswith("max_")})
    print("psi rel L2 by record:", r["records"]["psi_rel_l2"])
    assert r["max_rel_F"] < 1e-6
    assert r["max_abs_mu"] < 1e-5
    assert r["max_drift32"] <= 1e-12 and r["max_drift64"] <= 1e-12
    assert r["max_psi_rel_l2"] < 2e-3
    assert np.all(np.isfinite(r["records"]["F32"]))
