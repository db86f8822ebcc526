"""Generate tests/golden/extv.npz from the reference's logpfc_extv model.

Run in a container where the reference checkout exists (it is not needed, and not
present, where the tests run):

    PFC_CUPY_STANDIN_DEVICE=cpu PYTHONPYCACHEPREFIX=<scratch dir> \
        python tests/golden/make_extv_golden.py <reference checkout>

The model (src/pfc_models/models/logpfc_extv/simulation.py) is CuPy-only; the torch-backed
`cupy` stand-in of ``baseline/cupy_standin`` runs it unmodified in FP64 on the host
(cuFFT's arithmetic replaced by torch's CPU FFT: round-off about 1e-16 relative). Every
case starts from the reference's perfect crystal with a central vacancy
(fields/initial_conditions_2d.py) and records, per step, the M the model's
ValidatePhiRange / OptimizeM chose for the step and the field's min and max before it,
plus F (CalculateFreeEnergy), the mean and the field at chosen steps.

Cases:
  smoke   the reference smoke test's configuration (tests/test_smoke_models.py:173-189):
          264^2, Lx = 28 a, Ly = 16 h, beta 0.5, eps -0.9, g -2, dt 0.1, mean 0.55 with a
          vacancy at 0.3, A0 0.15, V = 0 (the test never sets a potential), 100 steps, F
          and mean every step.
  dipole  128^2, Lx = 14 a, Ly = 8 h, same model, with the reference's Gaussian dipole
          potential (external_potentials.py SetGaussianDipolePotential: V0 0.05, poles at
          (0.3 Lx, 0.5 Ly) and (0.7 Lx, 0.5 Ly), sigma 3), 300 steps.
  tanh    96 x 112, Lx = 10 a, Ly = 7 h, with the reference's double-vacancy tanh
          potential (SetDoubleVacancyAlongX_TanhPotential: x 0.35 .. 0.65 Lx, y 0.4 ..
          0.6 Ly, widths 2 and 3, V0 0.02), dt 0.05, 400 steps.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

A = 4 * np.pi / 3**0.5
H = 4 * np.pi


def run_case(ref, fields, nx, ny, lx, ly, dt, steps, record, potential, every_F):
    import cupy as cp
    g = ref.BuildGeometry(nx, ny, lx, ly)
    prm = ref.BuildLogPFCModel_withVacancyForce_Parameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0,
                                                           dt=dt, meanDensity=0.55, V0=-1e-3, potWidth=10.0)
    sim = ref.BuildCupyGPU_Simulation(prm, g)
    phi0 = fields.GeneratePerfectCrystalInitialWithCentralVacancy(g, 0.55, 0.3, A0=0.15, q0=1.0)
    sim.State.phi[...] = cp.asarray(phi0)
    if potential is not None:
        potential(sim, g)
    V = sim._externalV.V.get()
    out = {"phi0": phi0, "V": V, "config": np.array([nx, ny, lx, ly, dt, steps], dtype=np.float64)}
    M, pmin, pmax, F, mean, Fstep = [], [], [], [], [], []
    fields_at = {}
    F.append(float(sim.CalculateFreeEnergy()))
    mean.append(float(sim.State.phi.mean()))
    Fstep.append(0)
    for s in range(1, steps + 1):
        pmin.append(float(sim.State.phi.min()))
        pmax.append(float(sim.State.phi.max()))
        sim.TimeStep()
        M.append(float(sim.State.M))
        if s % every_F == 0:
            F.append(float(sim.CalculateFreeEnergy()))
            mean.append(float(sim.State.phi.mean()))
            Fstep.append(s)
        if s in record:
            fields_at[s] = sim.State.phi.get()
    out.update(M=np.array(M), phi_min=np.array(pmin), phi_max=np.array(pmax), F=np.array(F),
               mean=np.array(mean), F_step=np.array(Fstep), record=np.array(sorted(fields_at)),
               fields=np.stack([fields_at[k] for k in sorted(fields_at)]))
    return out


def main(refdir):
    sys.path[:0] = [os.path.join(ROOT, "baseline", "cupy_standin"), os.path.join(refdir, "src")]
    from pfc_models.fields import initial_conditions_2d as fields
    from pfc_models.models.logpfc_extv import simulation as ref

    def dipole(sim, g):
        sim._externalV.SetGaussianDipolePotential(0.05, (0.3 * g.Lx, 0.5 * g.Ly), (0.7 * g.Lx, 0.5 * g.Ly), 3.0)

    def tanh(sim, g):
        sim._externalV.SetDoubleVacancyAlongX_TanhPotential(0.35 * g.Lx, 0.65 * g.Lx, 0.4 * g.Ly, 0.6 * g.Ly,
                                                            2.0, 3.0, 0.02)

    cases = {
        "smoke": run_case(ref, fields, 264, 264, 28 * A, 16 * H, 0.1, 100, {100}, None, 1),
        "dipole": run_case(ref, fields, 128, 128, 14 * A, 8 * H, 0.1, 300, {100, 300}, dipole, 50),
        "tanh": run_case(ref, fields, 96, 112, 10 * A, 7 * H, 0.05, 400, {400}, tanh, 100),
    }
    flat = {f"{c}/{k}": v for c, d in cases.items() for k, v in d.items()}
    np.savez_compressed(os.path.join(HERE, "extv.npz"), **flat)
    for c, d in cases.items():
        print(c, "F", d["F"][-1], "M changes", int(np.sum(np.diff(d["M"]) != 0)) + 1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
