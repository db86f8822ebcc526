"""Log PFC with an external potential (the reference's logpfc_extv model) on B200, FP64,
against the reference model run unmodified (fixtures of tests/golden/make_extv_golden.py)
and the oracle's restatement: the M chosen before every step, the field's range, F and
the mean at the recorded steps (1e-10 relative) and the fields (1e-10 relative L2); plus
the reference smoke test's behaviour (tests/test_smoke_models.py:173-189: 100 steps of the
264^2 crystal, finite F, positive field, mass conserved to 1e-12)."""
import numpy as np
import pytest

from pfc_models_b200 import _lib, logpfc_extv

pytestmark = pytest.mark.gpu


def _build(d, case):
    g = lambda k: d[f"{case}/{k}"]  # noqa: E731
    nx, ny, lx, ly, dt, steps = g("config")
    geom = logpfc_extv.BuildGeometry(int(nx), int(ny), lx, ly)
    prm = logpfc_extv.BuildLogPFCModel_withVacancyForce_Parameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9,
                                                                   g=-2.0, dt=dt, meanDensity=0.55, V0=-1e-3,
                                                                   potWidth=10.0)
    sim = logpfc_extv.BuildCupyGPU_Simulation(prm, geom)
    sim.State.phi[...] = g("phi0")
    if np.any(g("V") != 0):
        sim._externalV.SetPotential(1.0, g("V"))
    return sim, g, int(steps)


@pytest.mark.parametrize("case", ["smoke", "dipole", "tanh"])
def test_extv_matches_the_reference(golden, case):
    d = golden("extv")
    sim, g, steps = _build(d, case)
    assert sim.plan.path() == "mixed_radix"
    F_steps = list(g("F_step"))
    rec = list(g("record"))
    M = []
    for s in range(1, steps + 1):
        sim.TimeStep()
        st = sim.State._read()
        M.append(st[0])
        assert st[3] == pytest.approx(g("phi_min")[s - 1], rel=1e-10), s
        assert st[4] == pytest.approx(g("phi_max")[s - 1], rel=1e-10), s
        if s in F_steps:
            i = F_steps.index(s)
            assert float(sim.CalculateFreeEnergy()) == pytest.approx(g("F")[i], rel=1e-10), s
            assert float(sim.State.phi.mean()) == pytest.approx(g("mean")[i], abs=1e-12), s
        if s in rec:
            f = g("fields")[rec.index(s)]
            got = sim.State.phi.get()
            assert np.linalg.norm(got - f) / np.linalg.norm(f) < 1e-10, s
    np.testing.assert_allclose(M, g("M"), rtol=1e-10)
    assert sim.State.optimizations == len(set(g("M")))


def test_extv_smoke_behaviour(golden):
    d = golden("extv")
    sim, g, _ = _build(d, "smoke")
    m0 = float(sim.State.phi.mean())
    F = [float(sim.CalculateFreeEnergy())]
    for _ in range(100):
        sim.TimeStep()
        F.append(float(sim.CalculateFreeEnergy()))
    phi = sim.State.phi.get()
    assert np.all(np.isfinite(F)) and phi.min() > 0
    assert abs(float(phi.mean()) - m0) < 1e-12
    assert sim.State.M != 0 and sim.State.phi_min is not None


def test_extv_refuses_other_forms():
    from pfc_models_b200 import logpfc
    from pfc_models_b200.simulation import Simulation
    geom = logpfc.Build2DGeometry(64, 64, 50.0, 50.0)
    prm = logpfc.BuildLogPFCModelParameters(beta=0.5, epsilon=-0.9, g=-2.0, dt=0.1)
    for precision, clamp in (("fp32", True), ("fp64", False)):
        with pytest.raises(_lib.PfcError) as e:
            Simulation("log", prm, geom, precision=precision, clamp_log=clamp, _flags=_lib.FLAG_EXTV)
        assert e.value.code == _lib.PFC_E_ARG
    sim = logpfc.Simulation(prm, geom, precision="fp64", clamp_log=True)
    v = np.zeros(64 * 64)
    import torch
    dv = torch.as_tensor(v, device="cuda")
    with pytest.raises(_lib.PfcError):
        _lib.check(sim.plan.lib.pfc_set_potential(sim.plan.handle, dv.data_ptr(), None))
