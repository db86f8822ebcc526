"""Pin the oracle: it must reproduce the unmodified reference's outputs.

The fixtures under tests/golden/ were produced by running the reference itself
(tests/golden/make_golden.py). Two kinds of pins:

* the reference's own recorded values, copied from its test files
  (stdpfc_cpu/test_regression.py:64, logpfc_cpu/test_regression.py:28-32),
  at the reference's tolerance rtol 1e-10;
* full fields and free-energy trajectories from the fixtures, at 1e-12
  relative L2 (same FFT library, so only operation order differs).
"""
import numpy as np
import pytest

from oracle import pfc_oracle as orc

REF_STD_F200 = -0.11237092135766821          # stdpfc_cpu/test_regression.py:64
REF_LOG_F = {10: -0.5162767800170736,         # logpfc_cpu/test_regression.py:28-32
             100: -0.554845641895177,
             1000: -0.5548456430520675}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _params(c):
    return orc.Params(Gamma=c["Gamma"], beta=c["beta"], q0=c["q0"], epsilon=c["epsilon"],
                      g=c["g"], dt=c["dt"])


def _cfg(d):
    import json
    import os
    from tests.conftest import GOLDEN
    man = json.load(open(os.path.join(GOLDEN, "manifest.json")))
    return man["cases"][d]["config"]


def test_std_regression(golden):
    d, c = golden("std_regression"), _cfg("std_regression")
    geom = orc.build_geometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    n, rec = orc.run("std", _params(c), geom, d["n0"], c["steps"], c["record_every"])
    F = np.array([r[1] for r in rec])
    np.testing.assert_allclose(F, d["F"], rtol=1e-12)
    assert F[-1] == pytest.approx(REF_STD_F200, rel=1e-10)
    assert rel_l2(n, d["n_final"]) < 1e-12
    assert abs(rec[-1][2] - rec[0][2]) < 1e-12


def test_log_regression(golden):
    d, c = golden("log_regression"), _cfg("log_regression")
    geom = orc.build_geometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    sim = orc.OracleSim("log", _params(c), geom)
    sim.set_field(d["phi0"])
    done = 0
    for s, f_gold in zip(d["steps"], d["F"]):
        for _ in range(int(s) - done):
            sim.step()
        done = int(s)
        F = sim.free_energy()
        assert F == pytest.approx(float(f_gold), rel=1e-12)
        assert F == pytest.approx(REF_LOG_F[int(s)], rel=1e-10)
    assert rel_l2(sim.n, d["phi_final"]) < 1e-12
    assert sim.n.mean() == pytest.approx(c["mean"], abs=1e-12)


def test_config1_trajectory(golden):
    d, c = golden("config1"), _cfg("config1")
    geom = orc.build_geometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    psi0 = c["mean"] + c["noise"] * np.random.default_rng(c["seed"]).uniform(-1, 1, (c["Ny"], c["Nx"]))
    sim = orc.OracleSim("std", _params(c), geom)
    sim.set_field(psi0)
    for s in range(c["steps"] + 1):
        if s % c["record_every"] == 0:
            k = s // c["record_every"]
            assert sim.free_energy() == pytest.approx(float(d["F"][k]), rel=1e-11)
            if f"psi_{s}" in d:
                assert rel_l2(sim.n, d[f"psi_{s}"]) < 1e-11
        if s < c["steps"]:
            sim.step()


@pytest.mark.parametrize("family", ["std", "log"])
def test_smoke_march(golden, family):
    d, c = golden(f"smoke_{family}"), _cfg(f"smoke_{family}")
    from pfc_models_b200 import fields
    geom = orc.build_geometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    f0 = fields.GeneratePerfectCrystalInitialWithCentralVacancy(
        geom, c["mean_solid"], c["mean_vacancy"], A0=c["A0"], q0=1.0)
    sim = orc.OracleSim(family, orc.Params(Gamma=1.0, beta=c["beta"], q0=1.0, epsilon=c["epsilon"],
                                           g=c["g"], dt=c["dt"]), geom)
    sim.set_field(f0)
    F = [sim.free_energy()]
    for _ in range(c["steps"]):
        sim.step()
        F.append(sim.free_energy())
    np.testing.assert_allclose(F, d["F"], rtol=1e-12)
    assert np.all(np.diff(F) < 0)
    assert rel_l2(sim.n, d["field_final"]) < 1e-12


def test_log_noise(golden):
    d, c = golden("log_noise"), _cfg("log_noise")
    geom = orc.build_geometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    phi0 = c["mean"] + c["noise"] * np.random.default_rng(c["seed"]).uniform(-1, 1, (c["Ny"], c["Nx"]))
    n, rec = orc.run("log", _params(c), geom, phi0, c["steps"], c["record_every"])
    np.testing.assert_allclose([r[1] for r in rec], d["F"], rtol=1e-12)
    assert rel_l2(n, d["phi_final"]) < 1e-12


def test_substrate(golden):
    d, c = golden("substrate"), _cfg("substrate")
    geom = orc.build_geometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    for k in ("X", "Y", "KX", "KY", "K2"):
        np.testing.assert_array_equal(getattr(geom, k), d[k])
    lap = orc.laplacian(geom)
    np.testing.assert_array_equal(lap, d["d2_dlap"])
    A, B = orc.etd1(orc.linear_n(c["Gamma"], c["beta"], c["q0"], c["epsilon"], lap), c["dt"])
    np.testing.assert_array_equal(A, d["A"])
    np.testing.assert_array_equal(B, d["B"])
    assert B.flat[0] == c["dt"]
    np.testing.assert_array_equal(orc.gaussian(geom, 2 * np.pi), d["gauss"])


@pytest.mark.parametrize("case", ["smoke", "dipole", "tanh"])
def test_extv_oracle_reproduces_the_reference(golden, case):
    """The logpfc_extv restatement against the reference model run unmodified
    (tests/golden/make_extv_golden.py): the M it chose for every step, the field's range
    it saw, F and the mean at the recorded steps, and the fields."""
    d = golden("extv")
    g = lambda k: d[f"{case}/{k}"]  # noqa: E731
    nx, ny, lx, ly, dt, steps = g("config")
    nx, ny, steps = int(nx), int(ny), int(steps)
    geom = orc.build_geometry(nx, ny, lx, ly)
    prm = orc.Params(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=dt, smallZTol=1e-8)
    sim = orc.OracleExtv(prm, geom, V=g("V"))
    sim.set_field(g("phi0"))
    F_steps = list(g("F_step"))
    rec = list(g("record"))
    M = []
    for s in range(1, steps + 1):
        assert sim.n.min() == pytest.approx(g("phi_min")[s - 1], rel=1e-12)
        assert sim.n.max() == pytest.approx(g("phi_max")[s - 1], rel=1e-12)
        sim.step()
        M.append(sim.M)
        if s in F_steps:
            i = F_steps.index(s)
            assert sim.free_energy() == pytest.approx(g("F")[i], rel=1e-12), s
            assert float(sim.n.mean()) == pytest.approx(g("mean")[i], abs=1e-13), s
        if s in rec:
            f = g("fields")[rec.index(s)]
            assert np.linalg.norm(sim.n - f) / np.linalg.norm(f) < 1e-12, s
    np.testing.assert_allclose(M, g("M"), rtol=1e-12)
    assert sim.optimizations >= 2
