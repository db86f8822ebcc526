"""Parity of the sm_100a stepper with the reference (through its pinned values and
the golden fixtures made by running it) and with the oracle on the same inputs.

Tolerances are stated per test. FP64 plain: 1e-10 relative (L2 in psi, and F)
against the reference, as the reference's own regressions use. FP32 mixed: F per
site within 1e-6 relative and mass drift within 1e-12.
"""
import json
import os

import numpy as np
import pytest

from oracle import pfc_oracle as orc
from pfc_models_b200 import fields, logpfc, stdpfc
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

REF_STD_F200 = -0.11237092135766821          # stdpfc_cpu/test_regression.py:64
REF_LOG_F = {10: -0.5162767800170736,         # logpfc_cpu/test_regression.py:28-32
             100: -0.554845641895177,
             1000: -0.5548456430520675}
MASS_TOL = 1e-12


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _cfg(name):
    return json.load(open(os.path.join(GOLDEN, "manifest.json")))["cases"][name]["config"]


def _std(c, precision="fp64", **over):
    p = dict(c, **over)
    geom = stdpfc.Build2DGeometry(Nx=p["Nx"], Ny=p["Ny"], Lx=p["Lx"], Ly=p["Ly"])
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=p.get("Gamma", 1.0), beta=p["beta"], q0=p.get("q0", 1.0),
                                            epsilon=p["epsilon"], g=p["g"], dt=p["dt"])
    return stdpfc.BuildB200_Simulation(prm, geom, precision=precision), geom


def _log(c, precision="fp64"):
    geom = logpfc.Build2DGeometry(Nx=c["Nx"], Ny=c["Ny"], Lx=c["Lx"], Ly=c["Ly"])
    prm = logpfc.BuildLogPFCModelParameters(Gamma=c.get("Gamma", 1.0), beta=c["beta"], q0=c.get("q0", 1.0),
                                            epsilon=c["epsilon"], g=c["g"], dt=c["dt"])
    return logpfc.BuildB200_Simulation(prm, geom, precision=precision), geom


# ------------------------------------------------------------------ pinned regressions
@pytest.mark.parametrize("precision,ftol", [("fp64", 1e-10), ("fp32", 1e-6)])
def test_std_regression(golden, precision, ftol):
    """stdpfc_cpu/test_regression.py:87-115: vacancy crystal, 132^2, 200 steps."""
    d, c = golden("std_regression"), _cfg("std_regression")
    sim, geom = _std(c, precision)
    sim.State.n[...] = d["n0"]
    mass_start = float(sim.State.n.mean())
    for _ in range(c["steps"]):
        sim.TimeStep()
    F = float(sim.CalculateFreeEnergy())
    assert abs(float(sim.State.n.mean()) - mass_start) < MASS_TOL
    assert F == pytest.approx(REF_STD_F200, rel=ftol)
    assert rel_l2(sim.State.n.get(), d["n_final"]) < (1e-10 if precision == "fp64" else 1e-4)
    assert sim.t == pytest.approx(c["steps"] * c["dt"])


@pytest.mark.parametrize("precision,ftol", [("fp64", 1e-10), ("fp32", 1e-6)])
def test_log_regression(golden, precision, ftol):
    """logpfc_cpu/test_regression.py:58-66: F at steps 10/100/1000, mean conserved."""
    d, c = golden("log_regression"), _cfg("log_regression")
    sim, _ = _log(c, precision)
    sim.State.phi[...] = d["phi0"]
    done = 0
    for s in c["steps"]:
        sim.TimeSteps(s - done)
        done = s
        assert float(sim.CalculateFreeEnergy()) == pytest.approx(REF_LOG_F[s], rel=ftol), s
    assert float(sim.phi.mean()) == pytest.approx(c["mean"], abs=1e-12)
    if precision == "fp64":
        assert rel_l2(sim.State.phi.get(), d["phi_final"]) < 1e-10


# ------------------------------------------------------------------ config 1 (256^2, 1000 steps)
def _config1_initial(c):
    rng = np.random.default_rng(c["seed"])
    return c["mean"] + c["noise"] * rng.uniform(-1.0, 1.0, (c["Ny"], c["Nx"]))


def test_config1_fp64(golden):
    d, c = golden("config1"), _cfg("config1")
    sim, _ = _std(c, "fp64")
    sim.State.n[...] = _config1_initial(c)
    for k, s in enumerate(d["steps"]):
        if s:
            sim.TimeSteps(c["record_every"])
        assert float(sim.CalculateFreeEnergy()) == pytest.approx(float(d["F"][k]), rel=1e-10)
        if f"psi_{s}" in d:
            assert rel_l2(sim.State.n.get(), d[f"psi_{s}"]) < 1e-10
    drift = abs(float(sim.State.n.mean()) - float(d["mean"][0]))
    assert drift < MASS_TOL


def test_config1_fp32_mixed(golden):
    """The mixed form's error against the FP64 reference: F within 1e-6 relative at every
    record, psi within 1e-3 relative L2 after 1000 steps, mass drift within 1e-12."""
    d, c = golden("config1"), _cfg("config1")
    sim, _ = _std(c, "fp32")
    sim.State.n[...] = _config1_initial(c)
    worst_f = 0.0
    for k, s in enumerate(d["steps"]):
        if s:
            sim.TimeSteps(c["record_every"])
        F, mu, mean = sim.Reduce()
        worst_f = max(worst_f, abs(F / d["F"][k] - 1))
        assert abs(mean - d["mean"][0]) < MASS_TOL
    assert worst_f < 1e-6, worst_f
    assert rel_l2(sim.State.n.get(), d["psi_1000"]) < 1e-3
    assert abs(float(sim.State.n.mean()) - float(d["mean"][0])) < MASS_TOL


# ------------------------------------------------------------------ smoke marches (264^2)
@pytest.mark.parametrize("family", ["std", "log"])
def test_smoke_march(golden, family):
    """tests/test_smoke_models.py:136-170, 261-295: F falls every step, mass holds;
    here also every F matches the reference's to 1e-10."""
    d, c = golden(f"smoke_{family}"), _cfg(f"smoke_{family}")
    sim, geom = (_std if family == "std" else _log)(c)
    f0 = fields.GeneratePerfectCrystalInitialWithCentralVacancy(geom, c["mean_solid"], c["mean_vacancy"],
                                                                A0=c["A0"], q0=1.0)
    field = sim.State.n if family == "std" else sim.State.phi
    field[...] = f0
    F, mass = [float(sim.CalculateFreeEnergy())], [float(field.mean())]
    for _ in range(c["steps"]):
        sim.TimeStep()
        F.append(float(sim.CalculateFreeEnergy()))
        mass.append(float(field.mean()))
    F = np.array(F)
    np.testing.assert_allclose(F, d["F"], rtol=1e-10)
    assert np.all(np.diff(F) < 0)
    assert np.ptp(mass) < MASS_TOL
    if family == "log":
        assert field.min() > 0
    assert rel_l2(field.get(), d["field_final"]) < 1e-10


def test_log_noise(golden):
    d, c = golden("log_noise"), _cfg("log_noise")
    sim, _ = _log(c)
    rng = np.random.default_rng(c["seed"])
    sim.State.phi[...] = c["mean"] + c["noise"] * rng.uniform(-1.0, 1.0, (c["Ny"], c["Nx"]))
    for k, s in enumerate(d["steps"]):
        if s:
            sim.TimeSteps(c["record_every"])
        assert float(sim.CalculateFreeEnergy()) == pytest.approx(float(d["F"][k]), rel=1e-10)
    assert rel_l2(sim.State.phi.get(), d["phi_final"]) < 1e-10


# ------------------------------------------------------------------ closed forms (stdpfc_cpu/test_regression.py)
A_LAT = 4 * np.pi / 3**0.5
C12, C34, C14 = (3 / 4) ** 0.5, (3 / 4) ** 0.75, (3 / 4) ** 0.25
BETA, EPSILON, G = C12 * 0.5, C12 * (-0.9 + 2 * (-2.0) + 4), C34 * (-2.0 + 2.5)
MEAN_SOLID, AMPLITUDE = C14 * (0.55 - 1), C14 * 0.19
MODE = dict(Nx=64, Ny=64, Lx=28 * A_LAT, Ly=28 * A_LAT, beta=BETA, epsilon=EPSILON, g=G, dt=0.1)


def test_free_energy_single_mode():
    """stdpfc_cpu/test_regression.py:153-174 (rel 1e-12)."""
    n_bar, amp, mode = -0.3, 0.07, 4
    sim, geom = _std(MODE)
    k = 2 * np.pi * mode / MODE["Lx"]
    sim.State.n[...] = n_bar + 2 * amp * np.cos(k * geom.X)
    expected = ((BETA / 2) * (n_bar**2 + 2 * amp**2 * (1 - k**2) ** 2) + (EPSILON / 2) * (n_bar**2 + 2 * amp**2)
                + (G / 3) * (n_bar**3 + 6 * n_bar * amp**2) + 0.25 * (n_bar**4 + 12 * n_bar**2 * amp**2 + 6 * amp**4))
    assert float(sim.CalculateFreeEnergy()) == pytest.approx(expected, rel=1e-12, abs=1e-14)


@pytest.mark.parametrize("mode", [3, 4, 5])
def test_etd_is_exact_in_the_linear_regime(mode):
    """stdpfc_cpu/test_regression.py:177-199 (rel 1e-8 over 100 steps)."""
    amp = 1e-6
    sim, geom = _std(MODE)
    k = 2 * np.pi * mode / MODE["Lx"]
    sim.State.n[...] = amp * np.cos(k * geom.X)
    linear = -k**2 * (BETA * (1 - k**2) ** 2 + EPSILON)
    sim.TimeSteps(100)
    got = float(np.abs(np.fft.rfft2(sim.State.n.get())[0, mode])) / (64 * 64 / 2)
    assert got == pytest.approx(amp * np.exp(linear * 0.1 * 100), rel=1e-8)


def _removal_offsets(mean_density):
    s = G / 3
    energy = (BETA * s * (mean_density + s / 2) + (EPSILON * s - 2 * s**3) * mean_density
              + 0.5 * EPSILON * s**2 - 1.25 * s**4)
    potential = EPSILON * s - 2 * s**3 + BETA * s
    return s, energy, potential


def test_cubic_removal_is_exact_at_fixed_field():
    """stdpfc_cpu/test_regression.py:235-270."""
    sim_a, geom = _std(MODE)
    rng = np.random.default_rng(7)
    field = MEAN_SOLID + 0.3 * np.fft.irfft2(np.fft.rfft2(rng.normal(size=geom.X.shape))
                                             * np.exp(-(geom.KX**2 + geom.KY**2)), s=geom.X.shape)
    mean_density = float(field.mean())
    s, e_off, p_off = _removal_offsets(mean_density)
    sim_b, _ = _std(MODE, epsilon=EPSILON - G**2 / 3, g=0.0)
    sim_a.State.n[...] = field
    sim_b.State.n[...] = field + s
    delta_f = float(sim_b.CalculateFreeEnergy()) - float(sim_a.CalculateFreeEnergy())
    assert delta_f == pytest.approx(e_off, rel=1e-10, abs=1e-15)
    for sim in (sim_a, sim_b):
        sim._Batch1_CalcNonlinMu()
        sim._Batch2_CalcMu_Terms()
    delta_mu = sim_b.State.mu - sim_a.State.mu
    assert np.ptp(delta_mu) < 1e-11
    assert float(delta_mu.mean()) == pytest.approx(p_off, rel=1e-9)


def test_cubic_removal_converges_as_dt_shrinks():
    """stdpfc_cpu/test_regression.py:273-300: first order in dt."""
    c = dict(Nx=132, Ny=132, Lx=14 * A_LAT, Ly=8 * 4 * np.pi, beta=BETA, epsilon=EPSILON, g=G)
    s = G / 3
    gaps = []
    for dt in (0.1, 0.05, 0.025):
        sim_a, geom = _std(c, dt=dt)
        init = fields.GeneratePerfectCrystalInitialConditions(geom, MEAN_SOLID, A0=AMPLITUDE, q0=1.0)
        sim_b, _ = _std(c, dt=dt, epsilon=EPSILON - G**2 / 3, g=0.0)
        sim_a.State.n[...] = init
        sim_b.State.n[...] = init + s
        nsteps = int(round(2.0 / dt))
        sim_a.TimeSteps(nsteps)
        sim_b.TimeSteps(nsteps)
        gaps.append(float(np.abs(sim_b.State.n.get() - (sim_a.State.n.get() + s)).max()))
    ratios = [gaps[i] / gaps[i + 1] for i in range(len(gaps) - 1)]
    assert all(r > 1.8 for r in ratios), (gaps, ratios)
    assert gaps[-1] < 1e-4


# ------------------------------------------------------------------ sizes and radices vs the oracle
SIZES = [(8, 4), (28, 24), (64, 64), (132, 132), (30, 50), (44, 26), (256, 128), (128, 256),
         (2 * 3 * 5 * 7, 2 * 11 * 13), (512, 512), (2048, 64), (64, 2048)]


@pytest.mark.parametrize("nx,ny", SIZES)
@pytest.mark.parametrize("model", ["std", "log"])
def test_sizes_against_oracle(nx, ny, model):
    """20 steps of a noisy field on grids with every supported radix; FP64 within
    1e-12 relative L2 of the oracle, FP32 mixed within 2e-5."""
    geom_o = orc.build_geometry(nx, ny, nx * 0.9, ny * 0.8)
    if model == "std":
        prm = dict(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.3, dt=0.2)
        mean = -0.2
    else:
        prm = dict(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
        mean = 0.55
    rng = np.random.default_rng(nx * 1000 + ny)
    f0 = mean + 0.05 * rng.uniform(-1, 1, (ny, nx))
    ref, _ = orc.run(model, orc.Params(**prm), geom_o, f0, 20)
    for precision, tol in (("fp64", 1e-12), ("fp32", 2e-5)):
        mod = stdpfc if model == "std" else logpfc
        geom = mod.Build2DGeometry(nx, ny, nx * 0.9, ny * 0.8)
        builder = mod.BuildStdPFCModelParameters if model == "std" else mod.BuildLogPFCModelParameters
        sim = mod.BuildB200_Simulation(builder(**prm), geom, precision=precision)
        field = sim.State.n if model == "std" else sim.State.phi
        field[...] = f0
        sim.TimeSteps(20)
        assert rel_l2(field.get() - mean, ref - mean) < tol, precision


@pytest.mark.parametrize("model", ["std", "log"])
def test_large_mixed_radix_fp32_against_oracle(model):
    """A grid of at least 2^20 sites with radices 3, 5 and 7 in FP32-mixed form runs the
    mixed-radix step kernels built for two CTAs per SM (128 registers); 20 steps within
    2e-5 relative L2 of the oracle, as the other sizes."""
    nx, ny = 1120, 1008
    geom_o = orc.build_geometry(nx, ny, nx * 0.9, ny * 0.8)
    if model == "std":
        prm = dict(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.3, dt=0.2)
        mean = -0.2
    else:
        prm = dict(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
        mean = 0.55
    f0 = mean + 0.05 * np.random.default_rng(11).uniform(-1, 1, (ny, nx))
    ref, _ = orc.run(model, orc.Params(**prm), geom_o, f0, 20)
    mod = stdpfc if model == "std" else logpfc
    builder = mod.BuildStdPFCModelParameters if model == "std" else mod.BuildLogPFCModelParameters
    sim = mod.BuildB200_Simulation(builder(**prm), mod.Build2DGeometry(nx, ny, nx * 0.9, ny * 0.8), precision="fp32")
    assert sim.plan.variant()["fast"] == 0
    field = sim.State.n if model == "std" else sim.State.phi
    field[...] = f0
    sim.TimeSteps(20)
    assert rel_l2(field.get() - mean, ref - mean) < 2e-5


# ------------------------------------------------------------------ observables and views
def test_views_and_reductions():
    """n_hat, mu, local fields and the reductions against the oracle's definitions."""
    nx = ny = 96
    geom_o = orc.build_geometry(nx, ny, 96 * np.pi / 4, 96 * np.pi / 4)
    p = orc.Params(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.5)
    rng = np.random.default_rng(5)
    f0 = -0.3 + 0.05 * rng.uniform(-1, 1, (ny, nx))
    o = orc.OracleSim("std", p, geom_o)
    o.set_field(f0)
    for _ in range(3):
        o.step()
    prev = o.n.copy()
    o.step()
    geom = stdpfc.Build2DGeometry(nx, ny, geom_o.Lx, geom_o.Ly)
    sim = stdpfc.BuildB200_Simulation(stdpfc.BuildStdPFCModelParameters(
        Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.5), geom)
    sim.State.n[...] = f0
    sim.TimeSteps(4)
    F, mu, mean = sim.Reduce()
    assert F == pytest.approx(o.free_energy(), rel=1e-12)
    assert mu == pytest.approx(o.mu_per_site(), rel=1e-12)
    assert mean == pytest.approx(f0.mean(), abs=1e-15)
    # reference semantics: n_hat, mu, local fields belong to the state at the start of the last step
    assert rel_l2(sim.State.n_hat.get(), np.fft.rfft2(prev)) < 1e-13
    o_prev = orc.OracleSim("std", p, geom_o)
    o_prev.set_field(prev)
    assert rel_l2(sim.State.mu.get(), o_prev.mu()) < 1e-12
    assert rel_l2(sim.Get_local_n(), o_prev.local_field()) < 1e-12
    local_mu = np.fft.irfft2(orc.gaussian(geom_o, 2 * np.pi) * np.fft.rfft2(o_prev.mu()), s=(ny, nx))
    assert rel_l2(sim.State.local_mu.get(), local_mu) < 1e-12
    assert rel_l2(sim.State.nonlin_mu.get(), orc.nonlin_mu("std", prev, 0.2)) < 1e-12


def test_errors_and_state_order():
    from pfc_models_b200 import _lib
    geom = stdpfc.Build2DGeometry(16, 16, 10.0, 10.0)
    sim = stdpfc.BuildB200_Simulation(stdpfc.BuildStdPFCModelParameters(dt=0.1), geom)
    with pytest.raises(_lib.PfcError) as e:
        sim.TimeStep()
    assert e.value.code == _lib.PFC_E_STATE
    with pytest.raises(_lib.PfcError):
        stdpfc.BuildB200_Simulation(stdpfc.BuildStdPFCModelParameters(dt=0.1),
                                    stdpfc.Build2DGeometry(34, 16, 10.0, 10.0))


def test_fp32_log_near_singular():
    """Mixed-precision log PFC where phi/mean - 1 < -0.875 (the FP64 log branch): a
    one-mode crystal at mean 0.3 whose troughs start at phi = 0.016. FP64 within 1e-12
    and FP32 within 2e-5 relative L2 of the oracle after 1 and 10 steps."""
    a_lat, h_lat = 4 * np.pi / 3**0.5, 4 * np.pi
    geom_o = orc.build_geometry(64, 64, 4 * a_lat, 2 * h_lat)
    prm = dict(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
    f0 = fields.GeneratePerfectCrystalInitialConditions(geom_o, 0.3, A0=0.095)
    assert f0.min() / 0.3 - 1 < -0.9
    for nsteps in (1, 10):
        ref, _ = orc.run("log", orc.Params(**prm), geom_o, f0, nsteps)
        for precision, tol in (("fp64", 1e-12), ("fp32", 2e-5)):
            geom = logpfc.Build2DGeometry(64, 64, 4 * a_lat, 2 * h_lat)
            sim = logpfc.BuildB200_Simulation(logpfc.BuildLogPFCModelParameters(**prm), geom, precision=precision)
            sim.State.phi[...] = f0
            sim.TimeSteps(nsteps)
            assert rel_l2(sim.State.phi.get(), ref) < tol, (nsteps, precision)
            assert abs(float(sim.phi.mean()) - f0.mean()) < MASS_TOL


# ------------------------------------------------------------------ power-of-two kernels vs the generic kernels
FAST_SIZES = [(64, 64), (128, 32), (64, 128), (256, 256), (512, 128), (1024, 1024), (2048, 256), (256, 2048),
              (4096, 64)]


@pytest.mark.parametrize("nx,ny", FAST_SIZES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("model", ["std", "log"])
def test_fast_kernels_match_generic(nx, ny, precision, model):
    """The specialised power-of-two step kernels against the mixed-radix kernels:
    8 steps of the same field; FP64 within 1e-13, FP32 within 1e-5 relative L2."""
    mod = stdpfc if model == "std" else logpfc
    if model == "std":
        prm = mod.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.3)
        mean = -0.3
    else:
        prm = mod.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
        mean = 0.55
    geom = mod.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    f0 = mean + 0.05 * np.random.default_rng(nx + 7 * ny).uniform(-1, 1, (ny, nx))
    out = {}
    for kernels in ("auto", "generic"):
        sim = mod.BuildB200_Simulation(prm, geom, precision=precision, kernels=kernels)
        if kernels == "auto":
            assert sim.plan.info()["fast"] == 1
        field = sim.State.n if model == "std" else sim.State.phi
        field[...] = f0
        sim.TimeSteps(8)
        out[kernels] = (field.get(), sim.Reduce())
    tol = 1e-13 if precision == "fp64" else 1e-5
    assert rel_l2(out["auto"][0] - mean, out["generic"][0] - mean) < tol
    assert out["auto"][1][0] == pytest.approx(out["generic"][1][0], rel=1e-12 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("nx,ny", [(64, 8192), (8192, 32)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fast_kernels_long_transforms(nx, ny, precision):
    """8192-point transforms (beyond the mixed-radix kernels' block size) against the
    oracle: 6 steps, FP64 within 1e-12, FP32 within 2e-5 relative L2."""
    prm = dict(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.3)
    geom_o = orc.build_geometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    f0 = -0.3 + 0.05 * np.random.default_rng(nx + ny).uniform(-1, 1, (ny, nx))
    ref, _ = orc.run("std", orc.Params(**prm), geom_o, f0, 6)
    geom = stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    sim = stdpfc.BuildB200_Simulation(stdpfc.BuildStdPFCModelParameters(**prm), geom, precision=precision)
    assert sim.plan.info()["fast"] == 1
    sim.State.n[...] = f0
    sim.TimeSteps(6)
    tol = 1e-12 if precision == "fp64" else 2e-5
    assert rel_l2(sim.State.n.get() + 0.3, ref + 0.3) < tol


VARIANT_SIZES = [(256, 256), (1024, 512), (64, 2048)]


@pytest.mark.parametrize("nx,ny", VARIANT_SIZES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_kernel_variants_match_generic(nx, ny, precision):
    """Every built variant of the power-of-two step kernels (values per thread of the
    row and column kernels, rows per CTA) against the mixed-radix kernels, 8 steps."""
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.3)
    geom = stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    f0 = -0.3 + 0.05 * np.random.default_rng(nx + ny).uniform(-1, 1, (ny, nx))
    gen = stdpfc.BuildB200_Simulation(prm, geom, precision=precision, kernels="generic")
    gen.State.n[...] = f0
    gen.TimeSteps(8)
    ref = gen.State.n.get()
    ees = (8, 16, 32) if precision == "fp32" else (8, 16)
    tol = 1e-13 if precision == "fp64" else 1e-5
    for ee_r in ees:
        for ee_c in ees:
            for tile in (1, 4, 16):
                v = {"ee_row": ee_r, "ee_col": ee_c, "row_tile": tile}
                sim = stdpfc.BuildB200_Simulation(prm, geom, precision=precision, kernels=v)
                got = sim.plan.variant()
                assert got["fast"] == 1 and got["ee_row"] == ee_r and got["ee_col"] == ee_c, (v, got)
                sim.State.n[...] = f0
                sim.TimeSteps(8)
                assert rel_l2(sim.State.n.get() + 0.3, ref + 0.3) < tol, v
                sim.plan.close()


def test_kernel_variant_errors():
    from pfc_models_b200 import _lib
    prm = stdpfc.BuildStdPFCModelParameters(epsilon=-0.3, g=0.0, dt=0.5)
    geom = stdpfc.Build2DGeometry(128, 128, 32 * np.pi, 32 * np.pi)
    for bad in ({"ee_row": 4}, {"ee_col": 64}, {"row_tile": 17}, {"row_tile": 3, "packed": 1}):
        with pytest.raises(_lib.PfcError) as e:
            stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels=bad)
        assert e.value.code == _lib.PFC_E_ARG


@pytest.mark.parametrize("nx,ny", [(256, 384), (448, 448), (224, 392), (1120, 1008)])
def test_mixed_radix_tiles_leave_no_sm_idle(nx, ny):
    """The mixed-radix kernels' row and column tiles give at least two CTAs per SM, or are
    already at their smallest (whole warps of rows, or the starting column count)."""
    import torch
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.0, dt=0.5)
    for precision in ("fp32", "fp64"):
        sim = stdpfc.BuildB200_Simulation(prm, stdpfc.Build2DGeometry(nx, ny, nx * 0.8, ny * 0.8), precision=precision,
                                          kernels="generic")
        info = sim.plan.info()
        assert info["fast"] == 0
        rows_min = max(1, 32 // info["row_threads_per_fft"])
        cols_min = max(1, 32 // info["col_threads_per_fft"])
        assert info["row_ctas"] >= 2 * n_sm or info["rows_per_cta"] == rows_min, info
        assert info["col_ctas"] >= 2 * n_sm or info["cols_per_cta"] == cols_min, info
        sim.plan.close()


MIX_SIZES = [(96, 80), (160, 112), (448, 448), (256, 384), (1792, 1792), (3072, 48)]


@pytest.mark.parametrize("nx,ny", MIX_SIZES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_register_resident_mixed_radix_against_oracle(nx, ny, precision):
    """Grids whose sides have one odd factor (3, 5 or 7 times 16 .. 512, or powers of two)
    step with the register-resident kernels (compile-time radix sequences ending in the
    odd radix); 20 steps of both models within 1e-12 (FP64) / 2e-5 (FP32-mixed) relative
    L2 of the oracle, as the other sizes. (Untuned defaults: where the run-time kernels are
    faster, the tuned table selects those instead.)"""
    geom_o = orc.build_geometry(nx, ny, nx * 0.9, ny * 0.8)
    for model in ("std", "log"):
        if model == "std":
            prm = dict(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.3, dt=0.2)
            mean = -0.2
        else:
            prm = dict(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
            mean = 0.55
        f0 = mean + 0.05 * np.random.default_rng(nx + ny).uniform(-1, 1, (ny, nx))
        ref, _ = orc.run(model, orc.Params(**prm), geom_o, f0, 20)
        mod = stdpfc if model == "std" else logpfc
        builder = mod.BuildStdPFCModelParameters if model == "std" else mod.BuildLogPFCModelParameters
        sim = mod.BuildB200_Simulation(builder(**prm), mod.Build2DGeometry(nx, ny, nx * 0.9, ny * 0.8),
                                       precision=precision, kernels="default")
        assert sim.plan.path() == "fast_mixed", (model, sim.plan.path())
        field = sim.State.n if model == "std" else sim.State.phi
        field[...] = f0
        sim.TimeSteps(20)
        tol = 1e-12 if precision == "fp64" else 2e-5
        assert rel_l2(field.get() - mean, ref - mean) < tol, model
        assert float(sim.CalculateFreeEnergy()) == pytest.approx(orc_F(model, prm, geom_o, ref), rel=1e-10 if
                                                                  precision == "fp64" else 1e-6)


def orc_F(model, prm, geom, field):
    s = orc.OracleSim(model, orc.Params(**prm), geom)
    s.set_field(field)
    return s.free_energy()


@pytest.mark.parametrize("precision,ee", [("fp32", 32), ("fp32", 16), ("fp64", 16), ("fp64", 8)])
@pytest.mark.parametrize("model", ["std", "log"])
def test_row_tile_heights_other_than_powers_of_two(precision, ee, model):
    """Row tiles of 3, 5, 6 and 7 rows (the heights that spread a grid's rows evenly over the
    SMs; the last tile of 2048 rows in 7s holds 4) partition the same row transforms as
    8-row tiles: the states are bit-identical after 12 steps, on the power-of-two and the
    odd-factor register-resident kernels."""
    for nx, ny in ((128, 2048), (96, 2048)):
        mod = stdpfc if model == "std" else logpfc
        if model == "std":
            prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.3)
            mean = -0.3
        else:
            prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
            mean = 0.55
        geom = mod.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
        f0 = mean + 0.05 * np.random.default_rng(nx + ny).uniform(-1, 1, (ny, nx))
        out = {}
        for tile in (8, 7, 6, 5, 3):
            sim = mod.BuildB200_Simulation(prm, geom, precision=precision,
                                           kernels={"ee_row": ee, "ee_col": 8, "row_tile": tile})
            v = sim.plan.variant()
            assert v["fast"] and v["row_tile"] == tile, (nx, tile, v)
            (sim.State.n if model == "std" else sim.State.phi)[...] = f0
            sim.TimeSteps(12)
            out[tile] = sim.plan.get_state().cpu().numpy()
            sim.plan.close()
        for tile in (7, 6, 5, 3):
            assert np.array_equal(out[tile], out[8]), (nx, tile)


@pytest.mark.parametrize("nx,ny", [(2560, 2560), (1792, 3584), (640, 5120)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("model", ["std", "log"])
def test_long_odd_factor_sides_against_oracle(nx, ny, precision, model):
    """Sides whose radix-5 or radix-7 pass has more than 256 butterflies (2560 = 5 x 512,
    3584 = 7 x 512, 5120 = 5 x 1024): the state upload and the fields run the run-time
    kernels built for 1024-thread blocks, the steps the register-resident kernels where the
    length allows (else the run-time ones); 12 steps within 1e-12 (FP64) / 2e-5 (FP32-mixed)
    relative L2 of the oracle."""
    geom_o = orc.build_geometry(nx, ny, nx * 0.9, ny * 0.8)
    if model == "std":
        prm = dict(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.3, dt=0.2)
        mean = -0.2
    else:
        prm = dict(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
        mean = 0.55
    f0 = mean + 0.05 * np.random.default_rng(nx + ny).uniform(-1, 1, (ny, nx))
    ref, rec = orc.run(model, orc.Params(**prm), geom_o, f0, 12, record_every=12)
    mod = stdpfc if model == "std" else logpfc
    builder = mod.BuildStdPFCModelParameters if model == "std" else mod.BuildLogPFCModelParameters
    sim = mod.BuildB200_Simulation(builder(**prm), mod.Build2DGeometry(nx, ny, nx * 0.9, ny * 0.8),
                                   precision=precision)
    info = sim.plan.info()
    assert info["row_threads_per_fft"] > 256 or info["col_threads_per_fft"] > 256, info
    field = sim.State.n if model == "std" else sim.State.phi
    field[...] = f0
    sim.TimeSteps(12)
    tol = 1e-12 if precision == "fp64" else 2e-5
    got = field.get()
    assert rel_l2(got - f0.mean(), ref - f0.mean()) < tol, sim.plan.path()
    # the reductions and the fields of these plans (Parseval and the materialising passes)
    assert float(sim.CalculateFreeEnergy()) == pytest.approx(rec[-1][1], rel=1e-10 if precision == "fp64" else 1e-6)
    from pfc_models_b200 import _lib
    o = orc.OracleSim(model, orc.Params(**prm), geom_o)
    o.set_field(ref)
    local = sim.plan.get_field(_lib.FIELD_LOCAL_N | _lib.FIELD_OF_CURRENT).cpu().numpy()
    assert rel_l2(local - f0.mean(), o.local_field() - f0.mean()) < tol
