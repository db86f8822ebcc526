"""3-mode diagnostics (models/stdpfc_cpu/phase_diagram.py:178-215): the oracle's
restatement against the reference's own `diagnose` outputs (tests/golden/diagnose.npz,
made by make_diagnose_golden.py), and the device path (pfc_diagnose_modes through
diagnostics.diagnose) against the same fixtures.

Tolerances: the oracle repeats the reference's NumPy operations, so it must agree to the
last bit. The device path takes n_hat from the plan's own FFT and the deviation by
Parseval instead of an inverse FFT and a real-space difference: FP64 plan, fitness
within 1e-12 absolute and amplitudes within 1e-11 relative; FP32-mixed plan (state
held as an FP32 deviation), fitness within 1e-7 and amplitudes within 1e-5. The maxima
count is an integer and must match exactly.

Frozen-field moments (logpfc_cpu/phase_diagram.py:465-505) likewise: the oracle equal to
the reference's FrozenField (tests/golden/frozen.npz, make_frozen_golden.py), the device
moments within 1e-12 relative, and the reference test's property that f(q) equals the
free energy of the field in the box scaled by q, here within 1e-11 through this
package's own logPFC reduction. The defect screen (logpfc_cpu/phase_diagram.py:509-528):
oracle equal to the reference's, device peak count and flag exact, spread and ratio within
1e-9 relative.
"""
import ctypes
import math

import numpy as np
import pytest

from oracle import pfc_oracle as orc
from pfc_models_b200 import _lib, diagnostics


def _cases(golden):
    d = golden("diagnose")
    for name, sname in zip(d["names"], d["structures"]):
        name, sname = str(name), str(sname)
        uNx, uNy, Mx, My = (int(v) for v in d["cell_" + name])
        yield (name, sname, dict(uNx=uNx, uNy=uNy, Mx=Mx, My=My), d["field_" + name], d["result_" + name],
               tuple(float(v) for v in d["geom_" + name]))


def _sets(sname, cell):
    rows, cols, sets = diagnostics.mode_table(sname, cell)
    return [(rows[sets == s], cols[sets == s]) for s in range(3)]


def test_mode_table_scales_the_reference_kvectors():
    rows, cols, sets = diagnostics.mode_table("triangle", dict(uNx=16, uNy=28, Mx=4, My=2))
    assert list(zip(rows, cols, sets))[:4] == [(2, 4, 0), (4, 0, 0), (-4, 0, 0), (-2, 4, 0)]
    assert list(sets) == [0] * 4 + [1] * 3 + [2] * 4
    with pytest.raises(ValueError):
        diagnostics.mode_table("triangle", dict(uNx=16, uNy=28, Mx=4))


def test_oracle_matches_reference_diagnose(golden):
    n = 0
    for name, sname, cell, field, want, _ in _cases(golden):
        st = diagnostics.STRUCTURES[sname]
        cells = cell["Mx"] * cell["My"]
        if want[5]:
            with pytest.raises(IndexError):
                orc.diagnose_modes(field, _sets(sname, cell), st.amplitudeSign, cells)
            continue
        got = orc.diagnose_modes(field, _sets(sname, cell), st.amplitudeSign, cells)
        assert got == tuple(want[:5]), name
        n += 1
    assert n == 4


def test_entry_point_checks_arguments_without_touching_the_device(built_lib):
    lib = _lib.load()
    z = ctypes.c_void_p(0)
    assert lib.pfc_diagnose_modes(z, z, z, z, z, 0, 1.0, z, z) == _lib.PFC_E_ARG
    assert "null plan" in _lib.last_error()


# ---------------------------------------------------------------- GPU
def _sim(cell, geom_l, precision, field):
    from pfc_models_b200 import stdpfc
    nx, ny = cell["uNx"] * cell["Mx"], cell["uNy"] * cell["My"]
    geom = stdpfc.Build2DGeometry(nx, ny, geom_l[0], geom_l[1])
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
    sim = stdpfc.BuildB200_Simulation(prm, geom, precision=precision)
    sim.State.n[...] = field
    return sim


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol_f,tol_a", [("fp64", 1e-12, 1e-11), ("fp32", 1e-7, 1e-5)])
def test_device_diagnose_matches_reference(golden, precision, tol_f, tol_a):
    n = 0
    for name, sname, cell, field, want, geom_l in _cases(golden):
        if want[5]:
            continue
        sim = _sim(cell, geom_l, precision, field)
        d = diagnostics.diagnose(sim, sname, cell)
        assert d.fitness == pytest.approx(want[0], abs=tol_f), name
        assert d.amplitudes == pytest.approx(tuple(want[1:4]), rel=tol_a), name
        assert d.details["maxima_per_cell"] == want[4], name
        assert d.details["mean"] == pytest.approx(field.mean(), abs=1e-14 if precision == "fp64" else 1e-12)
        n += 1
    assert n == 4


@pytest.mark.gpu
def test_device_diagnose_after_steps_matches_oracle_on_the_same_field():
    """A relaxing crystal: the plan's field after 40 steps, diagnosed on the device and by
    the oracle on its host copy (the maxima count bit for bit)."""
    from pfc_models_b200 import stdpfc
    cell = dict(uNx=16, uNy=28, Mx=4, My=2)
    st = diagnostics.STRUCTURES["triangle"]
    a, h = 4 * math.pi / math.sqrt(3), 4 * math.pi
    geom = stdpfc.Build2DGeometry(64, 56, 4 * a, 2 * h)
    X = np.arange(64) * geom.dx
    Y = np.arange(56) * geom.dy
    XX, YY = np.meshgrid(X, Y)
    q = 1.0
    n0 = -0.25 + 0.15 * (np.cos(q * XX) * np.cos(q * YY / math.sqrt(3)) - 0.5 * np.cos(2 * q * YY / math.sqrt(3)))
    n0 = n0 + 0.01 * np.random.default_rng(9).uniform(-1, 1, n0.shape)
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.0, dt=0.5)
    sim = stdpfc.BuildB200_Simulation(prm, geom, precision="fp64")
    sim.State.n[...] = n0
    sim.TimeSteps(40)
    host = sim.plan.get_state().cpu().numpy()
    want = orc.diagnose_modes(host, _sets("triangle", cell), st.amplitudeSign, 8)
    d = diagnostics.diagnose(sim, "triangle", cell)
    assert d.fitness == pytest.approx(want[0], abs=1e-12)
    assert d.amplitudes == pytest.approx(want[1:4], rel=1e-11)
    assert d.details["maxima_per_cell"] == want[4]


@pytest.mark.gpu
def test_device_diagnose_raises_where_the_reference_does():
    cell = dict(uNx=2, uNy=8, Mx=8, My=4)     # 3-mode column 2 Mx = 16 > Nx / 2 = 8
    field = -0.3 + 0.01 * np.random.default_rng(0).uniform(-1, 1, (32, 16))
    sim = _sim(cell, (16 * 0.8, 32 * 0.8), "fp64", field)
    with pytest.raises(IndexError):
        diagnostics.diagnose(sim, "triangle", cell)


# ---------------------------------------------------------------- frozen field
FROZEN_CELL = dict(uNx=14, uNy=24, Mx=2, My=1)


def test_oracle_frozen_moments_match_reference(golden):
    d = golden("frozen")
    for k, (beta, g, temp) in enumerate(d["params"]):
        A, local = orc.frozen_moments(d[f"phi_{k}"], temp, g, 1.0, FROZEN_CELL)
        assert np.array_equal(A, d[f"A_{k}"])
        assert local == d[f"local_{k}"][0]


def test_frozen_field_formulas_match_reference(golden):
    d = golden("frozen")
    for k, (beta, g, temp) in enumerate(d["params"]):
        ff = diagnostics.FrozenField(d[f"A_{k}"], d[f"local_{k}"][0], beta, 1.0)
        assert [float(ff.f(q)) for q in d["qs"]] == list(d[f"f_{k}"])
        assert ff.q_opt() == d[f"qopt_{k}"][0]


@pytest.mark.gpu
def test_device_frozen_field_matches_reference(golden):
    d = golden("frozen")
    for k, (beta, g, temp) in enumerate(d["params"]):
        ff = diagnostics.frozen_field(d[f"phi_{k}"], {"beta": beta, "g": g, "v0": 1.0}, temp, FROZEN_CELL)
        assert ff.A == pytest.approx(d[f"A_{k}"], rel=1e-12)
        assert ff.local == pytest.approx(d[f"local_{k}"][0], rel=1e-13)
        assert ff.q_opt() == pytest.approx(d[f"qopt_{k}"][0], rel=1e-12)
        assert [float(ff.f(q)) for q in d["qs"]] == pytest.approx(list(d[f"f_{k}"]), rel=1e-12)


@pytest.mark.gpu
def test_frozen_f_equals_free_energy_in_the_rescaled_box(golden):
    """The reference test's property (tests/test_phase_diagram_frozen_q.py:22-34): f(q) of
    the frozen field equals the free energy of the same field in the box scaled by q; here
    F comes from this package's logPFC plan (its own reduction) and from the reference's
    adapter (the fixture)."""
    from pfc_models_b200 import logpfc
    d = golden("frozen")
    a, h = 4 * math.pi / math.sqrt(3), 4 * math.pi
    for k, (beta, g, temp) in enumerate(d["params"]):
        phi = d[f"phi_{k}"]
        ny, nx = phi.shape
        ff = diagnostics.frozen_field(phi, {"beta": beta, "g": g, "v0": 1.0}, temp, FROZEN_CELL)
        for q, f_ref in zip(d["qs"], d[f"f_adapter_{k}"]):
            prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=beta, q0=1.0, epsilon=temp, g=g, dt=0.01)
            geom = logpfc.Build2DGeometry(nx, ny, FROZEN_CELL["Mx"] * a / q, FROZEN_CELL["My"] * h / q)
            sim = logpfc.BuildB200_Simulation(prm, geom, precision="fp64")
            sim.State.phi[...] = phi
            F = float(sim.CalculateFreeEnergy())
            assert float(ff.f(q)) == pytest.approx(F, rel=1e-11, abs=1e-12)
            assert F == pytest.approx(f_ref, rel=1e-11, abs=1e-12)


# ---------------------------------------------------------------- defect screen
def _defect_cases(d):
    for k in range(3):
        yield f"phi_{k}", d[f"phi_{k}"], d[f"defect_{k}"]
    for name in ("clean", "vacancy"):
        yield name, d[f"dfield_{name}"], d[f"dres_{name}"]


def test_oracle_defect_screen_matches_reference(golden):
    d = golden("frozen")
    flags = []
    for name, phi, want in _defect_cases(d):
        assert orc.defect_screen(phi, FROZEN_CELL) == (want[0], want[1], int(want[2])), name
        flags.append(bool(want[3]))
    assert flags == [False, False, False, False, True]    # the vacancy is the one flagged


@pytest.mark.gpu
def test_device_defect_screen_matches_reference(golden):
    """Peak count and flag exactly; spread and sub-q ratio within 1e-9 relative, or 1e-12
    absolute where the reference's value is round-off (the clean ansatz)."""
    d = golden("frozen")
    for name, phi, want in _defect_cases(d):
        dd = diagnostics.defect_diagnostics(phi, FROZEN_CELL)
        assert dd["n_peaks"] == int(want[2]), name
        assert dd["defect_flag"] == bool(want[3]), name
        assert dd["peak_spread"] == pytest.approx(want[0], rel=1e-9, abs=1e-12), name
        assert dd["subq_ratio"] == pytest.approx(want[1], rel=1e-9, abs=1e-12), name
