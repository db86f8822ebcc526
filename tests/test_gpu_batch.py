"""Batched stepping (pfc_batch_*), CUDA-graph replay of steps and programmatic
dependent launch of the step kernels.

These only change how the step kernels are launched, never what they compute, so
the results must be bit-identical to stepping each plan on its own with every
kernel launched directly and serialised.
"""
import numpy as np
import pytest

from pfc_models_b200 import _lib, logpfc, stdpfc
from pfc_models_b200.simulation import Batch

pytestmark = pytest.mark.gpu


def _std_sim(nx, ny, eps, mean, precision, seed, graphs=True, pdl=None, kernels="auto"):
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=eps, g=0.0, dt=0.5)
    geom = stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    sim = stdpfc.BuildB200_Simulation(prm, geom, precision=precision, graphs=graphs, pdl=pdl, kernels=kernels)
    sim.State.n[...] = mean + 0.05 * np.random.default_rng(seed).uniform(-1, 1, (ny, nx))
    return sim


def _log_sim(nx, ny, precision, seed, graphs=True, pdl=None, kernels="auto"):
    prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
    geom = logpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    sim = logpfc.BuildB200_Simulation(prm, geom, precision=precision, graphs=graphs, pdl=pdl, kernels=kernels)
    sim.State.phi[...] = 0.55 + 0.05 * np.random.default_rng(seed).uniform(-1, 1, (ny, nx))
    return sim


def _mixed(precision, graphs, pdl=None):
    """Six plans in four classes: 64^2 std (x2), 128^2 std (x2), 64^2 log, 128x64 std."""
    specs = [("std", 64, 64, -0.3, -0.3), ("std", 128, 128, -0.25, -0.2), ("std", 64, 64, -0.6, -0.45),
             ("log", 64, 64, None, None), ("std", 128, 64, -0.1, -0.05), ("std", 128, 128, -0.5, -0.4)]
    sims = []
    for i, (m, nx, ny, eps, mean) in enumerate(specs):
        if m == "std":
            sims.append(_std_sim(nx, ny, eps, mean, precision, seed=i, graphs=graphs, pdl=pdl))
        else:
            sims.append(_log_sim(nx, ny, precision, seed=i, graphs=graphs, pdl=pdl))
    return sims


def _field(sim):
    return (sim.State.phi if sim.model == "log" else sim.State.n).get()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_matches_individual_plans(precision):
    """37 steps (two replayed 16-step blocks and 5 direct steps) of a batch equal the
    same plans stepped one by one with serialised launches; a second call continues
    from the other parity."""
    ref = _mixed(precision, graphs=False, pdl=False)
    for s in ref:
        s.TimeSteps(37)
    sims = _mixed(precision, graphs=True, pdl=True)
    b = Batch(sims)
    assert b.classes == 4
    b.step(37)
    red = b.reduce()
    for i, (s, r) in enumerate(zip(sims, ref)):
        assert np.array_equal(_field(s), _field(r)), i
        assert s.t == pytest.approx(r.t)
        assert tuple(red[i]) == pytest.approx(r.Reduce(), rel=1e-15, abs=1e-300)
    assert b.launches() == 2 * 4 * 37
    b.step(21)
    for s in ref:
        s.TimeSteps(21)
    for s, r in zip(sims, ref):
        assert np.array_equal(_field(s), _field(r))
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_graph_replay_matches_direct_launches(precision):
    a = _std_sim(256, 128, -0.25, -0.25, precision, seed=3, graphs=True)
    d = _std_sim(256, 128, -0.25, -0.25, precision, seed=3, graphs=False)
    for n in (40, 1, 16, 33):
        a.TimeSteps(n)
        d.TimeSteps(n)
        assert np.array_equal(a.State.n.get(), d.State.n.get())
    # the count includes the launches that materialise the fields read above
    assert a.plan.launches() == d.plan.launches() >= 2 * 90


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("model", ["std", "log"])
def test_launch_modes_match_serialised_launches(precision, model):
    """A step kernel that starts while the previous one drains (griddepcontrol; both
    kernels, or the column kernel only), and column kernels of 1, 2 or 4 columns per CTA,
    give the same bits as serialised launches of the default shape, replayed from graphs or
    launched directly."""
    def make(graphs, pdl, col_cta=0, pdl_col=False):
        kernels = "auto"
        if col_cta or pdl_col:
            v = make(False, False).plan.variant()
            kernels = {"ee_row": v["ee_row"], "ee_col": v["ee_col"], "row_tile": v["row_tile"], "col_cta": col_cta,
                       "pdl": 2 if pdl_col else 0}
        if model == "std":
            return _std_sim(512, 256, -0.25, -0.25, precision, seed=5, graphs=graphs, pdl=pdl, kernels=kernels)
        return _log_sim(256, 256, precision, seed=5, graphs=graphs, pdl=pdl, kernels=kernels)
    ref = make(False, False)
    sims = [make(True, True), make(False, True), make(True, False, 1), make(True, True, 4),
            make(True, None, pdl_col=True), make(False, None, pdl_col=True)]
    assert sims[2].plan.info()["fast_col_ctas"] == sims[2].Geometry.Nx // 2    # one column per CTA
    for n in (17, 1, 32, 3):
        ref.TimeSteps(n)
        want = _field(ref)
        for s in sims:
            s.TimeSteps(n)
            assert np.array_equal(_field(s), want)
    assert all(s.Reduce() == ref.Reduce() for s in sims)


def test_batch_rejects_mixed_parity_precisions_and_repeats():
    s1 = _std_sim(64, 64, -0.3, -0.3, "fp32", seed=0)
    s2 = _std_sim(64, 64, -0.3, -0.3, "fp32", seed=1)
    s1.TimeStep()
    b = Batch([s1, s2])
    with pytest.raises(_lib.PfcError) as e:
        b.step(2)
    assert e.value.code == _lib.PFC_E_STATE
    s2.TimeStep()
    b.step(2)
    b.close()
    f64 = _std_sim(64, 64, -0.3, -0.3, "fp64", seed=0)
    with pytest.raises(_lib.PfcError) as e:
        Batch([s1, f64])
    assert e.value.code == _lib.PFC_E_ARG
    with pytest.raises(_lib.PfcError) as e:
        Batch([s1, s1])
    assert e.value.code == _lib.PFC_E_ARG


def _generic_mix(precision, graphs, pdl=None):
    """Mixed-radix and power-of-two plans in one batch: 224x392 std (x2), 96x80 log,
    448^2 std (untuned defaults: the register-resident kernels, which the tuned table
    trades for the run-time ones in FP64), and a 64^2 std forced onto the mixed-radix
    kernels next to a 64^2 std on the power-of-two ones."""
    specs = [("std", 224, 392, -0.3, -0.3, "auto"), ("std", 224, 392, -0.25, -0.2, "auto"),
             ("log", 96, 80, None, None, "auto"), ("std", 448, 448, -0.5, -0.4, "default"),
             ("std", 64, 64, -0.3, -0.3, "generic"), ("std", 64, 64, -0.3, -0.3, "auto")]
    sims = []
    for i, (mdl, nx, ny, eps, mean, kern) in enumerate(specs):
        if mdl == "std":
            sims.append(_std_sim(nx, ny, eps, mean, precision, seed=10 + i, graphs=graphs, pdl=pdl, kernels=kern))
        else:
            sims.append(_log_sim(nx, ny, precision, seed=10 + i, graphs=graphs, pdl=pdl, kernels=kern))
    return sims


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_of_mixed_radix_plans_matches_individual_plans(precision):
    """Grids with factors 3 and 7 (the phase-diagram cells' kind) batch like the
    power-of-two ones: 37 and then 21 steps equal each plan stepped on its own."""
    ref = _generic_mix(precision, graphs=False, pdl=False)
    for s in ref:
        s.TimeSteps(37)
    sims = _generic_mix(precision, graphs=True)
    # 96 x 80 and 448^2 (3 x 16, 5 x 16; 7 x 32, 7 x 64) run the register-resident kernels
    assert [s.plan.variant()["fast"] for s in sims] == [0, 0, 1, 1, 0, 1]
    b = Batch(sims)
    assert b.classes == 5
    b.step(37)
    for i, (s, r) in enumerate(zip(sims, ref)):
        assert np.array_equal(_field(s), _field(r)), i
    b.step(21)
    for s in ref:
        s.TimeSteps(21)
    for i, (s, r) in enumerate(zip(sims, ref)):
        assert np.array_equal(_field(s), _field(r)), i
    red = b.reduce()
    for i, (s, r) in enumerate(zip(sims, ref)):
        assert tuple(red[i]) == pytest.approx(r.Reduce(), rel=1e-15, abs=1e-300)
    b.close()


@pytest.mark.parametrize("kernels", ["auto", "generic"])
def test_smaller_plan_created_later_leaves_earlier_plan_launchable(kernels):
    """Kernel functions are shared between plans; a plan that needs less shared
    memory must not lower the limit an earlier, larger plan launches with."""
    prm = stdpfc.BuildStdPFCModelParameters(epsilon=-0.25, g=0.0, dt=0.5)
    big = stdpfc.BuildB200_Simulation(prm, stdpfc.Build2DGeometry(1024, 512, 256 * np.pi, 128 * np.pi),
                                      precision="fp64", kernels=kernels)
    f0 = -0.25 + 0.01 * np.random.default_rng(0).uniform(-1, 1, (512, 1024))
    big.State.n[...] = f0
    small = stdpfc.BuildB200_Simulation(prm, stdpfc.Build2DGeometry(64, 64, 16 * np.pi, 16 * np.pi),
                                        precision="fp64", kernels=kernels)
    small.State.n[...] = -0.25
    big.TimeSteps(3)
    f, mu, mean = big.Reduce()
    assert np.isfinite(f) and mean == pytest.approx(f0.mean(), abs=1e-14)
    assert big.Get_local_n().shape == (512, 1024)


def test_auto_kernels_use_the_packaged_table():
    import json
    import torch
    from pfc_models_b200 import tune
    table = json.load(open(tune.PACKAGED))
    key = f"{torch.cuda.get_device_name()}|256x256|fp32|std"
    sim = _std_sim(256, 256, -0.25, -0.25, "fp32", seed=0)
    v = sim.plan.variant()
    if key in table and tune.lookup(256, 256, _lib.FP32_MIXED, _lib.MODEL_STD) == \
            {k: int(table[key].get(k) or 0) for k in tune.VARIANT_KEYS}:
        assert (v["ee_row"], v["ee_col"]) == (table[key]["ee_row"], table[key]["ee_col"])
    assert v["fast"] == 1


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_nonfinite_member_is_flagged_alone(precision):
    """A NaN seeded on the host into one member's field: after a batch run that member's
    device status word reads PFC_STATUS_NONFINITE (set by the compensated reduction that
    met it) while every other member's reads 0, and their fields equal the same plans
    stepped alone bit for bit. The reference leaves such a NaN for its caller to find in
    f (phase_diagram/q0star.py:277-281)."""
    ref = [_std_sim(128, 128, -0.25, -0.2, precision, seed=i, graphs=False, pdl=False) for i in range(4)]
    sims = [_std_sim(128, 128, -0.25, -0.2, precision, seed=i) for i in range(4)]
    f = sims[2].State.n.get()
    f[5, 7] = np.nan
    sims[2].State.n[...] = f
    b = Batch(sims)
    b.step(37)
    red = b.reduce()
    assert [s.plan.status() for s in sims] == [0, 0, _lib.STATUS_NONFINITE, 0]
    assert np.isnan(red[2, 0]) and np.all(np.isfinite(np.delete(red, 2, axis=0)))
    for i in (0, 1, 3):
        ref[i].TimeSteps(37)
        assert np.array_equal(_field(sims[i]), _field(ref[i])), i
    b.close()
