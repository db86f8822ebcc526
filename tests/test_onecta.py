"""The one-CTA step (pfc_onecta.cu) for small FP64 mixed-radix grids against the
two-kernel step of the same plan settings (PFC_FLAG_NO_ONE_CTA): the state, the free
energy and the chemical-potential field after an odd and an even number of steps must
agree to the last bit or within 1e-15 relative (both run the same butterflies in the same
order; only the compiler's fused multiply-adds may differ), and a batch of one-CTA plans
must equal the plans stepped alone bit for bit."""
import math

import numpy as np
import pytest

from pfc_models_b200 import _lib


def test_header_declares_the_path_query(built_lib):
    lib = _lib.load()
    assert hasattr(lib, "pfc_plan_path")
    assert (_lib.PATH_MIXED_RADIX, _lib.PATH_POW2, _lib.PATH_ONE_CTA) == (0, 1, 2)
    assert _lib.FLAG_NO_ONE_CTA == 8


GRIDS = [("std", 28, 24), ("log", 28, 24), ("std", 32, 56), ("log", 48, 20)]


def _sim(model, nx, ny, one_cta, seed=0, eps=None, precision="fp64"):
    from pfc_models_b200 import logpfc, stdpfc
    mod = logpfc if model == "log" else stdpfc
    a, h = 4 * math.pi / math.sqrt(3), 4 * math.pi
    geom = mod.Build2DGeometry(nx, ny, 2 * a * nx / 28, h * ny / 24)
    if model == "log":
        prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9 if eps is None else eps,
                                                g=-2.0, dt=0.05)
        base = 0.63
    else:
        prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25 if eps is None else eps,
                                                g=0.0, dt=0.5)
        base = -0.25
    sim = mod.BuildB200_Simulation(prm, geom, precision=precision, one_cta=one_cta)
    X, Y = np.meshgrid(np.arange(nx) * geom.dx, np.arange(ny) * geom.dy)
    n0 = base + 0.2 * abs(base) * np.cos(X) * np.cos(Y / math.sqrt(3))
    field = n0 + 0.01 * abs(base) * np.random.default_rng(seed).uniform(-1, 1, n0.shape)
    getattr(sim.State, "phi" if model == "log" else "n")[...] = field
    return sim


def _close(a, b, rel=1e-15):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.max(np.abs(b)), 1e-300)
    return np.max(np.abs(a - b)) <= rel * scale * 4


@pytest.mark.gpu
@pytest.mark.parametrize("model,nx,ny", GRIDS)
def test_one_cta_step_matches_the_two_kernel_step(model, nx, ny):
    one = _sim(model, nx, ny, True)
    two = _sim(model, nx, ny, False)
    assert one.plan.path() == "one_cta" and two.plan.path() == "mixed_radix"
    for n in (37, 20, 1):
        one.TimeSteps(n)
        two.TimeSteps(n)
        s1, s2 = one.plan.get_state().cpu().numpy(), two.plan.get_state().cpu().numpy()
        assert _close(s1, s2), (model, nx, ny, n, np.max(np.abs(s1 - s2)))
        r1, r2 = one.Reduce(), two.Reduce()
        assert r1 == pytest.approx(r2, rel=1e-14, abs=1e-15)
        assert _close(one.mu.get(), two.mu.get(), rel=1e-14)


@pytest.mark.gpu
def test_one_cta_paths_and_fallbacks():
    assert _sim("std", 28, 24, True, precision="fp32").plan.path() == "mixed_radix"
    assert _sim("std", 64, 64, True).plan.path() == "pow2"
    # 36 KB spectrum: two kernels (224 = 7 x 32: the register-resident kernels)
    assert _sim("std", 224, 224, True).plan.path() == "fast_mixed"


@pytest.mark.gpu
def test_batch_of_one_cta_plans_equals_plans_alone():
    from pfc_models_b200.simulation import Batch
    eps = [-0.9, -0.8, -0.7]
    sims = [_sim("log", 28, 24, True, seed=i, eps=e) for i, e in enumerate(eps)]
    sims.append(_sim("std", 28, 24, True, seed=7))
    alone = [_sim("log", 28, 24, True, seed=i, eps=e) for i, e in enumerate(eps)] + [_sim("std", 28, 24, True, seed=7)]
    b = Batch(sims)
    assert b.classes == 2
    launches = b.launches()
    b.step(4099)          # three launches per class: 2048 + 2048 + 3
    assert b.launches() - launches == 6
    for s in alone:
        s.TimeSteps(4099)
    F = b.reduce()
    for i, (s, t) in enumerate(zip(sims, alone)):
        assert np.array_equal(s.plan.get_state().cpu().numpy(), t.plan.get_state().cpu().numpy()), i
        assert tuple(F[i]) == t.Reduce()
    b.close()


@pytest.mark.gpu
def test_batch_of_more_plans_than_sms_equals_plans_alone():
    """160 cells: more plans than the B200's 148 SMs, so the batch runs the one-CTA build
    that fits two CTAs per SM; it must still equal each plan stepped alone."""
    from pfc_models_b200.simulation import Batch
    n = 160
    sims = [_sim("log", 28, 24, True, seed=i, eps=-0.9 + 0.001 * i) for i in range(n)]
    alone = [_sim("log", 28, 24, True, seed=i, eps=-0.9 + 0.001 * i) for i in range(n)]
    b = Batch(sims)
    b.step(101)
    for s in alone:
        s.TimeSteps(101)
    for i, (s, t) in enumerate(zip(sims, alone)):
        assert np.array_equal(s.plan.get_state().cpu().numpy(), t.plan.get_state().cpu().numpy()), i
    b.close()


@pytest.mark.gpu
def test_batch_mixing_one_cta_and_two_kernel_classes_equals_plans_alone():
    """A batch with a one-CTA class (28 x 24 log) and a two-kernel class (64 x 56 std):
    its 16-step graphs hold one one-CTA launch per block next to the row and column
    launches of the other class; 37 steps equal each plan stepped alone."""
    from pfc_models_b200.simulation import Batch
    sims = [_sim("log", 28, 24, True, seed=1), _sim("std", 64, 56, True, seed=2), _sim("log", 28, 24, True, seed=3)]
    alone = [_sim("log", 28, 24, True, seed=1), _sim("std", 64, 56, True, seed=2), _sim("log", 28, 24, True, seed=3)]
    assert [s.plan.path() for s in sims] == ["one_cta", "mixed_radix", "one_cta"]
    b = Batch(sims)
    assert b.classes == 2
    b.step(37)
    for s in alone:
        s.TimeSteps(37)
    for i, (s, t) in enumerate(zip(sims, alone)):
        assert np.array_equal(s.plan.get_state().cpu().numpy(), t.plan.get_state().cpu().numpy()), i
    b.close()
