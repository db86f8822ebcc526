"""The two-lane packed FP32 step kernels (PFC_FLAG_PACKED): two rows, or two columns, per
thread in packed f32x2 arithmetic. They compute the same step as the one-lane kernels
with the same buffers, so every variant must match the mixed-radix kernels and the
oracle within the FP32-mixed tolerance, batch bit for bit with its plans stepped alone,
and feed the reductions and fields unchanged."""
import numpy as np
import pytest

from oracle import pfc_oracle as orc
from pfc_models_b200 import logpfc, stdpfc
from pfc_models_b200.simulation import Batch

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


SIZES = [(128, 128), (256, 256), (1024, 512), (128, 2048), (2048, 64)]


@pytest.mark.parametrize("nx,ny", SIZES)
def test_packed_variants_match_generic(nx, ny):
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.3)
    geom = stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    f0 = -0.3 + 0.05 * np.random.default_rng(nx + 3 * ny).uniform(-1, 1, (ny, nx))
    gen = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels="generic")
    gen.State.n[...] = f0
    gen.TimeSteps(8)
    ref = gen.State.n.get()
    for ee_r in (8, 16):
        for ee_c in (8, 16):
            for tile in (2, 8):
                v = {"ee_row": ee_r, "ee_col": ee_c, "row_tile": tile, "packed": 1}
                sim = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels=v)
                got = sim.plan.variant()
                assert got["fast"] == 2 and got["ee_row"] == ee_r and got["ee_col"] == ee_c, (v, got)
                sim.State.n[...] = f0
                sim.TimeSteps(8)
                assert rel_l2(sim.State.n.get() + 0.3, ref + 0.3) < 1e-5, v
                sim.plan.close()
    # one pass packed, the other one-lane (16 values per lane / 32 per thread)
    for packed, code in ((2, 3), (3, 4)):
        v = {"ee_row": 16 if packed == 2 else 32, "ee_col": 16 if packed == 3 else 32, "packed": packed}
        sim = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels=v)
        assert sim.plan.variant()["fast"] == code, v
        sim.State.n[...] = f0
        sim.TimeSteps(8)
        assert rel_l2(sim.State.n.get() + 0.3, ref + 0.3) < 1e-5, v
        sim.plan.close()


@pytest.mark.parametrize("model", ["std", "log"])
def test_packed_matches_oracle(model):
    nx, ny = 256, 128
    if model == "std":
        p = dict(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.0, dt=0.5)
        geom = stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
        sim = stdpfc.BuildB200_Simulation(stdpfc.BuildStdPFCModelParameters(**p), geom, precision="fp32",
                                          kernels={"packed": 1})
        f0 = -0.25 + 0.02 * np.random.default_rng(5).uniform(-1, 1, (ny, nx))
        field = sim.State.n
    else:
        p = dict(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
        geom = logpfc.Build2DGeometry(nx, ny, nx * 0.75, ny * 0.75)
        sim = logpfc.BuildB200_Simulation(logpfc.BuildLogPFCModelParameters(**p), geom, precision="fp32",
                                          kernels={"packed": 1})
        f0 = 0.55 + 0.05 * np.random.default_rng(5).uniform(-1, 1, (ny, nx))
        field = sim.State.phi
    assert sim.plan.variant()["fast"] == 2
    ref, rec = orc.run(model, orc.Params(**p), orc.build_geometry(nx, ny, geom.Lx, geom.Ly), f0, 200,
                       record_every=100)
    field[...] = f0
    sim.TimeSteps(200)
    got = field.get()
    mean = float(np.mean(f0))
    assert rel_l2(got - mean, ref - mean) < 2e-5
    assert float(sim.CalculateFreeEnergy()) == pytest.approx(rec[-1][1], rel=1e-6)
    assert float(np.mean(got)) == pytest.approx(mean, abs=1e-12)


def test_packed_batch_is_bit_identical():
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.25, g=0.0, dt=0.5)
    geom = stdpfc.Build2DGeometry(256, 256, 64 * np.pi, 64 * np.pi)

    def make(seed, graphs):
        s = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels={"packed": 1}, graphs=graphs)
        s.State.n[...] = -0.25 + 0.03 * np.random.default_rng(seed).uniform(-1, 1, (256, 256))
        return s

    ref = [make(i, False) for i in range(3)]
    sims = [make(i, True) for i in range(3)]
    b = Batch(sims)
    assert b.classes == 1
    b.step(37)
    for r in ref:
        r.TimeSteps(37)
    for s, r in zip(sims, ref):
        assert np.array_equal(s.State.n.get(), r.State.n.get())
    b.close()


@pytest.mark.parametrize("nx,ny", [(256, 256), (2048, 128), (8192, 32)])
def test_tma_staged_tile_matches_copies(nx, ny):
    """The packed row kernel with its tile staged by the tensor memory accelerator
    (PFC_FLAG_TMA: boxes from the tensor map of W, swizzled per tile width) steps exactly as
    with 16-byte copies, for every row tile (2 to 16 rows: no swizzle, 32-, 64-, 128-byte
    swizzle), and no bounded wait gives up."""
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.2, dt=0.3)
    geom = stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    f0 = -0.3 + 0.05 * np.random.default_rng(nx + ny).uniform(-1, 1, (ny, nx))
    for tile in (2, 4, 8, 16):
        out = []
        for tma in (0, 1):
            sim = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32",
                                              kernels={"packed": 1, "row_tile": tile, "tma": tma})
            sim.State.n[...] = f0
            sim.TimeSteps(5)
            out.append(sim.State.n.get())
            assert sim.plan.status() == 0
            sim.plan.close()
        assert np.array_equal(out[0], out[1]), tile


def test_tma_wait_runs_out_and_reports():
    """The TMA-staged row pass waits on its mbarrier a bounded number of polls. With the
    barrier made to expect 16 bytes more than the tile (pfc_test_tma_wait), the wait runs
    out, the pass leaves without computing and sets PFC_STATUS_TIMEOUT; the context stays
    usable and, with the normal count restored, a new plan steps exactly as before."""
    from pfc_models_b200 import _lib
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
    geom = stdpfc.Build2DGeometry(512, 256, 128 * np.pi, 64 * np.pi)
    f0 = -0.3 + 0.05 * np.random.default_rng(9).uniform(-1, 1, (256, 512))
    v = {"packed": 2, "ee_row": 16, "ee_col": 16, "row_tile": 8, "tma": 1}
    ref = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels=v)
    ref.State.n[...] = f0
    ref.TimeSteps(3)
    sim = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels=v)
    sim.State.n[...] = f0
    lib, h = sim.plan.lib, sim.plan.handle
    _lib.check(lib.pfc_test_tma_wait(h, 16, 1 << 12))
    sim.TimeSteps(1)
    assert sim.plan.status() & _lib.STATUS_TIMEOUT
    _lib.check(lib.pfc_test_tma_wait(h, 0, 0))
    again = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32", kernels=v)
    again.State.n[...] = f0
    again.TimeSteps(3)
    assert again.plan.status() == 0
    assert np.array_equal(again.State.n.get(), ref.State.n.get())
    with pytest.raises(_lib.PfcError):
        _lib.check(lib.pfc_test_tma_wait(h, 8, 0))
