"""The work-queue batch (pfc_queue_*): the members' row and column tiles of a block of steps
as the items of one persistent, cooperative launch, each item waiting only for its own
member's tiles.

It changes how the step bodies are scheduled, never what they compute, so the members
must come out bit-identical to the same plans stepped alone. The bounded waits are
exercised without any fault: a test hook makes one item wait for a completion that never
comes, and the launch must end with PFC_STATUS_TIMEOUT and leave the device usable.
"""
import numpy as np
import pytest

from pfc_models_b200 import _lib, logpfc, stdpfc
from pfc_models_b200.simulation import Batch, QueueBatch, queue_kernels

pytestmark = pytest.mark.gpu

# (nx, ny, epsilon, mean): every row length 64 .. 1024 and column length 64 .. 1024, several
# members per class, rectangular grids both ways
SPECS = [(64, 64, -0.3, -0.3), (128, 128, -0.25, -0.2), (64, 64, -0.6, -0.45), (256, 128, -0.1, -0.05),
         (128, 256, -0.5, -0.4), (512, 512, -0.3, -0.25), (128, 128, -0.4, -0.35), (1024, 64, -0.2, -0.15),
         (64, 1024, -0.3, -0.2)]


def _ic(nx, ny, mean, seed):
    return mean + 0.05 * np.random.default_rng(seed).uniform(-1, 1, (ny, nx))


def _sim(nx, ny, eps, mean, precision, seed, kernels):
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=eps, g=0.0, dt=0.5)
    geom = stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4)
    sim = stdpfc.BuildB200_Simulation(prm, geom, precision=precision, kernels=kernels)
    sim.State.n[...] = _ic(nx, ny, mean, seed)
    return sim


def _state(sim):
    return sim.plan.get_state().cpu().numpy()


def _reduce(sims):
    import torch
    out = torch.empty((len(sims), 3), dtype=torch.float64, device=sims[0].plan.device)
    for i, s in enumerate(sims):
        s.plan.reduce(out[i])
    return out.cpu().numpy()


def _members(precision, specs=SPECS):
    return [_sim(nx, ny, eps, mean, precision, i, queue_kernels(nx, ny, precision))
            for i, (nx, ny, eps, mean) in enumerate(specs)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_queue_matches_plans_stepped_alone(precision):
    """1 + 16 + 15 + 33 steps (direct launches and replayed 16-step blocks at both
    parities) of a work-queue batch of nine plans in seven classes equal the same plans
    stepped alone, bit for bit: states, F, mu and mean."""
    ref = _members(precision)
    sims = _members(precision)
    q = QueueBatch(sims)
    info = q.info()
    assert info["classes"] == 7 and info["ctas"] >= 148 and info["ctas_per_sm"] >= 2, info
    done = 0
    for k in (1, 16, 15, 33):
        q.step(k)
        done += k
        for r in ref:
            r.TimeSteps(k)
        for a, b in zip(ref, sims):
            assert np.array_equal(_state(a), _state(b)), (a.plan.shape, done)
    assert q.status() == 0
    assert np.array_equal(q.reduce(), _reduce(ref))
    assert q.launches() == 6   # 1, 16 (a block), 15, 33 (two blocks and one step)
    q.close()


def test_queue_equals_batch_fp32_sweep_boxes():
    """On the sweep's box sizes the queue variants are the batch-tuned ones (FP32), so a
    queue batch and a `Batch` of the same members agree bit for bit after 48 steps."""
    specs = [(128, 128, -0.6, -0.4), (256, 256, -0.4, -0.3), (512, 512, -0.2, -0.15), (128, 128, -0.3, -0.2),
             (256, 256, -0.5, -0.45)]
    a, b = _members("fp32", specs), _members("fp32", specs)
    qa, bb = QueueBatch(a), Batch(b)
    qa.step(48)
    bb.step(48)
    for x, y in zip(a, b):
        assert np.array_equal(_state(x), _state(y))
    assert np.array_equal(qa.reduce(), bb.reduce())
    qa.close()
    bb.close()


def test_queue_refuses_plans_it_cannot_step():
    """Plans outside the work-queue kernel's set are refused with the reason."""
    def refused(sim, what):
        with pytest.raises(_lib.PfcError, match=what):
            QueueBatch([sim])

    refused(_sim(128, 128, -0.3, -0.3, "fp32", 0, {"ee_row": 16, "ee_col": 8, "row_tile": 8}), "values per thread")
    refused(_sim(2048, 64, -0.3, -0.3, "fp32", 0, "default"), "64 .. 1024")
    refused(_sim(96, 80, -0.3, -0.3, "fp64", 0, "default"), "power-of-two")
    refused(_sim(128, 128, -0.3, -0.3, "fp32", 0, dict(queue_kernels(128, 128), packed=1)), "one-lane")
    prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.05)
    log = logpfc.BuildB200_Simulation(prm, logpfc.Build2DGeometry(64, 64, 50.0, 50.0), kernels=queue_kernels(64, 64))
    log.State.phi[...] = 0.55
    refused(log, "stdPFC")
    with pytest.raises(_lib.PfcError, match="precisions"):
        QueueBatch(_members("fp32", SPECS[:1]) + _members("fp64", SPECS[1:2]))


def test_queue_wait_runs_out_and_reports():
    """A wait that never completes (the first column item waits for one completion more
    than exist) gives up after its poll limit: the launch ends early with
    PFC_STATUS_TIMEOUT in the queue's status, and the device stays usable: the same queue
    steps correctly again once the hook is cleared and the states are set anew."""
    sims = _members("fp32", SPECS[:3])
    q = QueueBatch(sims)
    q._test_wait(1, 2000)
    q.step(2)
    assert q.status() & _lib.STATUS_TIMEOUT
    q._test_wait(0, 0)
    ref = _members("fp32", SPECS[:3])
    for i, (s, r) in enumerate(zip(sims, ref)):
        nx, ny, _, mean = SPECS[i]
        s.State.n[...] = _ic(nx, ny, mean, i)
        r.TimeSteps(20)
    q.step(20)
    for s, r in zip(sims, ref):
        assert np.array_equal(_state(s), _state(r))
    q.close()
