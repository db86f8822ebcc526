"""pfc_field_mean_noalloc: the field mean for callers that must not allocate.

Some callers cannot allocate device memory: another allocator (a caching pool
such as PyTorch's) may have reserved the GPU's memory, so an allocation could
fail part-way through a run, or the caller's loop cannot afford cudaFree, which
waits for all work on the device. This entry point keeps its partial sums in a
fixed array inside the library instead. Its result is checked against the mean
that pfc_reduce (the existing entry point) reports after pfc_set_state of the
same field, on consecutive calls of different sizes, so that a call that read
the previous call's leftovers in the shared array would show. Tolerance: 1e-13
absolute on means of magnitude 0.2-0.6 (both are compensated FP64 sums; they
differ only in summation order and, for the FP64 plan, by the FFT round trip).

This file is named to be collected last.
"""
import ctypes
import math

import numpy as np
import pytest

from pfc_models_b200 import _lib, stdpfc

pytestmark = pytest.mark.gpu

MAX_SITES = 1 << 26   # 8192 x 8192, the size the fixed scratch array holds


def _noalloc_mean(lib, torch, field):
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=field.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.pfc_field_mean_noalloc(ctypes.c_void_p(field.data_ptr()), field.numel(),
                                    ctypes.c_void_p(out.data_ptr()), stream)
    _lib.check(rc)
    return float(out.cpu()[0])


def _reduce_mean(nx, ny, precision, f0):
    prm = stdpfc.BuildStdPFCModelParameters(epsilon=-0.25, g=0.0, dt=0.5)
    sim = stdpfc.BuildB200_Simulation(prm, stdpfc.Build2DGeometry(nx, ny, nx * np.pi / 4, ny * np.pi / 4),
                                      precision=precision)
    sim.State.n[...] = f0
    return float(sim.Reduce()[2])


def test_noalloc_mean_matches_reduce_on_consecutive_calls():
    import torch
    lib = _lib.load()
    cases = [(512, 384, "fp32", -0.25, 0), (300, 200, "fp64", -0.55, 1), (512, 384, "fp32", -0.25, 0),
             (2048, 2048, "fp32", -0.3, 2)]
    for nx, ny, precision, mean, seed in cases:
        f0 = mean + 0.05 * np.random.default_rng(seed).uniform(-1, 1, (ny, nx))
        expected = _reduce_mean(nx, ny, precision, f0)
        field = torch.as_tensor(f0, device="cuda")
        got = _noalloc_mean(lib, torch, field)
        again = _noalloc_mean(lib, torch, field)
        assert got == again
        assert got == pytest.approx(expected, abs=1e-13)
        assert got == pytest.approx(math.fsum(f0.ravel()) / f0.size, abs=1e-15)


def test_noalloc_mean_rejects_sizes_beyond_its_scratch():
    import torch
    lib = _lib.load()
    field = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.pfc_field_mean_noalloc(ctypes.c_void_p(field.data_ptr()), MAX_SITES + 1,
                                    ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == _lib.PFC_E_ARG
    assert "exceed the maximum" in _lib.last_error()
    assert lib.pfc_field_mean_noalloc(ctypes.c_void_p(field.data_ptr()), 0, ctypes.c_void_p(out.data_ptr()),
                                      stream) == _lib.PFC_E_ARG
