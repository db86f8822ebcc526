"""The large workloads at their full sizes, checked through size-independent
properties (no oracle runs at these sizes): mass is conserved to round-off, and
the FP32-mixed form keeps F per site within 1e-6 relative and mu within 1e-5 of
the FP64 plain form over the first steps."""
import numpy as np
import pytest

from pfc_models_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,steps,every", [("solidify8192", 200, 50), ("logpfc1024", 1000, 250),
                                             ("polycrystal2048", 2000, 500)])
def test_fp32_mixed_tracks_fp64_at_full_size(name, steps, every):
    r32 = workloads.run(name, "fp32", steps, every)
    r64 = workloads.run(name, "fp64", steps, every)
    assert r32["mass_drift"] <= 1e-12 and r64["mass_drift"] <= 1e-12
    F32, F64 = np.array(r32["F"]), np.array(r64["F"])
    assert np.all(np.isfinite(F32)) and np.all(np.isfinite(F64))
    assert np.max(np.abs(F32 - F64) / np.abs(F64)) < 1e-6
    assert np.max(np.abs(np.array(r32["mu"]) - np.array(r64["mu"]))) < 1e-5
    # the free energy of a relaxing state does not increase
    assert np.all(np.diff(F64) <= 1e-12 * np.abs(F64[1:]))
