"""Host-side substrate and initial conditions against the reference's outputs
(tests/golden/substrate.npz, produced by tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

from pfc_models_b200 import fields, spectral
from tests.conftest import GOLDEN


def _cfg():
    return json.load(open(os.path.join(GOLDEN, "manifest.json")))["cases"]["substrate"]["config"]


def test_geometry_and_kernels(golden):
    d, c = golden("substrate"), _cfg()
    g = spectral.Build2DGeometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    for k in ("X", "Y", "KX", "KY", "K2"):
        np.testing.assert_array_equal(getattr(g, k), d[k])
    dk = spectral.BuildDerivativeKernels(g)
    np.testing.assert_array_equal(dk.d2_dlap, d["d2_dlap"])
    ln = spectral.linear_kernel_n(c["Gamma"], c["beta"], c["q0"], c["epsilon"], dk.d2_dlap)
    A, B = spectral.kernel_etd(ln, c["dt"])
    np.testing.assert_array_equal(A, d["A"])
    np.testing.assert_array_equal(B, d["B"])
    np.testing.assert_array_equal(spectral.kernel_local(g, 2 * np.pi), d["gauss"])


def test_geometry_contract():
    """tests/test_smoke_models.py:298-319: the contract names and the ETD k=0 coefficient."""
    g = spectral.Build2DGeometry(Nx=64, Ny=64, Lx=32.0, Ly=32.0)
    for name in ("Nx", "Ny", "Lx", "Ly", "dx", "dy", "x", "y", "X", "Y", "kx", "ky", "KX", "KY", "K2"):
        assert hasattr(g, name)
    assert g.px_to_x(3) == 3 * g.dx and g.x_to_ix(g.dx * 5.5) == 5
    dk = spectral.BuildDerivativeKernels(g)
    A, B = spectral.kernel_etd(dk.d2_dlap, 0.1)
    assert np.isfinite(A).all() and np.isfinite(B).all()
    assert B.flat[0] == 0.1


@pytest.mark.parametrize("name", ["crystal", "vacancy", "vacancies", "solid_liquid", "ring", "hot", "lognormal"])
def test_initial_conditions(golden, name):
    d, c = golden("substrate"), _cfg()
    g = spectral.Build2DGeometry(c["Nx"], c["Ny"], c["Lx"], c["Ly"])
    got = {
        "crystal": lambda: fields.GeneratePerfectCrystalInitialConditions(g, 0.3, A0=0.1, q0=1.0),
        "vacancy": lambda: fields.GeneratePerfectCrystalInitialWithCentralVacancy(g, 0.3, 0.1, A0=0.1),
        "vacancies": lambda: fields.GeneratePerfectCrystalInitialWithVancies(g, 0.3, 0.1, [(0, 0), (1, 0)], A0=0.1),
        "solid_liquid": lambda: fields.GeneratePerfectCrystalInitialWithSolidLiquid(g, 0.3, 0.2, [(0, 0, 1, 1)], A0=0.1),
        "ring": lambda: fields.GenerateDislocationRingInitialConditions(g, 0.3, A0=0.1, radius=5.0, theta=0.3),
        "hot": lambda: fields.GenerateHotInitialConditions(g, 0.4, 0.1, kMax=0.9, seed=3),
        "lognormal": lambda: fields.GenerateLogNormalHotInitialConditions(g, 0.4, 0.1, kMax=0.9, seed=3),
    }[name]()
    np.testing.assert_allclose(got, d[f"ic_{name}"], rtol=1e-13, atol=1e-14)


def test_polycrystal_generator():
    g = spectral.Build2DGeometry(256, 256, 256 * np.pi / 4, 256 * np.pi / 4)
    a = fields.GeneratePolycrystalInitialConditions(g, -0.3, 0.01, nSeeds=4, radius=12 * g.dx)
    b = fields.GeneratePolycrystalInitialConditions(g, -0.3, 0.01, nSeeds=4, radius=12 * g.dx)
    np.testing.assert_array_equal(a, b)
    liquid = fields.GenerateNoisyLiquid(g, -0.3, 0.01, seed=0)
    changed = a != liquid
    # four disks of radius 12 dx cover at most 4 * pi * 144 sites
    assert 0 < changed.sum() <= 4 * np.pi * 144 + 50
    # the profile A (cos u cos v - cos(2v)/2) peaks at 0.75 A
    assert -0.3 + 0.7 * 0.5 < a[changed].max() <= -0.3 + 0.75 * 0.5 + 1e-12
