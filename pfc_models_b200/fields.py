"""Initial conditions on the host (FP64 NumPy), with the reference generators'
names and arguments (fields/initial_conditions_2d.py), plus the seeded
polycrystal and noisy-liquid generators that the benchmark configurations use.

The one-mode triangular profile is written as the real cosine sum
n = n0 + 2 A0 (cos(q1.r) + cos(q2.r) + cos(q3.r)), which is the real part of the
reference's six complex exponentials (initial_conditions_2d.py:80-104).
"""
from __future__ import annotations

import numpy as np

npFloatType = np.float64
_SQ3 = 3**0.5


def _one_mode(X, Y, mean, A0, q0=1.0, theta=0.0):
    """Triangular one-mode profile with wave vectors q0 (-sqrt3/2, -1/2),
    q0 (sqrt3/2, -1/2), q0 (0, 1), rotated by theta."""
    base = np.array([[-_SQ3 / 2, -0.5], [_SQ3 / 2, -0.5], [0.0, 1.0]]) * q0
    c, s = np.cos(theta), np.sin(theta)
    rot = np.array([[c, -s], [s, c]])
    out = np.full(np.shape(X), mean, dtype=npFloatType)
    for q in base:
        qx, qy = rot @ q
        out += 2 * A0 * np.cos(qx * X + qy * Y)
    return out


def GenerateHotInitialConditions(geometry, meanDensity, stdDeviation, kMax, seed=None):
    """Gaussian noise, low-passed, rescaled to stdDeviation, shifted positive and
    rescaled to meanDensity (initial_conditions_2d.py:19-40). The cut keeps
    modes with |k| <= kMax**2, as the reference does."""
    rng = np.random.default_rng(seed)
    noise = rng.normal(loc=0, scale=1.0, size=geometry.X.shape)
    spec = np.fft.rfft2(noise)
    spec[np.sqrt(geometry.KX**2 + geometry.KY**2) > kMax**2] = 0
    field = np.fft.irfft2(spec, s=geometry.X.shape)
    field *= stdDeviation / field.std()
    if field.min() <= 0:
        field -= field.min()
    field *= meanDensity / field.mean()
    return field.astype(npFloatType)


def GenerateLogNormalHotInitialConditions(geometry, meanDensity, stdDeviation, kMax, seed=None):
    """Log-normal field with a Gaussian spectral filter exp(-(|k|/kMax)^2), mean
    meanDensity and relative spread stdDeviation (initial_conditions_2d.py:43-77)."""
    rng = np.random.default_rng(seed)
    tau2 = np.log(1 + stdDeviation**2)
    tau = np.sqrt(tau2)
    mu = np.log(meanDensity) - tau2 / 2
    z = rng.normal(0.0, 1.0, size=geometry.X.shape).astype(npFloatType)
    k = np.sqrt(geometry.KX**2 + geometry.KY**2)
    y_raw = np.fft.irfft2(np.fft.rfft2(z) * np.exp(-((k / kMax) ** 2))).real
    y = (y_raw - y_raw.mean()) * (tau / np.sqrt(y_raw.var()))
    x = np.exp(mu + y)
    x *= meanDensity / x.mean()
    return x.astype(npFloatType)


def GeneratePerfectCrystalInitialConditions(geometry, meanDensity, A0, q0=1.0):
    """One-mode triangular crystal (initial_conditions_2d.py:80-104)."""
    return _one_mode(geometry.X, geometry.Y, meanDensity, A0, q0)


def _cut_disk(field, X, Y, xc, yc, r2, value):
    field[((X - xc) ** 2 + (Y - yc) ** 2) < r2] = value


def GeneratePerfectCrystalInitialWithCentralVacancy(geometry, meanDensity_S, meanDensity_V, A0, q0=1.0):
    """Crystal with one vacancy: the disk of radius a/2 at the lattice site
    nearest the box centre set to meanDensity_V (initial_conditions_2d.py:107-144)."""
    a, h = 4 * np.pi / _SQ3 / q0, 4 * np.pi / q0
    field = _one_mode(geometry.X, geometry.Y, meanDensity_S, A0, q0)
    xc = (geometry.Lx / a // 2) * a
    yc = (geometry.Ly / h // 2) * h
    _cut_disk(field, geometry.X, geometry.Y, xc, yc, a**2 / 4, meanDensity_V)
    return field


def GeneratePerfectCrystalInitialWithVancies(geometry, meanDensity_S, meanDensity_V, vacancyCoordsSet, A0):
    """Crystal (q0 = 1) with vacancies at cell coordinates (mx, my) -> (mx a, my h)
    (initial_conditions_2d.py:147-183; the reference's spelling is kept)."""
    a, h = 4 * np.pi / _SQ3, 4 * np.pi
    field = _one_mode(geometry.X, geometry.Y, meanDensity_S, A0, 1.0)
    for mx, my in vacancyCoordsSet:
        _cut_disk(field, geometry.X, geometry.Y, mx * a, my * h, a**2 / 4, meanDensity_V)
    return field


def GeneratePerfectCrystalInitialWithSolidLiquid(geometry, meanDensity_S, meanDensity_L, liquidRegionCoords, A0,
                                                 q0=1.0):
    """Crystal with rectangular groups of sites melted to meanDensity_L: for each
    (mxL, myL, mxU, myU) both sites (m a, m' h) and (m a + a/2, m' h + h/2) of every
    cell in the range (initial_conditions_2d.py:186-227)."""
    a, h = 4 * np.pi / _SQ3 / q0, 4 * np.pi / q0
    field = _one_mode(geometry.X, geometry.Y, meanDensity_S, A0, q0)
    for mxL, myL, mxU, myU in liquidRegionCoords:
        for mx in range(mxL, mxU):
            for my in range(myL, myU):
                _cut_disk(field, geometry.X, geometry.Y, mx * a, my * h, a**2 / 4, meanDensity_L)
                _cut_disk(field, geometry.X, geometry.Y, mx * a + a / 2, my * h + h / 2, a**2 / 4, meanDensity_L)
    return field


def GenerateDislocationRingInitialConditions(geometry, meanDensity, A0, radius, theta):
    """Crystal with a disk of radius `radius` at the box centre rotated by theta,
    which bounds a dislocation ring (initial_conditions_2d.py:230-277)."""
    field = _one_mode(geometry.X, geometry.Y, meanDensity, A0, 1.0)
    grain = _one_mode(geometry.X, geometry.Y, meanDensity, A0, 1.0, theta)
    inside = ((geometry.X - geometry.Lx / 2) ** 2 + (geometry.Y - geometry.Ly / 2) ** 2) < radius**2
    field[inside] = grain[inside]
    return field


# ------------------------------------------------------------------ new generators
def GenerateNoisyLiquid(geometry, meanDensity, amplitude, seed=0):
    """meanDensity + amplitude * U[-1, 1), seeded with numpy default_rng(seed)."""
    rng = np.random.default_rng(seed)
    return (meanDensity + amplitude * rng.uniform(-1.0, 1.0, size=geometry.X.shape)).astype(npFloatType)


def GeneratePolycrystalInitialConditions(geometry, meanDensity, noise, nSeeds, radius, A=0.5,
                                         q=3**0.5 / 2, noise_seed=0, seed=1):
    """Noisy liquid with `nSeeds` circular crystal seeds.

    The liquid is meanDensity + noise * U[-1, 1) (default_rng(noise_seed)).
    Seed centres are uniform in the box and orientations uniform in [0, pi/3)
    (default_rng(seed)); each seed of radius `radius` is set to
    meanDensity + A (cos(q x') cos(q y'/sqrt3) - cos(2 q y'/sqrt3)/2) with (x', y')
    the position relative to the centre rotated by the orientation, using
    periodic (minimum-image) distances. Later seeds overwrite earlier ones.
    """
    g = geometry
    field = GenerateNoisyLiquid(g, meanDensity, noise, noise_seed)
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, size=(nSeeds, 2)) * np.array([g.Lx, g.Ly])
    angles = rng.uniform(0.0, np.pi / 3, size=nSeeds)
    r2 = radius**2
    # each seed touches a (2R) x (2R) window; work there instead of on the full grid
    wx = int(np.ceil(radius / g.dx)) + 1
    wy = int(np.ceil(radius / g.dy)) + 1
    for (cx, cy), th in zip(centres, angles):
        ix0 = int(np.floor(cx / g.dx))
        iy0 = int(np.floor(cy / g.dy))
        ix = (np.arange(ix0 - wx, ix0 + wx + 1)) % g.Nx
        iy = (np.arange(iy0 - wy, iy0 + wy + 1)) % g.Ny
        xs = g.x[ix] - cx
        ys = g.y[iy] - cy
        xs -= g.Lx * np.round(xs / g.Lx)
        ys -= g.Ly * np.round(ys / g.Ly)
        DX, DY = np.meshgrid(xs, ys)
        inside = DX**2 + DY**2 < r2
        c, s = np.cos(th), np.sin(th)
        xr = c * DX + s * DY
        yr = -s * DX + c * DY
        prof = meanDensity + A * (np.cos(q * xr) * np.cos(q * yr / _SQ3) - np.cos(2 * q * yr / _SQ3) / 2)
        sub = field[np.ix_(iy, ix)]
        sub[inside] = prof[inside]
        field[np.ix_(iy, ix)] = sub
    return field
