"""ORACLE — test infrastructure, not product code.

A CPU restatement (NumPy / SciPy FFT) of the reference's pseudo-spectral ETD1
stepper for standard and log PFC in 2D, used to check the CUDA path. Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
(and its ``--impl reference`` arm) may import it, and only as the checker or
as the timed CPU baseline; the product never routes through it.

Parity is pinned: ``tests/test_oracle_golden.py`` checks this module against
fixtures generated by running the unmodified reference
(``tests/golden/make_golden.py``), including the reference's own recorded
free energies (stdpfc_cpu/test_regression.py:64, logpfc_cpu/test_regression.py:28-32).

Each function cites the reference lines it restates (paths relative to the
reference project root, ``src/pfc_models/...``).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

try:  # threaded pocketfft (same algorithm as numpy.fft); optional
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None


# ---------------------------------------------------------------- substrate
@dataclass
class Geometry:
    """discretization/spectral/geometry_2d.py:70-88 (Build2DGeometry)."""
    Nx: int
    Ny: int
    Lx: float
    Ly: float
    dx: float
    dy: float
    X: np.ndarray
    Y: np.ndarray
    KX: np.ndarray
    KY: np.ndarray
    K2: np.ndarray


def build_geometry(Nx, Ny, Lx, Ly) -> Geometry:
    """geometry_2d.py:70-88: x, y by linspace(endpoint=False); kx = 2 pi rfftfreq(Nx, dx),
    ky = 2 pi fftfreq(Ny, dy); meshgrids of shape (Ny, Nx) and (Ny, Nx//2+1)."""
    dx, dy = Lx / Nx, Ly / Ny
    x = np.linspace(0, Lx, Nx, endpoint=False)
    y = np.linspace(0, Ly, Ny, endpoint=False)
    X, Y = np.meshgrid(x, y)
    kx = 2 * np.pi * np.fft.rfftfreq(Nx, d=dx)
    ky = 2 * np.pi * np.fft.fftfreq(Ny, d=dy)
    KX, KY = np.meshgrid(kx, ky)
    return Geometry(Nx, Ny, Lx, Ly, dx, dy, X, Y, KX, KY, KX**2 + KY**2)


def laplacian(geom: Geometry) -> np.ndarray:
    """kernels.py:45 (d2_dlap = -(KX^2 + KY^2)); the models take its real part
    (stdpfc/simulation.py:112)."""
    return -(geom.KX**2 + geom.KY**2)


def gaussian(geom: Geometry, w: float) -> np.ndarray:
    """kernels.py:49-52 (kernel_local): exp(-|k|^2 w^2 / 2)."""
    return np.exp(-((geom.KX) ** 2 + (geom.KY) ** 2) * w**2 / 2)


def linear_mu(beta, q0, epsilon, lap):
    """stdpfc/simulation.py:83-90 and logpfc/simulation.py:78-85: beta (q0^2 + lap)^2 + epsilon."""
    return beta * (q0**2 + lap) ** 2 + epsilon


def linear_n(Gamma, beta, q0, epsilon, lap):
    """stdpfc/simulation.py:92-96: Gamma lap (beta (q0^2 + lap)^2 + epsilon)."""
    return Gamma * lap * linear_mu(beta, q0, epsilon, lap)


def etd1(kLinear, dt, small_z_tol=2e-5):
    """kernels.py:55-71 (kernel_etd): A = exp(L dt); B = (A - 1)/L where |L dt| > tol,
    else dt (1 + z/2 + z^2/6)."""
    z = kLinear * dt
    A = np.exp(z)
    with np.errstate(divide="ignore", invalid="ignore"):
        B = np.where(np.abs(z) > small_z_tol, (A - 1) / kLinear, dt * (1 + z / 2 + z**2 / 6))
    return A, B


# ---------------------------------------------------------------- model
@dataclass
class Params:
    """stdpfc/simulation.py:60-80 (BuildStdPFCModelParameters) and
    logpfc/simulation.py:51-75 (BuildLogPFCModelParameters)."""
    Gamma: float = 1.0
    beta: float = 1.0
    q0: float = 1.0
    epsilon: float = 1.0
    g: float = 1.0
    dt: float = 0.01
    smallZTol: float = 2e-5


def nonlin_mu(model: str, n: np.ndarray, g: float) -> np.ndarray:
    """std: g n^2 + n^3 (stdpfc_cpu/simulation.py:323-333, stdpfc/simulation.py:297).
    log: ln(phi) + g phi^2 + phi^3, unclamped (logpfc_cpu/simulation.py:321-331,
    logpfc/simulation.py:296)."""
    if model == "std":
        return g * (n**2) + (n**3)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.log(n) + g * (n**2) + (n**3)


class OracleSim:
    """The reference CPU stepper (stdpfc_cpu/simulation.py:238-248, logpfc_cpu/simulation.py:233-243),
    restated without the unused diagnostics batch.

    ``fft`` selects numpy.fft (default; the algorithm the fixtures were generated with)
    or scipy.fft with ``workers`` threads (same pocketfft algorithm, used for timing).
    """

    def __init__(self, model, params: Params, geom: Geometry, fft="numpy", workers=1):
        assert model in ("std", "log")
        self.model, self.p, self.geom = model, params, geom
        self.t = 0.0
        lap = laplacian(geom)
        self.lap = lap
        self.lin_mu = linear_mu(params.beta, params.q0, params.epsilon, lap)
        kl = linear_n(params.Gamma, params.beta, params.q0, params.epsilon, lap)
        self.A, self.B = etd1(kl, params.dt, params.smallZTol)
        # the reference's update multiplies B by (Gamma * lap) per step
        # (stdpfc_cpu/simulation.py:365-372); both products are kept in the same order
        self.gauss = gaussian(geom, 2 * np.pi)
        self.n = np.zeros((geom.Ny, geom.Nx))
        self.n_hat = np.zeros((geom.Ny, geom.Nx // 2 + 1), dtype=complex)
        self.nonlin_mu_hat = np.zeros_like(self.n_hat)
        if fft == "scipy" and _sfft is not None:
            w = workers if workers and workers > 0 else os.cpu_count()
            self._rfft2 = lambda a: _sfft.rfft2(a, workers=w)
            self._irfft2 = lambda a, s: _sfft.irfft2(a, s=s, workers=w)
        else:
            self._rfft2 = lambda a: np.fft.rfft2(a)
            self._irfft2 = lambda a, s: np.fft.irfft2(a, s=s)

    def set_field(self, n):
        self.n = np.array(n, dtype=np.float64, copy=True)

    def step(self):
        """One ETD1 step: batch1 (nonlinearity + rfft2), batch3 (update + irfft2), n <- n_next."""
        p = self.p
        N = nonlin_mu(self.model, self.n, p.g)                     # _Batch1_CalcNonlinMu
        self.n_hat = self._rfft2(self.n)
        self.nonlin_mu_hat = self._rfft2(N)
        n_next_hat = self.A * self.n_hat + self.B * (p.Gamma * self.lap * self.nonlin_mu_hat)
        self.n = self._irfft2(n_next_hat, self.n.shape)            # _Batch3_CalcNNext
        self.t += p.dt

    def mu(self):
        """mu = irfft2(L_mu n_hat + N_hat) of the current field (stdpfc/simulation.py:299-308, batch2)."""
        N = nonlin_mu(self.model, self.n, self.p.g)
        mu_hat = self.lin_mu * self._rfft2(self.n) + self._rfft2(N)
        return self._irfft2(mu_hat, self.n.shape)

    def free_energy(self):
        """stdpfc_cpu/simulation.py:263-285 (std) and logpfc_cpu/simulation.py:259-283 (log):
        mean of n irfft2(beta/2 (q0^2 + lap)^2 n_hat) + eps/2 n^2 + g/3 n^3 + n^4/4 (+ n ln n)."""
        p, n = self.p, self.n
        n_hat = self._rfft2(n)
        lin_f = self._irfft2((p.beta / 2.0) * (p.q0**2 + self.lap) ** 2 * n_hat, n.shape)
        nonlin_f = (p.epsilon / 2.0) * n**2 + (p.g / 3.0) * n**3 + (1 / 4.0) * n**4
        if self.model == "log":
            with np.errstate(divide="ignore", invalid="ignore"):
                nonlin_f = n * np.log(n) + nonlin_f
        return float((n * lin_f + nonlin_f).mean())

    def mu_per_site(self):
        """Mean chemical potential: mu_hat(0)/(Nx Ny) = L_mu(0) mean(n) + mean(N(n));
        the quantity the adapters' liquid_chemical_potential gives in closed form for a
        uniform field (stdpfc_cpu/phase_diagram.py:312-320, logpfc_cpu/phase_diagram.py:336-347)."""
        p = self.p
        return float(linear_mu(p.beta, p.q0, p.epsilon, 0.0) * self.n.mean()
                     + nonlin_mu(self.model, self.n, p.g).mean())

    def local_field(self, w=2 * np.pi):
        """Get_local_n (stdpfc/simulation.py:237-247) on the current field: irfft2(G rfft2(n))."""
        return self._irfft2(gaussian(self.geom, w) * self._rfft2(self.n), self.n.shape)


def run(model, params: Params, geom: Geometry, field0, steps, record_every=None):
    """Step ``field0`` for ``steps`` steps; return (final field, [(step, F, mean), ...])."""
    sim = OracleSim(model, params, geom)
    sim.set_field(field0)
    rec = []
    for s in range(steps + 1):
        if record_every and s % record_every == 0:
            rec.append((s, sim.free_energy(), float(sim.n.mean())))
        if s < steps:
            sim.step()
    return sim.n, rec


# ---------------------------------------------------------------- log PFC with an external potential
class OracleExtv:
    """The reference's logpfc_extv stepper (models/logpfc_extv/simulation.py), restated.

    Per TimeStep (:301-330): ValidatePhiRange (:375-405) re-optimises the shift M when the
    field's range leaves the last optimised range by more than 10 % (relative, floor and
    ceiling); OptimizeM (:332-373) sets M = (N(max) - N(min)) / (max - min) with
    N(x) = g x^2 + x^3 + ln x (min replaced by minPhi when the field's minimum is <= 0) and
    rebuilds the linear mu kernel beta (q0^2 + lap)^2 + eps + M and the ETD1 coefficients
    (kernel_etd, smallZTol 1e-8 by default, :69-117); the nonlinearity is the clamped log
    where(phi > minPhi, ln phi, ln minPhi) + g phi^2 + phi^3 - M phi (:524-539); the update
    phi_next_hat = A phi_hat + B (Gamma lap N_hat + lap V_hat), with the k = 0 mode kept
    (:557-577). F is the logPFC free energy (:427-451). V is a real field (the reference's
    _ExternalPotential.V, zero unless set)."""

    def __init__(self, params: Params, geom: Geometry, min_phi=1e-6, V=None):
        self.p, self.geom = params, geom
        self.min_phi, self.min_log = min_phi, np.log(min_phi)
        self.lap = laplacian(geom)
        self.M = 0.0
        self.phi_min = self.phi_max = None
        self.floor_tol = self.ceiling_tol = 0.1
        self.optimizations = 0
        self.n = np.zeros((geom.Ny, geom.Nx))
        self.V_hat = np.fft.rfft2(np.zeros((geom.Ny, geom.Nx)) if V is None else np.asarray(V, dtype=np.float64))
        self._coefficients(0.0)

    def _coefficients(self, M):
        p = self.p
        kl = p.Gamma * self.lap * (p.beta * (p.q0**2 + self.lap) ** 2 + p.epsilon + M)
        self.A, self.B = etd1(kl, p.dt, p.smallZTol)

    def set_field(self, phi):
        self.n = np.array(phi, dtype=np.float64, copy=True)

    def optimize_m(self):
        g = self.p.g
        lo = float(np.min(self.n)) if self.n.min() > 0 else self.min_phi
        hi = float(np.max(self.n))
        nmu = lambda x: g * x**2 + x**3 + np.log(x)  # noqa: E731
        self.M = (nmu(hi) - nmu(lo)) / (hi - lo)
        self._coefficients(self.M)
        self.phi_min, self.phi_max = lo, hi
        self.optimizations += 1

    def validate_phi_range(self):
        lo, hi = float(self.n.min()), float(self.n.max())
        if self.phi_min is None or self.phi_max is None:
            self.optimize_m()
            return
        if (self.phi_min - lo) / self.phi_min > self.floor_tol or (hi - self.phi_max) / self.phi_max > self.ceiling_tol:
            self.optimize_m()

    def step(self):
        self.validate_phi_range()
        p, phi = self.p, self.n
        with np.errstate(divide="ignore", invalid="ignore"):
            N = np.where(phi > self.min_phi, np.log(phi), self.min_log) + p.g * phi**2 + phi**3 - self.M * phi
        phi_hat = np.fft.rfft2(phi)
        nxt = self.A * phi_hat + self.B * (p.Gamma * self.lap * np.fft.rfft2(N) + self.lap * self.V_hat)
        nxt.flat[0] = phi_hat.flat[0]
        self.n = np.fft.irfft2(nxt, s=phi.shape)

    def free_energy(self):
        p, phi = self.p, self.n
        lin_f = np.fft.irfft2((p.beta / 2.0) * (p.q0**2 + self.lap) ** 2 * np.fft.rfft2(phi), s=phi.shape)
        with np.errstate(divide="ignore", invalid="ignore"):
            nonlin_f = phi * np.log(phi) + (p.epsilon / 2.0) * phi**2 + (p.g / 3.0) * phi**3 + phi**4 / 4.0
        return float((phi * lin_f + nonlin_f).mean())


# ---------------------------------------------------------------- vacancy tracking
def _np_index(i: int, n: int) -> int:
    """An integer index on an axis of length n as NumPy reads it: negative counts from
    the end, out of range raises IndexError."""
    j = i + n if i < 0 else i
    if j < 0 or j >= n:
        raise IndexError(f"index {i} is out of bounds for axis with size {n}")
    return j


def _np_slice(start: int, stop: int, n: int) -> range:
    """range(*slice(start, stop).indices(n)) for a unit step, as NumPy slices an axis."""
    return range(*slice(start, stop).indices(n))


def locate_vacancy(local: np.ndarray, x0: float, y0: float, dx: float, dy: float):
    """analysis/vacancy_tracker.py:22-60 (_VacancyTracker.LocateVacancy), restated with
    the index rules spelled out: the nearest pixel of (x0, y0) by round-half-to-even,
    the first minimum (row-major) of the 3 x 3 neighbourhood as a NumPy slice cuts it
    (negative starts wrap, stops clip; an empty slice raises ValueError), the parabolic
    sub-pixel step along each axis from the 5-point cross (zero denominator: no step;
    index -1 wraps, one past the end raises IndexError). Returns (x, y)."""
    if not (np.isfinite(x0) and np.isfinite(y0)):
        raise ValueError("cannot convert a non-finite position to a pixel")
    ny_, nx_ = local.shape
    px = int(np.round(x0 / dx))
    py = int(np.round(y0 / dy))
    rows = _np_slice(py - 1, py + 2, ny_)
    cols = _np_slice(px - 1, px + 2, nx_)
    if len(rows) == 0 or len(cols) == 0:
        raise ValueError("attempt to get argmin of an empty sequence")
    best, bi, bj = None, 0, 0
    for i, r in enumerate(rows):
        for j, c in enumerate(cols):
            v = local[r, c]
            if best is None or (np.isnan(v) and not np.isnan(best)) or (not np.isnan(best) and v < best):
                best, bi, bj = v, i, j
    py += bi - 1
    px += bj - 1
    f_mid = local[_np_index(py, ny_), _np_index(px, nx_)]
    f_left = local[_np_index(py, ny_), _np_index(px - 1, nx_)]
    f_right = local[_np_index(py, ny_), _np_index(px + 1, nx_)]
    f_up = local[_np_index(py - 1, ny_), _np_index(px, nx_)]
    f_down = local[_np_index(py + 1, ny_), _np_index(px, nx_)]
    denom_x = 2.0 * (f_left - 2.0 * f_mid + f_right)
    delta_x = (f_left - f_right) / denom_x if denom_x != 0 else 0.0
    denom_y = 2.0 * (f_up - 2.0 * f_mid + f_down)
    delta_y = (f_up - f_down) / denom_y if denom_y != 0 else 0.0
    return (float(px + delta_x) * dx, float(py + delta_y) * dy)


# ---------------------------------------------------------------- 3-mode diagnostics
def diagnose_modes(n: np.ndarray, mode_sets, amplitude_sign: float, cells: int):
    """models/stdpfc_cpu/phase_diagram.py:178-215 (`_build3Mode`, `_calcFitness`,
    `_maxima_per_cell`; logpfc_cpu/phase_diagram.py has the same code): amplitudes A, B, C
    = sign * NaN-skipping mean of |rfft2(n)| over each set of (row, col) half-spectrum
    indices, per site; fitness = 1 - |mean((n - n3)^2)| with n3 the inverse rfft of the
    spectrum holding n_hat(0, 0) at DC and the set amplitudes times the site count at the
    set indices (later sets overwrite earlier ones); maxima per cell = the strict
    8-neighbour periodic maxima over `cells` cells. Returns
    (fitness, |A|, |B|, |C|, maxima per cell); raises IndexError for an index outside the
    half spectrum, as the reference does."""
    ny, nx = n.shape
    size = n.size
    n_hat = np.fft.rfft2(n)
    amps = []
    for rows, cols in mode_sets:
        amps.append(amplitude_sign * np.nanmean(np.abs(n_hat[rows, cols])) / size)
    rebuilt = np.zeros_like(n_hat)
    rebuilt[0, 0] = n_hat.flat[0] / size * size
    for (rows, cols), a in zip(mode_sets, amps):
        rebuilt[rows, cols] = a * size
    n3 = np.fft.irfftn(rebuilt, s=(ny, nx), axes=(0, 1)).real
    fitness = 1 - float(np.abs(np.power(n - n3, 2).mean()))
    is_max = np.ones(n.shape, dtype=bool)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dy or dx:
                is_max &= n > np.roll(n, (dy, dx), axis=(0, 1))
    return fitness, abs(amps[0]), abs(amps[1]), abs(amps[2]), int(is_max.sum()) / cells


# ---------------------------------------------------------------- frozen field (frozen_q)
def frozen_moments(phi: np.ndarray, temp: float, g: float, v0: float, cell: dict):
    """models/logpfc_cpu/phase_diagram.py:465-505 (`_k2_ref`, `FrozenField.__init__`):
    A_n = sum_k |fft2(phi)_k / N|^2 |k_ref|^(2n), n = 0, 1, 2, on the full FFT grid of the
    q00 = 1 box (Lx = Mx 4 pi / sqrt 3, Ly = My 4 pi), and the local term
    mean(phi ln phi + temp/2 phi^2 + g/3 phi^3 + v0/4 phi^4). Returns (A, local)."""
    phi = np.asarray(phi, dtype=float)
    ny, nx = phi.shape
    N = phi.size
    P = np.abs(np.fft.fft2(phi)) ** 2 / N ** 2
    Lx = cell['Mx'] * 4 * np.pi / np.sqrt(3.0)
    Ly = cell['My'] * 4 * np.pi
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=Lx / nx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=Ly / ny)
    KX, KY = np.meshgrid(kx, ky)
    K = KX ** 2 + KY ** 2
    A = np.array([P.sum(), (P * K).sum(), (P * K * K).sum()])
    local = float(np.mean(phi * np.log(phi) + temp / 2 * phi ** 2 + g / 3 * phi ** 3 + v0 / 4 * phi ** 4))
    return A, local


def defect_screen(phi: np.ndarray, cell: dict):
    """models/logpfc_cpu/phase_diagram.py:512-528 (`defect_diagnostics`): peak spread =
    (max - min) / mean of the heights above the mean of the sites >= their 8 periodic
    neighbours and above the mean; sub-q ratio = the largest |fft2(phi - mean)|^2 at
    0 < |k_ref| < 0.95 over the largest |fft2(phi - mean)|^2; the peak count.
    Returns (peak_spread, subq_ratio, n_peaks)."""
    phi = np.asarray(phi, dtype=float)
    m = phi.mean()
    nb = [np.roll(np.roll(phi, a, 0), b, 1) for a in (-1, 0, 1) for b in (-1, 0, 1) if (a, b) != (0, 0)]
    mask = np.all([phi >= x for x in nb], axis=0) & (phi > m)
    h = phi[mask] - m
    spread = float((h.max() - h.min()) / h.mean()) if h.size else float('nan')
    P = np.abs(np.fft.fft2(phi - m)) ** 2
    ny, nx = phi.shape
    Lx = cell['Mx'] * 4 * np.pi / np.sqrt(3.0)
    Ly = cell['My'] * 4 * np.pi
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=Lx / nx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=Ly / ny)
    KX, KY = np.meshgrid(kx, ky)
    kr = np.sqrt(KX ** 2 + KY ** 2)
    sub = (kr > 1e-9) & (kr < 0.95)
    ratio = float(P[sub].max() / P.max()) if P.max() > 0 else float('nan')
    return spread, ratio, int(mask.sum())
