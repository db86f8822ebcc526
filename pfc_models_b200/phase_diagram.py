"""Phase-diagram relaxation on B200 plans: the stdPFC and logPFC adapters and a batched
`Get_f_ABC`.

The reference computes a point of a phase diagram by relaxing a 3-mode crystal ansatz
at a fixed box scale q00 (src/pfc_models/phase_diagram/q0star.py:329-407, `Get_f_ABC`):
blocks of stepT time units are stepped, the free energy is checked after each block, a
block that raised f (or went NaN) is rolled back and redone at dt/divs in divs
sub-blocks (recursively, to maxDepth; :261-307), and the evaluation stops when f and the
leading amplitude have converged, the fit is poor, the amplitude vanished or totalT ran
out. A phase diagram is hundreds of such evaluations, each on a small cell grid.

* `StdAdapter` / `LogAdapter` implement the reference adapters' contract
  (models/stdpfc_cpu/phase_diagram.py:219-296, models/logpfc_cpu/phase_diagram.py:
  238-321: SLUG, STRUCTURES, validate_*, build, get/set_state, get/set_time, get_dt,
  step, free_energy, diagnose) on this package's plans, so the reference's own
  `MinimizeFreeEnergy` can drive them unchanged.
* `get_f_abc` is `Get_f_ABC` for one point on one plan (also the path for adaptive dt);
  `get_f_abc_batch` runs many points in lockstep through `simulation.Batch`: one launch
  per size class and pass for all members, device-side snapshots for the rollbacks, one
  device-to-host copy of every member's f per block, and the reference's decisions per
  member on the host. A member whose block must be rolled back leaves the lockstep for
  that block and runs the recursion on its own plans; a member that stops leaves the
  batch. Because a batch step is bit-identical to the same steps of the plan alone, the
  batch returns exactly what `get_f_abc` returns for each point.
* `find_q0star_batch` is `Find_q0Star` (q0star.py:409-478: passes of q00 scans refined
  by a cubic spline of f(q00)) for many (temp, meanDensity) at once, each pass one
  `get_f_abc_batch` over every target's q00 points; `find_q0star` is the one-target form.
* `scan_density_batch` is `scan_density` (q0star.py:566-635) over those searches, with
  the reference's result arrays and checkpoint files (fmin.npz, qscan.npz).
* `solve_frozen_q_batch` / `scan_density_frozen` are the frozen-q search
  (phase_diagram/frozen_q.py:92-243: relax at q, jump q to the frozen field's q_opt,
  tighten fTol) for many densities in lockstep, with the reference's edge pass.

The ansatz is built on the host with the reference's NumPy operations
(`_build3Mode`, stdpfc_cpu/phase_diagram.py:171-182 and logpfc_cpu/phase_diagram.py:
182-200, the log one rescaled to stay positive), so both start from the same bits; the
ansatz noise follows q0star.py:227-244 (relative noise from default_rng(seed), mean
restored).
"""
from __future__ import annotations

import os
import time
import warnings
from dataclasses import dataclass, replace

import numpy as np

from . import diagnostics as _diag
from . import logpfc as _logpfc
from . import stdpfc as _stdpfc
from .spectral import Build2DGeometry
from .simulation import Batch

# stop reasons (q0star.py:103-109)
STOP_CONVERGED = 'converged'
STOP_MAX_DEPTH = 'max_depth'
STOP_NAN = 'nan'
STOP_POOR_FIT = 'poor_fit'
STOP_MIN_AMPLITUDE = 'min_amplitude'
STOP_TOTALT = 'totalT'
FAILED_STOPS = (STOP_MAX_DEPTH, STOP_NAN)


class MaxDepthReached(RuntimeError):
    """The rollback recursion reached maxDepth (q0star.py:112-118); `nan` tells whether
    the last block went NaN."""

    def __init__(self, message, nan=False):
        super().__init__(message)
        self.nan = nan


@dataclass(frozen=True)
class RelaxSettings:
    """Relaxation settings with the reference's names and defaults (q0star.py:124-150)."""
    dt: float
    totalT: float
    stepT: float
    divs: int
    maxDepth: int
    requiredFitness: float | None
    minimumA: float
    fTol: float = 1e-12
    ATol: float = 1e-6
    seed: int = 0
    noise: float = 1e-10
    dtMax: float | None = None
    dtRate: float = 1e-8
    dtGrow: float = 2.0
    dtChecks: int = 10


@dataclass
class RelaxResult:
    """One evaluation: `Get_f_ABC`'s return (f, fitness, *amplitudes) and what the
    reference leaves in `last_stop`, `last_steps`, `last_dt_max` and `last_state`."""
    f: float
    fitness: float
    amplitudes: tuple
    stop: str
    steps: int
    dt_max: float
    state: np.ndarray | None = None

    def values(self):
        return (self.f, self.fitness, *self.amplitudes)


# ---------------------------------------------------------------- adapters
_PARAM_KEYS = ('beta', 'g', 'v0', 'Gamma', 'q0')
_ANSATZ_KEYS = ('mode', 'A1', 'A2', 'A3')


@dataclass(frozen=True)
class LogStructure:
    """A logPFC target lattice: the stdPFC mode sets with the log ansatz's amplitude
    bound `amplitudeMax` (logpfc_cpu/phase_diagram.py:57-99; honeycomb 1/6)."""
    name: str
    kvectors: tuple
    amplitudeSign: int
    amplitudeMax: float
    maxima_per_cell: int | None


LOG_STRUCTURES = {
    name: LogStructure(st.name, st.kvectors, st.amplitudeSign, 1.0 / 6 if name == 'honeycomb' else st.amplitudeScale,
                       st.maxima_per_cell)
    for name, st in _diag.STRUCTURES.items()
}


class _Adapter:
    """The adapter contract shared by both models; subclasses set the model.

    `precision` is the plans' form: "fp64" (the default) resolves f to round-off, as the
    relaxation's default tolerances assume (fTol 1e-12 relative per block); "fp32"
    (FP32-mixed) resolves the free energy to about 1e-7 relative, so its relaxations need an
    fTol above that or they run to totalT. Small FP64 cells step with the one-CTA kernel."""
    SLUG = None
    STRUCTURES = None
    FIELD = None

    def __init__(self, precision='fp64', device=None):
        self.precision = precision
        self.device = device

    # -- validation (stdpfc_cpu/phase_diagram.py:104-154)
    def validate_params(self, params):
        p = dict(params)
        unknown = sorted(set(p) - set(_PARAM_KEYS))
        if unknown:
            raise ValueError(f'{self.SLUG}: unknown model parameters {unknown}; allowed {list(_PARAM_KEYS)}')
        missing = [k for k in ('beta', 'g') if k not in p]
        if missing:
            raise ValueError(f'{self.SLUG}: missing model parameters {missing}')
        v0 = float(p.get('v0', 1.0))
        if v0 != 1.0:
            raise ValueError(f'{self.SLUG}: v0={v0} not supported; the quartic coefficient is 1 in the step')
        return {'beta': float(p['beta']), 'g': float(p['g']), 'v0': 1.0,
                'Gamma': float(p.get('Gamma', 1.0)), 'q0': float(p.get('q0', 1.0))}

    def validate_cell(self, cell):
        try:
            return _diag._cell(cell)
        except ValueError as e:
            raise ValueError(f'{self.SLUG}: {e}') from None

    def validate_ansatz(self, ansatz):
        a = dict(ansatz)
        if sorted(a) != sorted(_ANSATZ_KEYS):
            raise ValueError(f'{self.SLUG}: ansatz needs exactly {list(_ANSATZ_KEYS)}, got {sorted(a)}')
        if not isinstance(a['mode'], str):
            raise ValueError(f'{self.SLUG}: ansatz mode must be a string label')
        return {'mode': a['mode'], 'A1': float(a['A1']), 'A2': float(a['A2']), 'A3': float(a['A3'])}

    def _structure(self, structure):
        return self.STRUCTURES[structure] if isinstance(structure, str) else structure

    # -- box and ansatz
    @staticmethod
    def box(cell, q00):
        """Rectangular cell of the triangular lattice with its first shell at q00
        (stdpfc_cpu/phase_diagram.py:161-167)."""
        nx, ny = cell['uNx'] * cell['Mx'], cell['uNy'] * cell['My']
        a = 4 * np.pi / (3 ** 0.5 * q00)
        h = 4 * np.pi / q00
        return Build2DGeometry(Nx=nx, Ny=ny, Lx=cell['Mx'] * a, Ly=cell['My'] * h)

    @staticmethod
    def three_mode(structure, cell, mean, A, B, C):
        """The field with the given mean and 1-, 2-, 3-mode amplitudes, by the inverse
        real FFT of the sparse spectrum (stdpfc_cpu/phase_diagram.py:171-182)."""
        nx, ny = cell['uNx'] * cell['Mx'], cell['uNy'] * cell['My']
        size = nx * ny
        hat = np.zeros((ny, nx), dtype=complex)
        hat[0, 0] = mean * size
        for pos, amp in zip(structure.kvectors, (A, B, C)):
            rows, cols = np.array(pos).T
            hat[rows * cell['My'], cols * cell['Mx']] = amp * size
        return np.fft.irfftn(hat, s=(ny, nx), axes=(0, 1)).real

    # -- contract
    def build(self, params, structure, cell, ansatz, temp, meanDensity, q00, dt, state=None, nThreads=1):
        """Model + box at q00 + (the ansatz if state is None, else the state) -> Simulation."""
        params = self.validate_params(params)
        structure = self._structure(structure)
        cell = self.validate_cell(cell)
        ansatz = self.validate_ansatz(ansatz)
        field = self.ansatz_field(structure, cell, ansatz, meanDensity) if state is None else state
        sim = self._simulation(params, temp, dt, meanDensity, self.box(cell, q00))
        getattr(sim.State, self.FIELD)[...] = field
        return sim

    def get_state(self, sim):
        return sim.plan.get_state().cpu().numpy()

    def set_state(self, sim, state):
        getattr(sim.State, self.FIELD)[...] = state

    def get_time(self, sim):
        return sim.t

    def set_time(self, sim, t):
        sim.State.t = t

    def get_dt(self, sim):
        return sim.Model.dt

    def step(self, sim):
        sim.TimeStep()
        _count_steps(sim, 1)

    def free_energy(self, sim):
        return sim.CalculateFreeEnergy()

    # -- hooks of the relaxation driver (optional in an adapter; see _hook)
    def step_many(self, sim, n):
        """n steps in one call (graph replay, no host round trip between steps)."""
        sim.TimeSteps(n)
        _count_steps(sim, n)

    def lockstep_key(self, sim):
        """Plans step together only at the same ping-pong parity: the parity of the steps
        a plan has taken since it was built (setting a state keeps the parity)."""
        return getattr(sim, '_relax_steps', 0) & 1

    def snapshot(self, sim, out=None):
        """The state as a device array (into `out` when given); `set_state` takes it back."""
        return sim.plan.get_state(out)

    def release(self, sim):
        sim.plan.close()

    def lockstep(self, sims):
        return _PlanLockstep(sims)


def _count_steps(sim, n):
    sim._relax_steps = getattr(sim, '_relax_steps', 0) + n


# Times a lockstep group held plans at different ping-pong parities and stepped them one
# by one instead of as one batch launch (the schedulers group by parity, so this stays 0
# unless a step path bypasses _count_steps; the GPU tests assert it).
LOCKSTEP_FALLBACKS = {"parity": 0}
# Lockstep groups (batches) the adaptive-dt scheduler built; a group of unchanged members
# is reused from round to round.
LOCKSTEP_BUILDS = {"groups": 0}


class _PlanLockstep:
    """Simulations stepped together through one `Batch`; F of all of them in one copy."""

    def __init__(self, sims):
        self.sims = list(sims)
        self.batch = Batch(self.sims)

    def step(self, n):
        if len({getattr(s, '_relax_steps', 0) & 1 for s in self.sims}) > 1:
            # plans at different ping-pong parities cannot share a launch: step them one by
            # one (a batch step equals each plan's own steps), and say so
            LOCKSTEP_FALLBACKS["parity"] += 1
            warnings.warn("lockstep group at mixed ping-pong parities: stepping its plans one by one",
                          RuntimeWarning, stacklevel=2)
            for sim in self.sims:
                sim.TimeSteps(n)
        else:
            # any refusal here (a plan without a state, parities the host count missed) is a
            # fault of the caller and raises
            self.batch.step(n)
        for sim in self.sims:
            _count_steps(sim, n)

    def free_energies(self):
        return self.batch.reduce()[:, 0]

    def close(self):
        self.batch.close()


class _LoopLockstep:
    """The same interface for an adapter without batches: one member after another."""

    def __init__(self, ad, sims):
        self.ad, self.sims = ad, list(sims)

    def step(self, n):
        for sim in self.sims:
            _steps(self.ad, sim, n)

    def free_energies(self):
        return np.array([self.ad.free_energy(sim) for sim in self.sims], dtype=float)

    def close(self):
        pass


def _steps(ad, sim, n):
    if hasattr(ad, 'step_many'):
        ad.step_many(sim, n)
    else:
        for _ in range(n):
            ad.step(sim)


def _snapshot(ad, sim, out=None):
    return ad.snapshot(sim, out) if hasattr(ad, 'snapshot') else ad.get_state(sim)


def _release(ad, sim):
    if hasattr(ad, 'release'):
        ad.release(sim)


def _lockstep(ad, sims):
    return ad.lockstep(sims) if hasattr(ad, 'lockstep') else _LoopLockstep(ad, sims)


class StdAdapter(_Adapter):
    """stdPFC adapter (models/stdpfc_cpu/phase_diagram.py): absolute amplitudes, no
    rescale of the ansatz."""
    SLUG = 'stdpfc_b200'
    STRUCTURES = _diag.STRUCTURES
    FIELD = 'n'

    def ansatz_field(self, structure, cell, ansatz, mean):
        s = structure.amplitudeSign * structure.amplitudeScale
        return self.three_mode(structure, cell, mean, s * ansatz['A1'], s * ansatz['A2'], s * ansatz['A3'])

    def _simulation(self, params, temp, dt, mean, geometry):
        model = _stdpfc.BuildStdPFCModelParameters(Gamma=params['Gamma'], beta=params['beta'], q0=params['q0'],
                                                   epsilon=temp, g=params['g'], dt=dt, meanDensity=mean)
        return _stdpfc.BuildB200_Simulation(model, geometry, precision=self.precision, device=self.device)

    def diagnose(self, sim, structure, cell):
        """fitness, (|A|, |B|, |C|) and maxima per cell on the device
        (stdpfc_cpu/phase_diagram.py:286-296)."""
        d = _diag.diagnose(sim, self._structure(structure), self.validate_cell(cell))
        return _diag.Diagnostics(d.fitness, d.amplitudes, {'maxima_per_cell': d.details['maxima_per_cell']})


def scaled_fitness(fit_plus, fit_minus, e, s):
    """1 - |mean((d - s e)^2)| for a field deviation d (field minus its mean) and a rebuilt
    deviation e, from the fitnesses against the rebuilt field and its mirror about the
    mean, 1 - D+ and 1 - D- with D+- = mean((d -+ e)^2) = V -+ 2 X + E (V = mean(d^2),
    X = mean(d e), E = mean(e^2), taken from `e` on the host): the log adapter's fitness
    against its 3-mode field rescaled by s (logpfc_cpu/phase_diagram.py:196-199, 220-222)."""
    d_plus, d_minus = 1.0 - fit_plus, 1.0 - fit_minus
    E = float(np.mean(e * e))
    X = (d_minus - d_plus) / 4.0
    V = (d_plus + d_minus) / 2.0 - E
    return 1.0 - abs(V - 2.0 * s * X + s * s * E)


class LogAdapter(_Adapter):
    """logPFC adapter (models/logpfc_cpu/phase_diagram.py): amplitudes in units of the
    mean density, the 3-mode field rescaled towards the mean where it would go negative."""
    SLUG = 'logpfc_b200'
    STRUCTURES = LOG_STRUCTURES
    FIELD = 'phi'

    @classmethod
    def _positive(cls, field, mean):
        low = field.min()
        if low < 0:     # logpfc_cpu/phase_diagram.py:196-199
            field = mean + (field - mean) * mean / (mean - low)
        return field

    def ansatz_field(self, structure, cell, ansatz, mean):
        s = structure.amplitudeSign * structure.amplitudeMax * mean
        return self._positive(self.three_mode(structure, cell, mean, s * ansatz['A1'], s * ansatz['A2'],
                                              s * ansatz['A3']), mean)

    def _simulation(self, params, temp, dt, mean, geometry):
        model = _logpfc.BuildLogPFCModelParameters(Gamma=params['Gamma'], beta=params['beta'], q0=params['q0'],
                                                   epsilon=temp, g=params['g'], dt=dt, meanDensity=mean)
        return _logpfc.BuildB200_Simulation(model, geometry, precision=self.precision, device=self.device)

    def diagnose(self, sim, structure, cell):
        """logpfc_cpu/phase_diagram.py:211-223, 309-321: the device's absolute amplitudes
        divided by the mean. Where the rebuilt 3-mode field stays non-negative (its
        minimum is taken on the host from the four numbers) the fitness is the device's.
        Where the reference rescales it towards the mean by s = mean / (mean - min), a
        second device pass with the amplitude sign flipped gives the fitness against the
        rebuilt field mirrored about the mean, and the rescaled fitness follows from the
        two (`scaled_fitness`); the field stays on the device."""
        st, c = self._structure(structure), self.validate_cell(cell)
        d = _diag.diagnose(sim, st, c)
        mean = d.details['mean']
        amps = tuple(abs(a / mean) for a in d.amplitudes)
        sign = st.amplitudeSign
        rebuilt = self.three_mode(st, c, mean, *(sign * a * mean for a in amps))
        fitness = d.fitness
        low = rebuilt.min()
        if low < 0:
            mirrored = _diag.diagnose(sim, replace(st, amplitudeSign=-sign), c)
            fitness = scaled_fitness(d.fitness, mirrored.fitness, rebuilt - mean, mean / (mean - low))
        return _diag.Diagnostics(fitness, amps, {'maxima_per_cell': d.details['maxima_per_cell']})

    def frozen_field(self, state, params, temp, cell):
        """f(q) and q_opt of a field frozen on the grid (logpfc_cpu/phase_diagram.py:
        465-505), moments on the device."""
        return _diag.frozen_field(state, params, temp, cell)

    def defect_diagnostics(self, state, cell):
        """Peak spread, sub-q ratio, peak count and flag (logpfc_cpu/phase_diagram.py:
        509-528), on the device."""
        return _diag.defect_diagnostics(state, cell)


# ---------------------------------------------------------------- one evaluation
class _Run:
    """Settings of one set of evaluations (the MinimizeFreeEnergy attributes the
    relaxation reads, q0star.py:174-224)."""

    def __init__(self, adapter, params, structure, cell, ansatz, relax):
        self.ad = adapter
        self.params = adapter.validate_params(params)
        self.structure = adapter._structure(structure)
        self.cell = adapter.validate_cell(cell)
        self.ansatz = adapter.validate_ansatz(ansatz)
        self.relax = relax

    def generate(self, temp, mean, q00, dt, state=None):
        """q0star.py:227-252: build, and add the seeded relative noise to a fresh ansatz."""
        ad, r = self.ad, self.relax
        sim = ad.build(self.params, self.structure, self.cell, self.ansatz, temp, mean, q00, dt, state=state)
        if state is None and r.noise:
            rng = np.random.default_rng(r.seed)
            phi = ad.get_state(sim)
            m = phi.mean()
            phi = phi * (1.0 + r.noise * rng.standard_normal(phi.shape))
            ad.set_state(sim, phi + (m - phi.mean()))
        return sim

    def amplitude(self, sim):
        return self.ad.diagnose(sim, self.structure, self.cell).amplitudes[0]

    def take_step(self, sim, point, stepT, depth, counter, f_last=None):
        """One block on one plan with the rollback recursion (q0star.py:261-307); returns
        delta f. `counter` is a one-element list of steps taken."""
        ad, r = self.ad, self.relax
        dt = ad.get_dt(sim)
        mini = int(round(stepT / dt))
        phi_last = _snapshot(ad, sim)
        t_last = ad.get_time(sim)
        f_last = ad.free_energy(sim) if f_last is None else f_last
        _steps(ad, sim, mini)
        counter[0] += mini
        f = ad.free_energy(sim)
        delta_f = f - f_last
        if np.isnan(f) or delta_f > r.fTol * abs(f_last):
            return self.rollback(sim, point, stepT, depth, counter, phi_last, t_last, f_last, bool(np.isnan(f)))
        return delta_f

    def rollback(self, sim, point, stepT, depth, counter, phi_last, t_last, f_last, nan):
        """Restore the block's start and redo it at dt/divs in divs sub-blocks
        (q0star.py:278-305)."""
        ad, r = self.ad, self.relax
        ad.set_state(sim, phi_last)
        ad.set_time(sim, t_last)
        if depth >= r.maxDepth:
            raise MaxDepthReached(f'Max recursion depth reached at t={ad.get_time(sim):0.6f}', nan=nan)
        divs = r.divs
        sub = self.generate(*point, ad.get_dt(sim) / divs, state=phi_last)
        try:
            ad.set_time(sub, ad.get_time(sim))
            for _ in range(divs):
                self.take_step(sub, point, stepT / divs, depth + 1, counter)
                ad.set_state(sim, _snapshot(ad, sub))
                ad.set_time(sim, ad.get_time(sub))
        finally:
            _release(ad, sub)
        return ad.free_energy(sim) - f_last

    def adapt_dt(self, sim, point, stepT, delta_f, f, A, A_last, dt_max):
        """q0star.py:309-327: the next block's dt from the block's relative rate; a new
        plan only where dt changes. Returns (sim, dt_max)."""
        ad, r = self.ad, self.relax
        dt = ad.get_dt(sim)
        rate = max(abs(delta_f) / max(abs(f), 1e-300), abs(A - A_last) / max(A, 1e-300)) / stepT
        target = r.dtMax / np.sqrt(1.0 + (rate / r.dtRate) ** 2)
        target = min(max(target, r.dt), r.dtMax, dt * r.dtGrow)
        mini = int(np.ceil(stepT / target - 1e-9))
        new = stepT / mini
        if abs(new - dt) <= 1e-12 * dt:
            return sim, dt_max
        t = ad.get_time(sim)
        fresh = self.generate(*point, new, state=_snapshot(ad, sim))
        ad.set_time(fresh, t)
        _release(ad, sim)
        return fresh, max(dt_max, new)

    def first_dt(self):
        r = self.relax
        return r.stepT / int(np.ceil(r.stepT / r.dt))

    def check(self, sim, delta_f, f_last, A_last):
        """The stop tests after a block (q0star.py:384-398): (stop or None, A)."""
        r = self.relax
        diag = self.ad.diagnose(sim, self.structure, self.cell)
        fitness, A = diag.fitness, diag.amplitudes[0]
        if r.requiredFitness is not None and fitness < r.requiredFitness:
            return STOP_POOR_FIT, A
        if A < r.minimumA:
            return STOP_MIN_AMPLITUDE, A
        if abs(delta_f) <= r.fTol * abs(f_last) and abs(A - A_last) <= r.ATol * A:
            return STOP_CONVERGED, A
        return None, A

    def finish(self, sim, stop, steps, dt_max, keep_state):
        f = self.ad.free_energy(sim)
        diag = self.ad.diagnose(sim, self.structure, self.cell)
        state = self.ad.get_state(sim) if keep_state else None
        return RelaxResult(float(f), float(diag.fitness), tuple(float(a) for a in diag.amplitudes), stop, steps,
                           float(dt_max), state)


def get_f_abc(adapter, params, structure, cell, ansatz, relax, temp, meanDensity, q00, state=None,
              keep_state=False):
    """`Get_f_ABC` (q0star.py:329-407) for one point on one plan; returns a RelaxResult."""
    run = _Run(adapter, params, structure, cell, ansatz, relax)
    return _single(run, (temp, meanDensity, q00), state, keep_state)


def _single(run, point, state, keep_state):
    ad, r = run.ad, run.relax
    blocks = int(r.totalT / r.stepT)
    sim = run.generate(*point, run.first_dt(), state=state)
    try:
        f_last = ad.free_energy(sim)
        A_last = run.amplitude(sim)
        stop, counter, dt_max = STOP_TOTALT, [0], ad.get_dt(sim)
        for _ in range(blocks):
            try:
                if r.dtMax is None:
                    delta_f = run.take_step(sim, point, r.stepT, 0, counter, f_last)
                else:       # sub-blocks with dt adapted after each (q0star.py:362-372)
                    f0, sub_t = f_last, r.stepT / r.dtChecks
                    As = A_last
                    for k in range(r.dtChecks):
                        d_sub = run.take_step(sim, point, sub_t, 0, counter)
                        fs_new = ad.free_energy(sim)
                        As_new = run.amplitude(sim)
                        if k < r.dtChecks - 1:
                            sim, dt_max = run.adapt_dt(sim, point, sub_t, d_sub, fs_new, As_new, As, dt_max)
                        As = As_new
                    delta_f = ad.free_energy(sim) - f0
            except MaxDepthReached as e:
                stop = STOP_NAN if e.nan else STOP_MAX_DEPTH
                break
            f_last = ad.free_energy(sim)
            reason, A = run.check(sim, delta_f, f_last, A_last)
            if reason is not None:
                stop = reason
                break
            if r.dtMax is not None:
                sim, dt_max = run.adapt_dt(sim, point, r.stepT / r.dtChecks, delta_f / r.dtChecks, f_last, A,
                                           A_last, dt_max)
            A_last = A
        return run.finish(sim, stop, counter[0], dt_max, keep_state)
    finally:
        _release(ad, sim)


# ---------------------------------------------------------------- adaptive dt in lockstep
# The one-point evaluation again, written as a generator that yields (simulation, steps)
# wherever it steps and is resumed once those steps are done, so that a scheduler can
# step the members that ask for the same number of steps together (their dt may differ:
# each plan steps with its own coefficients). Every adapter call is the one `_single`,
# `_Run.take_step` and `_Run.rollback` make, in the same order.
def _take_step_gen(run, sim, point, stepT, depth, counter, f_last=None):
    ad, r = run.ad, run.relax
    mini = int(round(stepT / ad.get_dt(sim)))
    phi_last = _snapshot(ad, sim)
    t_last = ad.get_time(sim)
    f_last = ad.free_energy(sim) if f_last is None else f_last
    yield sim, mini
    counter[0] += mini
    f = ad.free_energy(sim)
    delta_f = f - f_last
    if np.isnan(f) or delta_f > r.fTol * abs(f_last):
        ad.set_state(sim, phi_last)
        ad.set_time(sim, t_last)
        if depth >= r.maxDepth:
            raise MaxDepthReached(f'Max recursion depth reached at t={ad.get_time(sim):0.6f}', nan=bool(np.isnan(f)))
        sub = run.generate(*point, ad.get_dt(sim) / r.divs, state=phi_last)
        try:
            ad.set_time(sub, ad.get_time(sim))
            for _ in range(r.divs):
                yield from _take_step_gen(run, sub, point, stepT / r.divs, depth + 1, counter)
                ad.set_state(sim, _snapshot(ad, sub))
                ad.set_time(sim, ad.get_time(sub))
        finally:
            _release(ad, sub)
        return ad.free_energy(sim) - f_last
    return delta_f


def _single_gen(run, point, state, keep_state):
    """`_single` with adaptive dt as a generator; returns the RelaxResult."""
    ad, r = run.ad, run.relax
    sim = run.generate(*point, run.first_dt(), state=state)
    try:
        f_last = ad.free_energy(sim)
        A_last = run.amplitude(sim)
        stop, counter, dt_max = STOP_TOTALT, [0], ad.get_dt(sim)
        for _ in range(int(r.totalT / r.stepT)):
            try:
                f0, sub_t = f_last, r.stepT / r.dtChecks
                As = A_last
                for k in range(r.dtChecks):
                    d_sub = yield from _take_step_gen(run, sim, point, sub_t, 0, counter)
                    fs_new = ad.free_energy(sim)
                    As_new = run.amplitude(sim)
                    if k < r.dtChecks - 1:
                        sim, dt_max = run.adapt_dt(sim, point, sub_t, d_sub, fs_new, As_new, As, dt_max)
                    As = As_new
                delta_f = ad.free_energy(sim) - f0
            except MaxDepthReached as e:
                stop = STOP_NAN if e.nan else STOP_MAX_DEPTH
                break
            f_last = ad.free_energy(sim)
            reason, A = run.check(sim, delta_f, f_last, A_last)
            if reason is not None:
                stop = reason
                break
            sim, dt_max = run.adapt_dt(sim, point, r.stepT / r.dtChecks, delta_f / r.dtChecks, f_last, A, A_last,
                                       dt_max)
            A_last = A
        return run.finish(sim, stop, counter[0], dt_max, keep_state)
    finally:
        _release(ad, sim)


def _adaptive_batch(run, points, states, keep_state):
    """Adaptive-dt evaluations in lockstep: each round, the members' pending step
    requests are grouped by step count and each group is stepped as one batch."""
    ad = run.ad
    gens = [_single_gen(run, p, s, keep_state) for p, s in zip(points, states)]
    results = [None] * len(gens)
    pending = {}
    # lockstep groups by their member simulations (the key holds them, so identities are
    # not reused while cached): a group of the same members, whatever its step count or
    # parity, steps through the same batch in the next round; a group whose members
    # changed is closed at the end of the round it was last used in
    locks = {}
    try:
        for i, g in enumerate(gens):
            try:
                pending[i] = next(g)
            except StopIteration as e:
                results[i] = e.value
        while pending:
            groups = {}
            for i, (sim, n) in pending.items():
                key = (n, ad.lockstep_key(sim) if hasattr(ad, 'lockstep_key') else None)
                groups.setdefault(key, []).append(i)
            used = set()
            for (n, _), idx in groups.items():
                members = tuple(pending[i][0] for i in idx)
                lock = locks.get(members)
                if lock is None:
                    lock = locks[members] = _lockstep(ad, list(members))
                    LOCKSTEP_BUILDS["groups"] += 1
                used.add(members)
                lock.step(n)
            for members in [m for m in locks if m not in used]:
                locks.pop(members).close()
            for i in sorted(pending):
                try:
                    pending[i] = gens[i].send(None)
                except StopIteration as e:
                    results[i] = e.value
                    del pending[i]
        return results
    finally:
        for lock in locks.values():
            lock.close()
        for g in gens:
            g.close()


# ---------------------------------------------------------------- many evaluations
class _Member:
    def __init__(self, index, point, sim, f_last, A_last):
        self.index, self.point, self.sim = index, point, sim
        self.f_last, self.A_last = f_last, A_last
        self.counter = [0]
        self.snapshot = None     # the state at the start of the block (device array)
        self.t_last = 0.0        # the time at the start of the block


def get_f_abc_batch(adapter, params, structure, cell, ansatz, relax, points, states=None, keep_state=False):
    """`Get_f_ABC` for every (temp, meanDensity, q00) of `points`, the members stepped
    together (see the module docstring). Returns RelaxResults in the order of `points`,
    each equal to what `get_f_abc` returns for that point. With adaptive dt
    (relax.dtMax set) every member has its own dt schedule: the members that ask for the
    same number of steps next are stepped together (`_adaptive_batch`)."""
    run = _Run(adapter, params, structure, cell, ansatz, relax)
    points = [tuple(float(v) for v in p) for p in points]
    states = [None] * len(points) if states is None else list(states)
    if len(states) != len(points):
        raise ValueError('states must match points')
    if relax.dtMax is not None:
        return _adaptive_batch(run, points, states, keep_state)
    ad, r = run.ad, run.relax
    dt = run.first_dt()
    mini = int(round(r.stepT / dt))
    results = [None] * len(points)
    members = []
    batch, in_batch = None, None
    try:
        for i, (p, s) in enumerate(zip(points, states)):
            sim = run.generate(*p, dt, state=s)
            members.append(_Member(i, p, sim, ad.free_energy(sim), run.amplitude(sim)))
        active = list(members)
        for _ in range(int(r.totalT / r.stepT)):
            if not active:
                break
            if in_batch != [m.index for m in active]:
                if batch is not None:
                    batch.close()
                batch = _lockstep(ad, [m.sim for m in active])
                in_batch = [m.index for m in active]
            for m in active:
                m.snapshot = _snapshot(ad, m.sim, m.snapshot)
                m.t_last = ad.get_time(m.sim)
            batch.step(mini)
            fs = batch.free_energies()
            still = []
            for m, f in zip(active, fs):
                m.counter[0] += mini
                delta_f = f - m.f_last
                stop = None
                if np.isnan(f) or delta_f > r.fTol * abs(m.f_last):
                    try:
                        delta_f = run.rollback(m.sim, m.point, r.stepT, 0, m.counter, m.snapshot, m.t_last,
                                               m.f_last, bool(np.isnan(f)))
                    except MaxDepthReached as e:
                        stop = STOP_NAN if e.nan else STOP_MAX_DEPTH
                    if stop is None:
                        f = ad.free_energy(m.sim)
                if stop is None:
                    m.f_last = f
                    stop, A = run.check(m.sim, delta_f, m.f_last, m.A_last)
                    m.A_last = A
                if stop is None:
                    still.append(m)
                else:
                    results[m.index] = run.finish(m.sim, stop, m.counter[0], dt, keep_state)
            active = still
        for m in active:
            results[m.index] = run.finish(m.sim, STOP_TOTALT, m.counter[0], dt, keep_state)
        return results
    finally:
        if batch is not None:
            batch.close()
        for m in members:
            _release(ad, m.sim)


# ---------------------------------------------------------------- q0* search
MSG_INSUFFICIENT_POINTS = 'Insufficient points found that satisfy fitness constraints.'
MSG_NO_LOCAL_MINIMUM = 'No local minimum found for q00.'
STATUS_OK = 'ok'
STATUS_INSUFFICIENT_POINTS = 'insufficient_points'
STATUS_NO_LOCAL_MINIMUM = 'no_local_minimum'


class InsufficientPoints(Exception):
    """Too few accepted q00 points (q0star.py:87-88)."""


class NoLocalMinimum(Exception):
    """The spline of f(q00) has no usable minimum (q0star.py:91-92)."""


@dataclass(frozen=True)
class QScanSettings:
    """q00 scan settings with the reference's names and defaults (q0star.py:153-164)."""
    passes: int
    Deltaq: float
    q00_Steps: int
    Deltaq_Refinement: float
    q00_start: float = 1.0
    minPoints: int = 5


@dataclass
class Q0StarResult:
    """One (temp, meanDensity): q0*, f at q0*, and the status and message that the
    reference's scan_density records for it (NaN q0* and fmin unless the status is ok)."""
    temp: float
    meanDensity: float
    q0star: float
    fmin: float
    status: str
    message: str


def _q_range(q_best, dq, n):
    return np.linspace(q_best - n // 2 * dq, q_best + n // 2 * dq, n, endpoint=True)


def _refine(q00_range, f_values, fit_values, A_values, relax, min_points):
    """One pass's decision (q0star.py:441-478): accept the points whose fitness and
    amplitude pass, spline f over the contiguous accepted run around the lowest accepted
    f, and return (the minimum of the spline nearest that point, the spline)."""
    from scipy.interpolate import CubicSpline
    rf = -np.inf if relax.requiredFitness is None else relax.requiredFitness
    accepted = (fit_values >= rf) & (A_values >= relax.minimumA)
    if q00_range[accepted].size < min_points:
        raise InsufficientPoints(MSG_INSUFFICIENT_POINTS)
    q_min = q00_range[accepted][np.argmin(f_values[accepted])]
    i_min = np.flatnonzero(accepted)[np.argmin(f_values[accepted])]
    lo, hi = i_min, i_min
    while lo > 0 and accepted[lo - 1]:
        lo -= 1
    while hi < accepted.size - 1 and accepted[hi + 1]:
        hi += 1
    if hi - lo + 1 < min_points:
        raise InsufficientPoints(MSG_INSUFFICIENT_POINTS)
    spline = CubicSpline(q00_range[lo:hi + 1], f_values[lo:hi + 1])
    roots = spline.derivative().roots(extrapolate=False)
    roots = roots[spline.derivative(2)(roots) > 0]
    if roots.size == 0:
        raise NoLocalMinimum(MSG_NO_LOCAL_MINIMUM)
    return np.abs(min(roots, key=lambda x: abs(x - q_min))), spline


def find_q0star_batch(adapter, params, structure, cell, ansatz, relax, qscan, targets, min_points=None,
                      record=None):
    """`Find_q0Star` (q0star.py:409-478) for every (temp, meanDensity) of `targets`: pass
    k of all targets still searching is one `get_f_abc_batch` over all their q00 points
    (passes x q00_Steps evaluations per target). Returns Q0StarResults in the order of
    `targets`; a target whose pass raised InsufficientPoints or NoLocalMinimum carries that
    status and message. `record`, if given, receives the reference's per-evaluation dict
    plus the target's index ('target')."""
    min_points = qscan.minPoints if min_points is None else min_points
    targets = [(float(t), float(m)) for t, m in targets]
    best = [qscan.q00_start] * len(targets)
    dq = [qscan.Deltaq] * len(targets)
    spline = [None] * len(targets)
    status = [None] * len(targets)
    message = [''] * len(targets)
    for pass_idx in range(qscan.passes):
        alive = [j for j in range(len(targets)) if status[j] is None]
        if not alive:
            break
        ranges = {j: _q_range(best[j], dq[j], qscan.q00_Steps) for j in alive}
        points = [(*targets[j], float(q)) for j in alive for q in ranges[j]]
        results = get_f_abc_batch(adapter, params, structure, cell, ansatz, relax, points)
        for k, j in enumerate(alive):
            rs = results[k * qscan.q00_Steps:(k + 1) * qscan.q00_Steps]
            f_values = np.array([r.f for r in rs])
            fit_values = np.array([np.nan if r.stop in FAILED_STOPS else r.fitness for r in rs])
            A_values = np.array([r.amplitudes[0] for r in rs])
            if record is not None:
                for q, r in zip(ranges[j], rs):
                    record({'target': j, 'pass': pass_idx, 'q00': float(q), 'f': r.f, 'fitness': r.fitness,
                            'amplitudes': r.amplitudes, 'stop': r.stop, 'steps': r.steps, 'dt_max': r.dt_max})
            try:
                best[j], spline[j] = _refine(ranges[j], f_values, fit_values, A_values, relax, min_points)
            except InsufficientPoints as e:
                status[j], message[j] = STATUS_INSUFFICIENT_POINTS, str(e)
            except NoLocalMinimum as e:
                status[j], message[j] = STATUS_NO_LOCAL_MINIMUM, str(e)
            else:
                dq[j] *= qscan.Deltaq_Refinement
    out = []
    for j, (t, m) in enumerate(targets):
        if status[j] is None:
            out.append(Q0StarResult(t, m, float(best[j]), float(spline[j](best[j])), STATUS_OK, ''))
        else:
            out.append(Q0StarResult(t, m, float('nan'), float('nan'), status[j], message[j]))
    return out


def find_q0star(adapter, params, structure, cell, ansatz, relax, qscan, temp, meanDensity, min_points=None,
                record=None):
    """`Find_q0Star` for one (temp, meanDensity): returns (q0*, fmin) or raises
    InsufficientPoints / NoLocalMinimum with the reference's messages."""
    r = find_q0star_batch(adapter, params, structure, cell, ansatz, relax, qscan, [(temp, meanDensity)],
                          min_points=min_points, record=record)[0]
    if r.status == STATUS_INSUFFICIENT_POINTS:
        raise InsufficientPoints(r.message)
    if r.status == STATUS_NO_LOCAL_MINIMUM:
        raise NoLocalMinimum(r.message)
    return r.q0star, r.fmin


# ---------------------------------------------------------------- density scans
FMIN_FILE = 'fmin.npz'
QSCAN_FILE = 'qscan.npz'
STATUS_ERROR = 'error'


def _fmin_arrays(phi, q0star, fmin, status, message, wall_s):
    """The per-density arrays of the reference's fmin.npz (q0star.py:500-509)."""
    return {'phi': np.asarray(phi, dtype=float), 'q0star': np.asarray(q0star, dtype=float),
            'fmin': np.asarray(fmin, dtype=float), 'status': np.asarray(status, dtype=str),
            'message': np.asarray(message, dtype=str), 'wall_s': np.asarray(wall_s, dtype=float)}


def _qscan_arrays(rows, seed, noise):
    """The per-evaluation arrays of the reference's qscan.npz (q0star.py:512-532):
    amplitudes padded with NaN to the widest row."""
    k = max((len(r['amplitudes']) for r in rows), default=0)
    amplitudes = np.full((len(rows), k), np.nan)
    for j, r in enumerate(rows):
        amplitudes[j, :len(r['amplitudes'])] = r['amplitudes']
    return {'phi_index': np.asarray([r['phi_index'] for r in rows], dtype=np.int64),
            'pass_index': np.asarray([r['pass_index'] for r in rows], dtype=np.int64),
            'q00': np.asarray([r['q00'] for r in rows], dtype=float),
            'f': np.asarray([r['f'] for r in rows], dtype=float),
            'fitness': np.asarray([r['fitness'] for r in rows], dtype=float),
            'amplitudes': amplitudes,
            'stop': np.asarray([r['stop'] for r in rows], dtype=str),
            'steps': np.asarray([r['steps'] for r in rows], dtype=np.int64),
            'dt_max': np.asarray([r['dt_max'] for r in rows], dtype=float),
            'seed': np.asarray(seed, dtype=np.int64), 'noise': np.asarray(noise, dtype=float)}


def _save_npz_atomic(path, arrays):
    tmp = path + '.tmp'
    with open(tmp, 'wb') as fh:
        np.savez(fh, **arrays)
    os.replace(tmp, path)


def _load_checkpoint(checkpoint, phi):
    """(old fmin arrays, indices with a status, their q-scan rows), or None without a
    checkpoint; a checkpoint of another density list is refused (q0star.py:535-563)."""
    path = os.path.join(checkpoint, FMIN_FILE)
    if not os.path.exists(path):
        return None
    with np.load(path, allow_pickle=False) as z:
        old = {k: z[k] for k in z.files}
    if old['phi'].shape != phi.shape or not np.array_equal(old['phi'], phi):
        raise ValueError(f'{path} holds a different density list; refusing to resume into it')
    done = {i for i, s in enumerate(old['status']) if str(s)}
    rows = []
    qpath = os.path.join(checkpoint, QSCAN_FILE)
    if os.path.exists(qpath):
        with np.load(qpath, allow_pickle=False) as z:
            q = {k: z[k] for k in z.files}
        for j in range(q['q00'].size):
            i = int(q['phi_index'][j])
            if i not in done:
                continue
            amps = q['amplitudes'][j]
            rows.append({'phi_index': i, 'pass_index': int(q['pass_index'][j]), 'q00': float(q['q00'][j]),
                         'f': float(q['f'][j]), 'fitness': float(q['fitness'][j]),
                         'amplitudes': tuple(float(a) for a in amps[~np.isnan(amps)]), 'stop': str(q['stop'][j]),
                         'steps': int(q['steps'][j]), 'dt_max': float(q['dt_max'][j])})
    return old, done, rows


def scan_density_batch(adapter, params, structure, cell, ansatz, relax, qscan, temp, densities, checkpoint=None,
                       chunk=None):
    """`scan_density` (q0star.py:566-635): q0* and fmin over a density list at one
    temperature, with the reference's result arrays, status codes and checkpoint files
    (fmin.npz and qscan.npz, rewritten atomically; a restart skips the densities that have
    a status). The densities run as batched searches (`find_q0star_batch`) of `chunk`
    densities (default: all), a checkpoint after each; `wall_s` is the chunk's wall time
    shared evenly by its densities. A chunk that raises anything but the two search
    failures is redone one density at a time, so the error costs that density only
    (status 'error', message 'Type: text')."""
    phi = np.asarray(list(densities), dtype=float)
    n = phi.size
    q0star, fmin = [np.nan] * n, [np.nan] * n
    status, message, wall_s = [''] * n, [''] * n, [np.nan] * n
    rows, done = [], set()
    if checkpoint is not None:
        prev = _load_checkpoint(checkpoint, phi)
        if prev is not None:
            old, done, rows = prev
            for i in done:
                q0star[i], fmin[i] = float(old['q0star'][i]), float(old['fmin'][i])
                status[i], message[i] = str(old['status'][i]), str(old['message'][i])
                wall_s[i] = float(old['wall_s'][i])
    todo = [i for i in range(n) if i not in done]
    size = len(todo) if not chunk else int(chunk)
    prov = (relax.seed, relax.noise)

    def search(indices):
        recs = []
        t0 = time.perf_counter()
        res = find_q0star_batch(adapter, params, structure, cell, ansatz, relax, qscan,
                                [(temp, phi[i]) for i in indices], record=recs.append)
        return res, recs, time.perf_counter() - t0

    for c0 in range(0, len(todo), max(size, 1)):
        part = todo[c0:c0 + max(size, 1)]
        try:
            outs = [search(part)]
            groups = [part]
        except Exception:
            outs, groups = [], []
            for i in part:
                try:
                    outs.append(search([i]))
                except Exception as e:
                    status[i], message[i] = STATUS_ERROR, f'{type(e).__name__}: {e}'
                    wall_s[i] = 0.0
                    continue
                groups.append([i])
        for (res, recs, wall), idx in zip(outs, groups):
            for r, i in zip(res, idx):
                q0star[i], fmin[i], status[i], message[i] = r.q0star, r.fmin, r.status, r.message
                wall_s[i] = wall / len(idx)
            for r in recs:
                rows.append({'phi_index': idx[r['target']], 'pass_index': r['pass'], 'q00': r['q00'], 'f': r['f'],
                             'fitness': r['fitness'], 'amplitudes': r['amplitudes'], 'stop': r['stop'],
                             'steps': r['steps'], 'dt_max': r['dt_max']})
        if checkpoint is not None:
            _save_npz_atomic(os.path.join(checkpoint, QSCAN_FILE), _qscan_arrays(rows, *prov))
            _save_npz_atomic(os.path.join(checkpoint, FMIN_FILE),
                             _fmin_arrays(phi, q0star, fmin, status, message, wall_s))
    result = _fmin_arrays(phi, q0star, fmin, status, message, wall_s)
    result['qscan'] = _qscan_arrays(rows, *prov)
    return result


# ---------------------------------------------------------------- frozen-q search
STATUS_NOT_CONVERGED = 'not_converged'
FROZEN_SCHEDULE = (1e-6, 1e-8, 1e-10, 1e-12)


@dataclass(frozen=True)
class FrozenQSettings:
    """Settings of the frozen-q search with the reference's names and defaults
    (phase_diagram/frozen_q.py:52-61): fTol per stage (the last is the final one), qTol
    on |q_opt - q| at the final stage, maxIter relax/jump iterations, and the edge pass
    of the density scan."""
    schedule: tuple = FROZEN_SCHEDULE
    qTol: float = 1e-8
    maxIter: int = 40
    edge: bool = True
    maxPast: int = 3


def _stage_relax(relax, settings, stage):
    """The relaxation settings of a stage (frozen_q.py:85-90): that stage's fTol, and ATol
    loosened with it except at the final stage."""
    f_tol = float(settings.schedule[stage])
    a_tol = relax.ATol if stage == len(settings.schedule) - 1 else max(relax.ATol, 1e6 * f_tol)
    return replace(relax, fTol=f_tol, ATol=a_tol)


def solve_frozen_q_batch(adapter, params, structure, cell, ansatz, relax, settings, temp, densities,
                         q_start=1.0, states=None):
    """`MinimizeFrozenQ.solve` (frozen_q.py:92-148) for every density at once: each
    iteration relaxes every unfinished density at its box scale q from its carried field
    (the densities at one stage of the fTol schedule in one `get_f_abc_batch`), then moves q
    to q_opt of the relaxed field frozen on the grid (`adapter.frozen_field`), tightening
    fTol stage by stage, until |q_opt - q| < qTol at the final stage with a converged
    stop. Returns one record per density with the reference's fields (status, q = q_opt
    of the final field, q_relaxed, f, f_frozen, fitness, A1.., stop, steps, iters, wall_s,
    q_start, message, and the adapter's defect diagnostics where it has them); statuses
    'ok', 'not_converged', a rejected relaxation's stop, or 'error'."""
    if not hasattr(adapter, 'frozen_field'):
        raise ValueError(f'adapter {getattr(adapter, "SLUG", adapter)!r} has no frozen_field')
    if len(settings.schedule) < 1:
        raise ValueError('schedule needs at least one fTol')
    params = adapter.validate_params(params)
    cell = adapter.validate_cell(cell)
    dens = [float(p) for p in densities]
    n = len(dens)
    last_stage = len(settings.schedule) - 1
    t0 = time.perf_counter()
    q = [float(q_start)] * n
    carry = [None] * n if states is None else list(states)
    stage, steps, last = [0] * n, [0] * n, [None] * n
    phi = [None] * n
    error = [None] * n
    active = list(range(n))
    for it in range(settings.maxIter):
        if not active:
            break
        nxt = []
        for stg in sorted({stage[i] for i in active}):
            group = [i for i in active if stage[i] == stg]
            rs = _stage_relax(relax, settings, stg)
            try:
                res = get_f_abc_batch(adapter, params, structure, cell, ansatz, rs,
                                      [(temp, dens[i], q[i]) for i in group], states=[carry[i] for i in group],
                                      keep_state=True)
            except Exception:   # isolate the failing density, as independent solves would
                res = []
                for i in group:
                    try:
                        res.append(get_f_abc(adapter, params, structure, cell, ansatz, rs, temp, dens[i], q[i],
                                             state=carry[i], keep_state=True))
                    except Exception as e:  # noqa: BLE001
                        error[i] = f'{type(e).__name__}: {e}'
                        res.append(None)
            for i, r in zip(group, res):
                if r is None:
                    continue
                try:
                    steps[i] += r.steps
                    phi[i] = r.state
                    ff = adapter.frozen_field(r.state, params, temp, cell)
                    qn = float(ff.q_opt())
                    last[i] = dict(q=q[i], q_opt=qn, f=float(r.f), f_frozen=float(ff.f(qn)),
                                   fitness=float(r.fitness), amps=[float(a) for a in r.amplitudes], stop=r.stop,
                                   it=it)
                except Exception as e:  # noqa: BLE001
                    error[i] = f'{type(e).__name__}: {e}'
                    continue
                if r.stop not in (STOP_CONVERGED, STOP_TOTALT):
                    continue
                dq = qn - q[i]
                carry[i], q[i] = r.state, qn
                if stage[i] < last_stage:
                    stage[i] += 1
                elif abs(dq) < settings.qTol and r.stop == STOP_CONVERGED:
                    continue
                nxt.append(i)
        active = sorted(nxt)
    wall = (time.perf_counter() - t0) / max(n, 1)
    out = []
    dd = getattr(adapter, 'defect_diagnostics', None)
    for i in range(n):
        rec = dict(method='frozen-q', q_start=float(q_start), message='')
        if error[i] is not None:
            rec.update(status=STATUS_ERROR, message=error[i], steps=steps[i], wall_s=wall)
            out.append(rec)
            continue
        lt = last[i]
        ok = lt['stop'] == STOP_CONVERGED and stage[i] == last_stage and abs(lt['q_opt'] - lt['q']) < settings.qTol
        if ok:
            status = STATUS_OK
        elif lt['stop'] in (STOP_CONVERGED, STOP_TOTALT):
            status = STATUS_NOT_CONVERGED
        else:
            status = lt['stop']
        rec.update(status=status, q=lt['q_opt'], q_relaxed=lt['q'], f=lt['f'], f_frozen=lt['f_frozen'],
                   fitness=lt['fitness'], stop=lt['stop'], steps=steps[i], iters=lt['it'] + 1)
        for j, a in enumerate(lt['amps']):
            rec[f'A{j + 1}'] = a
        if dd is not None and phi[i] is not None:
            rec.update(dd(phi[i], cell))
        rec['wall_s'] = wall
        out.append(rec)
    return out


def _is_ok(r):
    return r is not None and r.get('status') == STATUS_OK


def edge_walks(grid, results):
    """(i, d) for every accepted grid index i whose neighbour i + d (d = -1, +1) is not
    accepted (frozen_q.py:166-177). `grid`: sorted densities; `results`: density -> record."""
    out = []
    for i, p in enumerate(grid):
        if not _is_ok(results.get(p)):
            continue
        for d in (-1, 1):
            j = i + d
            if 0 <= j < len(grid) and not _is_ok(results.get(grid[j])):
                out.append((i, d))
    return out


def edge_walk(solve, grid, results, i, d, maxPast=3):
    """From accepted index i outward in direction d, reruns each non-accepted density by
    `solve(phi, q_start)` from a fresh ansatz at q_start = q* of grid[i], until an
    accepted original, the grid's end, or maxPast failures in a row (frozen_q.py:
    180-196). Returns the records with q_start, edge_from and edge_dir."""
    q_seed = float(results[grid[i]]['q'])
    out, fails, j = [], 0, i + d
    while 0 <= j < len(grid) and fails < maxPast:
        p = grid[j]
        if _is_ok(results.get(p)):
            break
        r = dict(solve(p, q_seed))
        r.update(phi=p, q_start=q_seed, edge_from=grid[i], edge_dir=d, pass_='edge')
        out.append(r)
        fails = 0 if _is_ok(r) else fails + 1
        j += d
    return out


def merge_edge(results, edge_records):
    """`results` with every accepted edge record in place of a non-accepted original (the
    lowest f among several accepted edge records of one density; frozen_q.py:199-210)."""
    out = dict(results)
    for r in edge_records:
        if not _is_ok(r):
            continue
        p = r['phi']
        cur = out.get(p)
        if not _is_ok(cur) or (cur.get('pass_') == 'edge' and r['f'] < cur['f']):
            out[p] = r
    return out


def scan_density_frozen(adapter, params, structure, cell, ansatz, relax, settings, temp, densities, q_start=1.0,
                        record=None, done=None):
    """The frozen-q density scan (frozen_q.py:213-243): pass 1 solves every density not
    in `done` (density -> pass-1 record) from q_start, all of them in one
    `solve_frozen_q_batch`; pass 2 (settings.edge) walks outward from the accepted
    densities. `record(rec)` is called after every solve. Returns (final, pass1, edge) as
    the reference does."""
    grid = [float(p) for p in densities]
    if any(b <= a for a, b in zip(grid, grid[1:])):
        raise ValueError('densities must be strictly increasing')
    pass1 = dict(done or {})
    todo = [p for p in grid if p not in pass1]
    if todo:
        for p, r in zip(todo, solve_frozen_q_batch(adapter, params, structure, cell, ansatz, relax, settings, temp,
                                                   todo, q_start=q_start)):
            r.update(phi=p, pass_='indep')
            pass1[p] = r
            if record is not None:
                record(r)
    edge = []
    if settings.edge:
        def solve(p, q):
            r = solve_frozen_q_batch(adapter, params, structure, cell, ansatz, relax, settings, temp, [p],
                                     q_start=q)[0]
            if record is not None:
                record({**r, 'phi': p, 'pass_': 'edge'})
            return r
        for i, d in edge_walks(grid, pass1):
            edge += edge_walk(solve, grid, pass1, i, d, settings.maxPast)
    return merge_edge(pass1, edge), pass1, edge
