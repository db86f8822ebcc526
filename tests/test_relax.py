"""Batched Get_f_ABC relaxation (pfc_models_b200.phase_diagram) against the reference's
phase_diagram/q0star.py:261-407.

CPU: the driver's decisions (convergence, rollback to dt/divs, NaN and depth stops,
poor fit, the amplitude guard, adaptive dt) on a toy adapter whose f and amplitudes are
closed-form functions of time; the batched driver must return exactly what the
one-point driver returns for every point, rollbacks included.

GPU: the logPFC adapter on B200 plans at the three points that the reference's own test
pins (tests/test_phase_diagram_q0star.py:44-58, 489-510: MinimizeFreeEnergy.Get_f_ABC
with run_vals[2] on the 14 x 24, 2 x 1 cell, beta 0.5, g -2): the stop, the step count
exactly (2000, 2000, and 22000 for the honeycomb, whose dt = 0.1 blocks go NaN and are
redone at dt 0.01), f within 1e-12 absolute (the reference test's bound for its
honeycomb value; the converged f differ here only by the FFT's round-off), fitness and
amplitudes within 1e-12 absolute (the reference test's bound). The same three points as
one batch must give the one-point results bit for bit.
"""
import math

import numpy as np
import pytest

from pfc_models_b200 import phase_diagram as pd


# ---------------------------------------------------------------- toy model
class _Diag:
    def __init__(self, fitness, amplitudes):
        self.fitness, self.amplitudes, self.details = fitness, amplitudes, {}


class _Toy:
    def __init__(self, floor, fitness, dt, state, regime):
        self.floor, self.fitness, self.dt, self.x, self.t, self.regime = floor, fitness, dt, state, 0.0, regime


class ToyAdapter:
    """f = floor(q00) + |x|^2 with x decaying by (1 - dt/2) per step; regimes by mean
    density: 0.75 goes NaN after t = 5 unless dt <= 0.05, 0.9 goes NaN after t = 5 at
    any dt, 0.6 keeps f fixed while the amplitude grows as 3e-6 e^t up to 0.3."""
    QSTAR = 1.03
    T_BAD = 5.0
    DT_OK = 0.05

    def __init__(self):
        self.dts, self.from_state, self.steps = [], 0, 0

    def validate_params(self, p):
        return dict(p)

    def validate_cell(self, c):
        return dict(c)

    def validate_ansatz(self, a):
        return dict(a)

    def _structure(self, s):
        return s

    def build(self, params, structure, cell, ansatz, temp, meanDensity, q00, dt, state=None, nThreads=1):
        self.dts.append(dt)
        regime = {0.75: 'stiff', 0.9: 'nan', 0.6: 'seed'}.get(meanDensity, 'plain')
        floor = temp + meanDensity ** 2 + (q00 - self.QSTAR) ** 2
        x = np.full(4, 0.0 if regime == 'seed' else 0.5) if state is None else np.array(state)
        if state is not None:
            self.from_state += 1
        return _Toy(floor, 1.0 - (q00 - self.QSTAR) ** 2, dt, x, regime)

    def get_state(self, sim):
        return sim.x.copy()

    def set_state(self, sim, state):
        sim.x[...] = state

    def get_time(self, sim):
        return sim.t

    def set_time(self, sim, t):
        sim.t = t

    def get_dt(self, sim):
        return sim.dt

    def step(self, sim):
        self.steps += 1
        sim.x *= 1 - 0.5 * sim.dt
        sim.t += sim.dt
        if sim.t >= self.T_BAD and (sim.regime == 'nan' or (sim.regime == 'stiff' and sim.dt > self.DT_OK)):
            sim.x[...] = np.nan

    def free_energy(self, sim):
        return sim.floor + float(np.mean(sim.x ** 2))

    def diagnose(self, sim, structure, cell):
        a = min(0.3, 3e-6 * math.exp(sim.t)) if sim.regime == 'seed' else 0.3
        return _Diag(sim.fitness, (a, 0.0))


TOY = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=0.99, minimumA=1e-6)


def _one(ad, rho, q00=1.0, relax=TOY):
    return pd.get_f_abc(ad, {}, 'blob', {}, {}, relax, 0.1, rho, q00)


def test_converges_in_whole_blocks():
    ad = ToyAdapter()
    r = _one(ad, 0.5)
    assert r.stop == pd.STOP_CONVERGED
    assert r.f == pytest.approx(0.1 + 0.25 + (1.0 - ToyAdapter.QSTAR) ** 2, abs=1e-11)
    assert r.steps == ad.steps and r.steps % 100 == 0 and ad.from_state == 0


def test_rollback_redoes_the_block_at_dt_over_divs():
    ad = ToyAdapter()
    r = _one(ad, 0.75)
    assert r.stop == pd.STOP_CONVERGED and np.isfinite(r.f)
    assert min(ad.dts) == pytest.approx(0.01) and ad.from_state >= 1
    assert r.steps == ad.steps


def test_nan_at_every_dt_stops_at_max_depth():
    ad = ToyAdapter()
    r = _one(ad, 0.9)
    assert r.stop == pd.STOP_NAN and np.isfinite(r.f)
    assert min(ad.dts) == pytest.approx(TOY.dt / TOY.divs ** TOY.maxDepth)


def test_amplitude_guard_waits_for_a_growing_seed():
    r = _one(ToyAdapter(), 0.6)        # A: 0.066 at t = 10, 0.3 at t = 20 and 30
    assert r.stop == pd.STOP_CONVERGED and r.amplitudes[0] == 0.3 and r.steps == 300


def test_poor_fit_and_minimum_amplitude_stops():
    assert _one(ToyAdapter(), 0.5, q00=1.3).stop == pd.STOP_POOR_FIT      # fitness 1 - 0.27^2
    relax = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=None,
                             minimumA=0.5)
    assert _one(ToyAdapter(), 0.5, relax=relax).stop == pd.STOP_MIN_AMPLITUDE


def test_total_time_stop():
    relax = pd.RelaxSettings(dt=0.1, totalT=20.0, stepT=10.0, divs=10, maxDepth=4, requiredFitness=None,
                             minimumA=1e-6)
    r = _one(ToyAdapter(), 0.6, relax=relax)
    assert r.stop == pd.STOP_TOTALT and r.steps == 200


def test_adaptive_dt_grows_the_step():
    relax = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=0.99,
                             minimumA=1e-6, dtMax=1.0)
    r = _one(ToyAdapter(), 0.5, relax=relax)
    assert r.stop == pd.STOP_CONVERGED and r.dt_max > 0.1


def test_batch_returns_the_one_point_results():
    points = [(0.1, 0.5, 1.0), (0.1, 0.75, 1.0), (0.1, 0.9, 1.0), (0.1, 0.6, 1.0), (0.1, 0.5, 1.3),
              (0.2, 0.5, 0.98)]
    ad = ToyAdapter()
    got = pd.get_f_abc_batch(ad, {}, 'blob', {}, {}, TOY, points)
    batch_steps = ad.steps
    want, total = [], 0
    for p in points:
        one = ToyAdapter()
        want.append(pd.get_f_abc(one, {}, 'blob', {}, {}, TOY, *p))
        total += one.steps
    for g, w in zip(got, want):
        assert (g.values(), g.stop, g.steps, g.dt_max) == (w.values(), w.stop, w.steps, w.dt_max)
    assert batch_steps == total == sum(g.steps for g in got)
    assert [g.stop for g in got] == [pd.STOP_CONVERGED, pd.STOP_CONVERGED, pd.STOP_NAN, pd.STOP_CONVERGED,
                                     pd.STOP_POOR_FIT, pd.STOP_CONVERGED]


def test_adapter_validation_and_log_ansatz():
    ad = pd.LogAdapter()
    with pytest.raises(ValueError, match='v0'):
        ad.validate_params({'beta': 1.0, 'g': 0.0, 'v0': 2.0})
    with pytest.raises(ValueError, match='missing'):
        ad.validate_params({'beta': 1.0})
    with pytest.raises(ValueError, match='cell'):
        ad.validate_cell({'uNx': 14, 'uNy': 24, 'Mx': 2})
    with pytest.raises(ValueError, match='ansatz'):
        ad.validate_ansatz({'mode': 'L2H', 'A1': 1.0})
    cell = dict(uNx=14, uNy=24, Mx=2, My=1)
    st = ad.STRUCTURES['triangle']
    # a large ansatz is rescaled towards the mean until its minimum is zero
    big = ad.ansatz_field(st, cell, dict(mode='H2L', A1=3.0, A2=1.0, A3=0.5), 0.5)
    assert big.min() == pytest.approx(0.0, abs=1e-15) and big.mean() == pytest.approx(0.5, abs=1e-15)
    small = ad.ansatz_field(st, cell, dict(mode='L2H', A1=1e-5, A2=1e-6, A3=1e-7), 0.63)
    assert small.min() > 0.62
    assert pd.LOG_STRUCTURES['honeycomb'].amplitudeMax == 1.0 / 6
    g = ad.box(cell, 1.0)
    assert (g.Nx, g.Ny) == (28, 24) and g.Lx == pytest.approx(2 * 4 * math.pi / math.sqrt(3))


# ---------------------------------------------------------------- B200 plans
RELAX = pd.RelaxSettings(dt=0.1, totalT=1e6, stepT=1e2, divs=10, maxDepth=4, requiredFitness=0.99, minimumA=1e-6)
CELL = dict(uNx=14, uNy=24, Mx=2, My=1)
ANSATZ = dict(mode='L2H', A1=1e-5, A2=1e-6, A3=1e-7)
LOG_PARAMS = dict(beta=0.5, g=-2.0, v0=1.0)
# structure, eps, phi, q00, f, fitness, A, B, C, steps: the reference test's pinned values
PINNED = [
    ('triangle', -0.9, 0.63, 0.9638831589013295, -0.553594984894113, 0.9997633941916881, 0.33320928950407136,
     0.03198014374195086, 0.003245425514830756, 2000),
    ('honeycomb', -0.9, 1.2, 1.0, -0.7600664077521084, None, None, None, None, 22000),
    ('stripe', -0.9, 0.88, 1.0, -0.6617397486488582, 0.99983068778873, 0.4718018020045463, 0.021804312871064338,
     0.005226927920294405, 2000),
]


def _check_pinned(r, ref):
    structure, _, _, _, f, fitness, A, B, C, steps = ref
    assert r.stop == pd.STOP_CONVERGED, structure
    assert r.steps == steps, structure
    assert r.f == pytest.approx(f, abs=1e-12), structure
    if fitness is not None:
        assert (r.fitness, *r.amplitudes) == pytest.approx((fitness, A, B, C), abs=1e-12), structure


@pytest.mark.gpu
@pytest.mark.parametrize('ref', PINNED, ids=[p[0] for p in PINNED])
def test_log_get_f_abc_matches_the_reference_pins(ref):
    structure, eps, phi, q00 = ref[:4]
    r = pd.get_f_abc(pd.LogAdapter(), LOG_PARAMS, structure, CELL, ANSATZ, RELAX, eps, phi, q00)
    _check_pinned(r, ref)


@pytest.mark.gpu
def test_log_batch_equals_one_point_runs_bit_for_bit():
    """The three pinned points and two more q00 of the triangle, one batch per
    structure, against the one-point driver."""
    ad = pd.LogAdapter()
    for structure in ('triangle', 'honeycomb', 'stripe'):
        refs = [p for p in PINNED if p[0] == structure]
        points = [p[1:4] for p in refs]
        if structure == 'triangle':
            points += [(-0.9, 0.63, 0.95), (-0.9, 0.63, 0.98)]
        got = pd.get_f_abc_batch(ad, LOG_PARAMS, structure, CELL, ANSATZ, RELAX, points)
        for g, p in zip(got, points):
            w = pd.get_f_abc(ad, LOG_PARAMS, structure, CELL, ANSATZ, RELAX, *p)
            assert (g.values(), g.stop, g.steps) == (w.values(), w.stop, w.steps), (structure, p)
        _check_pinned(got[0], refs[0])


@pytest.mark.gpu
def test_std_adapter_relaxes_a_triangle():
    """stdPFC through the same driver: a 16 x 28 cell at eps -0.25, nbar -0.25 relaxes to a
    converged triangle whose fitness and first amplitude the device and the host agree on."""
    ad = pd.StdAdapter()
    relax = pd.RelaxSettings(dt=0.5, totalT=2e4, stepT=50.0, divs=10, maxDepth=3, requiredFitness=0.9,
                             minimumA=1e-6)
    cell = dict(uNx=16, uNy=28, Mx=1, My=1)
    params = dict(beta=1.0, g=0.0)
    ansatz = dict(mode='L2H', A1=0.5, A2=0.0, A3=0.0)
    r = pd.get_f_abc(ad, params, 'triangle', cell, ansatz, relax, -0.25, -0.25, 1.0, keep_state=True)
    assert r.stop == pd.STOP_CONVERGED
    assert r.fitness > 0.99 and r.amplitudes[0] > 0.05
    b = pd.get_f_abc_batch(ad, params, 'triangle', cell, ansatz, relax, [(-0.25, -0.25, 1.0), (-0.25, -0.25, 0.97)])
    assert (b[0].values(), b[0].steps) == (r.values(), r.steps)


# ---------------------------------------------------------------- q0* search
QSCAN = pd.QScanSettings(passes=3, Deltaq=0.02, q00_Steps=21, Deltaq_Refinement=0.05)


def test_toy_find_q0star_finds_the_known_minimum():
    recs = []
    q, fmin = pd.find_q0star(ToyAdapter(), {}, 'blob', {}, {}, TOY, QSCAN, 0.1, 0.5, record=recs.append)
    assert q == pytest.approx(ToyAdapter.QSTAR, abs=1e-9)
    assert fmin == pytest.approx(0.1 + 0.25, abs=1e-10)
    assert len(recs) == QSCAN.passes * QSCAN.q00_Steps
    assert [r['pass'] for r in recs[::QSCAN.q00_Steps]] == list(range(QSCAN.passes))
    # the pass-0 edges (|q00 - 1.03| > 0.1) fail the fitness test and stop after one block
    assert all(r['stop'] == (pd.STOP_POOR_FIT if r['fitness'] < 0.99 else pd.STOP_CONVERGED) for r in recs)


def test_toy_find_q0star_batch_statuses_and_equality():
    """Several targets in one search equal the one-target searches; a target whose f has
    no minimum in the window and one with too few accepted points get their statuses."""
    class Sloped(ToyAdapter):
        def build(self, params, structure, cell, ansatz, temp, meanDensity, q00, dt, state=None, nThreads=1):
            sim = super().build(params, structure, cell, ansatz, temp, meanDensity, q00, dt, state, nThreads)
            if meanDensity == 0.3:          # f linear in q00: no minimum
                sim.floor, sim.fitness = temp + q00, 1.0
            if meanDensity == 0.2:          # poor fit everywhere
                sim.fitness = 0.5
            return sim
    targets = [(0.1, 0.5), (0.1, 0.3), (0.2, 0.5), (0.1, 0.2)]
    got = pd.find_q0star_batch(Sloped(), {}, 'blob', {}, {}, TOY, QSCAN, targets)
    assert [g.status for g in got] == [pd.STATUS_OK, pd.STATUS_NO_LOCAL_MINIMUM, pd.STATUS_OK,
                                       pd.STATUS_INSUFFICIENT_POINTS]
    assert got[1].message == pd.MSG_NO_LOCAL_MINIMUM and got[3].message == pd.MSG_INSUFFICIENT_POINTS
    assert math.isnan(got[1].q0star) and math.isnan(got[3].fmin)
    for g, (t, m) in zip(got, targets):
        if g.status == pd.STATUS_OK:
            assert (g.q0star, g.fmin) == pd.find_q0star(Sloped(), {}, 'blob', {}, {}, TOY, QSCAN, t, m)
    with pytest.raises(pd.NoLocalMinimum, match='No local minimum'):
        pd.find_q0star(Sloped(), {}, 'blob', {}, {}, TOY, QSCAN, 0.1, 0.3)


@pytest.mark.gpu
def test_log_find_q0star_matches_the_reference_pins():
    """tests/test_phase_diagram_q0star.py:53-56, 529-551: q0* within 1e-8 and fmin within
    1e-13 at (eps -0.9, phi 0.63); (-0.9, 0.51) and (-0.9, 0.52) have no local minimum.
    All three searches run as one batched search."""
    got = pd.find_q0star_batch(pd.LogAdapter(), LOG_PARAMS, 'triangle', CELL, ANSATZ, RELAX, QSCAN,
                               [(-0.9, 0.63), (-0.9, 0.51), (-0.9, 0.52)])
    assert got[0].status == pd.STATUS_OK
    assert got[0].q0star == pytest.approx(0.9638831589507376, abs=1e-8)
    assert got[0].fmin == pytest.approx(-0.5535949848941145, abs=1e-13)
    for g in got[1:]:
        assert (g.status, g.message) == (pd.STATUS_NO_LOCAL_MINIMUM, pd.MSG_NO_LOCAL_MINIMUM)
        assert math.isnan(g.q0star) and math.isnan(g.fmin)


def test_batch_from_given_states_keeps_them_noise_free():
    """The frozen-q use (phase_diagram/frozen_q.py: Get_f_ABC from a given field): no
    noise is added to a given state, and keep_state returns the field at the stop."""
    ad = ToyAdapter()
    relax = pd.RelaxSettings(dt=0.1, totalT=20.0, stepT=10.0, divs=10, maxDepth=4, requiredFitness=None,
                             minimumA=1e-6, noise=0.5)
    x0 = np.full(4, 0.25)
    got = pd.get_f_abc_batch(ad, {}, 'blob', {}, {}, relax, [(0.1, 0.5, 1.0), (0.1, 0.5, 1.03)],
                             states=[x0, x0 * 2], keep_state=True)
    decay = (1 - 0.5 * 0.1) ** 200
    assert got[0].state == pytest.approx(x0 * decay, rel=1e-12)
    assert got[1].state == pytest.approx(2 * x0 * decay, rel=1e-12)
    one = pd.get_f_abc(ToyAdapter(), {}, 'blob', {}, {}, relax, 0.1, 0.5, 1.0, state=x0, keep_state=True)
    assert np.array_equal(one.state, got[0].state) and one.values() == got[0].values()
    assert pd.get_f_abc_batch(ad, {}, 'blob', {}, {}, relax, []) == []
    with pytest.raises(ValueError, match='states'):
        pd.get_f_abc_batch(ad, {}, 'blob', {}, {}, relax, [(0.1, 0.5, 1.0)], states=[x0, x0])


def test_fresh_ansatz_noise_is_seeded_and_mean_preserving():
    """q0star.py:236-244: relative noise from default_rng(seed) with the mean restored,
    the same draws for every point."""
    class Flat(ToyAdapter):
        def build(self, *a, **k):
            sim = super().build(*a, **k)
            sim.x = np.linspace(0.2, 0.8, 4) if k.get('state') is None else sim.x
            return sim
    relax = pd.RelaxSettings(dt=0.1, totalT=10.0, stepT=10.0, divs=10, maxDepth=4, requiredFitness=None,
                             minimumA=1e-6, noise=1e-3, seed=3)
    run = pd._Run(Flat(), {}, 'blob', {}, {}, relax)
    a, b = run.generate(0.1, 0.5, 1.0, 0.1), run.generate(0.1, 0.5, 1.1, 0.1)
    base = np.linspace(0.2, 0.8, 4)
    want = base * (1.0 + 1e-3 * np.random.default_rng(3).standard_normal(4))
    want = want + (base.mean() - want.mean())
    assert np.array_equal(a.x, want) and np.array_equal(b.x, want)


# ---------------------------------------------------------------- density scans
class ScanToy(ToyAdapter):
    """Regimes by mean density: 0.3 no minimum (f linear in q00), 0.2 poor fit
    everywhere, negative densities fail to build, 0.45 fails in a step after t = 5,
    `interrupt_at` raises KeyboardInterrupt in build."""
    interrupt_at = None

    def build(self, params, structure, cell, ansatz, temp, meanDensity, q00, dt, state=None, nThreads=1):
        if meanDensity == self.interrupt_at:
            raise KeyboardInterrupt
        if meanDensity < 0:
            raise ValueError('negative density')
        sim = super().build(params, structure, cell, ansatz, temp, meanDensity, q00, dt, state, nThreads)
        if meanDensity == 0.3:
            sim.floor, sim.fitness = temp + q00, 1.0
        if meanDensity == 0.2:
            sim.fitness = 0.5
        sim.boom = meanDensity == 0.45
        return sim

    def step(self, sim):
        super().step(sim)
        if sim.boom and sim.t >= self.T_BAD:
            raise ValueError('toy step failed')


def _scan(ad, densities, **kw):
    return pd.scan_density_batch(ad, {}, 'blob', {}, {}, TOY, QSCAN, 0.1, densities, **kw)


def test_scan_density_statuses_and_arrays():
    r = _scan(ScanToy(), [0.5, 0.3, 0.2, -1.0, 0.45])
    assert list(r['status']) == ['ok', 'no_local_minimum', 'insufficient_points', 'error', 'error']
    assert list(r['message']) == ['', pd.MSG_NO_LOCAL_MINIMUM, pd.MSG_INSUFFICIENT_POINTS,
                                  'ValueError: negative density', 'ValueError: toy step failed']
    assert r['q0star'][0] == pytest.approx(ToyAdapter.QSTAR, abs=1e-9)
    assert np.isnan(r['q0star'][1:]).all() and np.isnan(r['fmin'][1:]).all()
    qs = r['qscan']
    assert np.bincount(qs['phi_index'], minlength=5).tolist() == [63, 21, 21, 0, 0]
    assert qs['amplitudes'].shape == (105, 2)
    assert set(qs) == {'phi_index', 'pass_index', 'q00', 'f', 'fitness', 'amplitudes', 'stop', 'steps', 'dt_max',
                       'seed', 'noise'}
    assert (int(qs['seed']), float(qs['noise'])) == (0, 1e-10)
    # the batched search equals the one-density searches
    q, f = pd.find_q0star(ScanToy(), {}, 'blob', {}, {}, TOY, QSCAN, 0.1, 0.5)
    assert (r['q0star'][0], r['fmin'][0]) == (q, f)


def test_scan_density_checkpoint_and_resume(tmp_path):
    densities = [0.5, 0.3, 0.55, 0.2]
    fresh = _scan(ScanToy(), densities)
    ad = ScanToy()
    ad.interrupt_at = 0.55
    with pytest.raises(KeyboardInterrupt):
        _scan(ad, densities, checkpoint=str(tmp_path), chunk=1)
    with np.load(tmp_path / pd.FMIN_FILE) as z:
        assert list(z['status']) == ['ok', 'no_local_minimum', '', '']
    resumed = _scan(ScanToy(), densities, checkpoint=str(tmp_path), chunk=2)
    for k in ('q0star', 'fmin', 'status', 'message'):
        assert np.array_equal(resumed[k], fresh[k]) or np.allclose(resumed[k], fresh[k], equal_nan=True), k
    assert resumed['qscan']['q00'].size == fresh['qscan']['q00'].size
    with pytest.raises(ValueError, match='different density list'):
        _scan(ScanToy(), [0.5, 0.3], checkpoint=str(tmp_path))


@pytest.mark.gpu
def test_log_scan_density_with_checkpoint(tmp_path):
    """The reference test's ok and no-local-minimum points through the batched density
    scan on B200 plans, with checkpoint files: the ok point's q0* and fmin equal the
    batched search's pins, and a rerun resumes everything from the files."""
    got = pd.scan_density_batch(pd.LogAdapter(), LOG_PARAMS, 'triangle', CELL, ANSATZ, RELAX, QSCAN, -0.9,
                                [0.63, 0.51], checkpoint=str(tmp_path))
    assert list(got['status']) == [pd.STATUS_OK, pd.STATUS_NO_LOCAL_MINIMUM]
    assert got['q0star'][0] == pytest.approx(0.9638831589507376, abs=1e-8)
    assert got['fmin'][0] == pytest.approx(-0.5535949848941145, abs=1e-13)
    again = pd.scan_density_batch(pd.LogAdapter(), LOG_PARAMS, 'triangle', CELL, ANSATZ, RELAX, QSCAN, -0.9,
                                  [0.63, 0.51], checkpoint=str(tmp_path))
    assert np.array_equal(again['q0star'][:1], got['q0star'][:1]) and list(again['status']) == list(got['status'])
    assert np.array_equal(again['qscan']['f'], got['qscan']['f'])


# ---------------------------------------------------------------- frozen-q search
class _Frozen:
    def __init__(self, q):
        self.q = q

    def q_opt(self):
        return ToyAdapter.QSTAR + 0.5 * (self.q - ToyAdapter.QSTAR)

    def f(self, q):
        return 0.35 + (q - ToyAdapter.QSTAR) ** 2


class FrozenToy(ToyAdapter):
    """The toy with the box scale carried in its state (last element), and a frozen
    field whose q_opt halves the distance to QSTAR: the frozen-q iteration converges
    geometrically."""

    def build(self, params, structure, cell, ansatz, temp, meanDensity, q00, dt, state=None, nThreads=1):
        sim = super().build(params, structure, cell, ansatz, temp, meanDensity, q00, dt,
                            None if state is None else np.asarray(state)[:-1], nThreads)
        sim.q = q00
        return sim

    def get_state(self, sim):
        return np.append(sim.x, sim.q)

    def set_state(self, sim, state):
        sim.x[...] = np.asarray(state)[:-1]

    def frozen_field(self, state, params, temp, cell):
        return _Frozen(float(np.asarray(state)[-1]))


def test_frozen_q_batch_converges_and_equals_one_density_solves():
    s = pd.FrozenQSettings()
    relax = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=0.99,
                             minimumA=1e-6)
    got = pd.solve_frozen_q_batch(FrozenToy(), {}, 'blob', {}, {}, relax, s, 0.1, [0.5, 0.55, 0.9])
    assert [g['status'] for g in got] == [pd.STATUS_OK, pd.STATUS_OK, pd.STOP_NAN]
    for g in got[:2]:
        assert g['q'] == pytest.approx(ToyAdapter.QSTAR, abs=2e-8)
        assert abs(g['q'] - g['q_relaxed']) < s.qTol and g['stop'] == pd.STOP_CONVERGED
        assert g['iters'] > len(s.schedule) and g['A1'] == 0.3
    for g, rho in zip(got, [0.5, 0.55, 0.9]):
        one = pd.solve_frozen_q_batch(FrozenToy(), {}, 'blob', {}, {}, relax, s, 0.1, [rho])[0]
        keys = set(g) - {'wall_s'}
        assert {k: g[k] for k in keys} == {k: one[k] for k in keys}
    with pytest.raises(ValueError, match='frozen_field'):
        pd.solve_frozen_q_batch(ToyAdapter(), {}, 'blob', {}, {}, relax, s, 0.1, [0.5])


def test_frozen_q_stage_settings():
    relax = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=0.99,
                             minimumA=1e-6)
    s = pd.FrozenQSettings()
    r0, r3 = pd._stage_relax(relax, s, 0), pd._stage_relax(relax, s, 3)
    assert (r0.fTol, r0.ATol) == (1e-6, 1.0) and (r3.fTol, r3.ATol) == (1e-12, relax.ATol)


@pytest.mark.gpu
def test_log_frozen_q_agrees_with_the_pinned_q0star():
    """The reference's agreement bounds between the frozen-q search and Find_q0Star
    (tests/test_phase_diagram_frozen_q.py:69-83: q within 1e-5, f within 1e-9, f_frozen
    within 1e-10 of f), here against the pinned Find_q0Star result at (-0.9, 0.63) with
    the q0* test's relaxation settings."""
    got = pd.solve_frozen_q_batch(pd.LogAdapter(), LOG_PARAMS, 'triangle', CELL, ANSATZ, RELAX,
                                  pd.FrozenQSettings(), -0.9, [0.63])[0]
    assert got['status'] == pd.STATUS_OK
    assert abs(got['q'] - 0.9638831589507376) < 1e-5
    assert abs(got['f'] - (-0.5535949848941145)) < 1e-9
    assert abs(got['f_frozen'] - got['f']) < 1e-10


def test_frozen_edge_helpers():
    grid = [0.1, 0.2, 0.3, 0.4, 0.5]
    res = {0.1: {'status': 'poor_fit'}, 0.2: {'status': 'ok', 'q': 0.97, 'f': -1.0},
           0.3: {'status': 'ok', 'q': 0.98, 'f': -1.1}, 0.4: {'status': 'poor_fit'}, 0.5: {'status': 'poor_fit'}}
    assert pd.edge_walks(grid, res) == [(1, -1), (2, 1)]
    calls = []

    def solve(p, q):
        calls.append((p, q))
        return {'status': 'ok' if p == 0.4 else 'poor_fit', 'q': q, 'f': -2.0}
    recs = pd.edge_walk(solve, grid, res, 2, 1, maxPast=3)
    assert calls == [(0.4, 0.98), (0.5, 0.98)]
    merged = pd.merge_edge(res, recs)
    assert merged[0.4]['status'] == 'ok' and merged[0.4]['edge_from'] == 0.3
    assert merged[0.5]['status'] == 'poor_fit'
    # two accepted edge records of one density: the lower f wins
    two = pd.merge_edge({0.4: {'status': 'poor_fit'}},
                        [{'status': 'ok', 'phi': 0.4, 'f': -1.0, 'pass_': 'edge'},
                         {'status': 'ok', 'phi': 0.4, 'f': -3.0, 'pass_': 'edge'}])
    assert two[0.4]['f'] == -3.0


def test_frozen_density_scan_batches_pass_one_and_walks_edges():
    s = pd.FrozenQSettings()
    relax = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=0.99,
                             minimumA=1e-6)
    recs = []
    final, pass1, edge = pd.scan_density_frozen(FrozenToy(), {}, 'blob', {}, {}, relax, s, 0.1,
                                                [0.5, 0.55, 0.9], record=recs.append)
    assert [pass1[p]['status'] for p in (0.5, 0.55, 0.9)] == [pd.STATUS_OK, pd.STATUS_OK, pd.STOP_NAN]
    assert [(r['phi'], r['q_start'], r['edge_from']) for r in edge] == [(0.9, pass1[0.55]['q'], 0.55)]
    assert final[0.9]['status'] == pd.STOP_NAN and final[0.5] is pass1[0.5]
    assert len(recs) == 4
    with pytest.raises(ValueError, match='increasing'):
        pd.scan_density_frozen(FrozenToy(), {}, 'blob', {}, {}, relax, s, 0.1, [0.5, 0.5])
    # densities with a pass-1 record are not solved again
    again = []
    pd.scan_density_frozen(FrozenToy(), {}, 'blob', {}, {}, relax, s, 0.1, [0.5, 0.55, 0.9], record=again.append,
                           done=pass1)
    assert [r['pass_'] for r in again] == ['edge']


def test_log_ansatz_equals_the_reference_build(golden):
    """The reference adapter's clean H2L triangle ansatz at mean 0.7 (the 'dfield_clean'
    field of tests/golden/frozen.npz, made by make_frozen_golden.py through
    logpfc_cpu/phase_diagram.py `build` + `get_state`) equals this adapter's host-built
    ansatz bit for bit."""
    d = golden("frozen")
    ad = pd.LogAdapter()
    got = ad.ansatz_field(ad.STRUCTURES['triangle'], dict(uNx=14, uNy=24, Mx=2, My=1),
                          dict(mode='H2L', A1=0.9, A2=0.0, A3=0.0), 0.7)
    assert got.shape == d["dfield_clean"].shape
    assert np.array_equal(got, d["dfield_clean"])


def test_scaled_fitness_identity():
    """The log adapter's rescaled fitness from the fitnesses against the rebuilt field and
    its mirror: equal to the direct mean of (d - s e)^2."""
    rng = np.random.default_rng(5)
    for _ in range(20):
        d = 0.1 * rng.standard_normal((24, 28))
        d -= d.mean()
        e = 0.1 * rng.standard_normal((24, 28))
        e -= e.mean()
        s = rng.uniform(0.3, 1.0)
        plus = 1 - float(np.mean((d - e) ** 2))
        minus = 1 - float(np.mean((d + e) ** 2))
        direct = 1 - float(np.mean((d - s * e) ** 2))
        assert pd.scaled_fitness(plus, minus, e, s) == pytest.approx(direct, abs=1e-14)


def test_adaptive_dt_batch_equals_one_point_runs():
    """With adaptive dt the members ask for different step counts; the batch steps the
    members that ask for the same count together and returns the one-point results."""
    relax = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=0.99,
                             minimumA=1e-6, dtMax=1.0)
    points = [(0.1, 0.5, 1.0), (0.1, 0.75, 1.0), (0.1, 0.9, 1.0), (0.1, 0.6, 1.0), (0.1, 0.5, 1.3),
              (0.2, 0.55, 0.98)]
    ad = ToyAdapter()
    got = pd.get_f_abc_batch(ad, {}, 'blob', {}, {}, relax, points)
    total = 0
    for g, p in zip(got, points):
        one = ToyAdapter()
        w = pd.get_f_abc(one, {}, 'blob', {}, {}, relax, *p)
        total += one.steps
        assert (g.values(), g.stop, g.steps, g.dt_max) == (w.values(), w.stop, w.steps, w.dt_max), p
    assert ad.steps == total
    assert {g.stop for g in got} == {pd.STOP_CONVERGED, pd.STOP_NAN, pd.STOP_POOR_FIT}
    assert max(g.dt_max for g in got) > 0.1


class _CountingLock(pd._LoopLockstep):
    """A lockstep group that records its life: steps only while open, closed once."""

    def __init__(self, ad, sims):
        super().__init__(ad, sims)
        self.closed = False
        ad.locks.append(self)

    def step(self, n):
        assert not self.closed
        assert all(not getattr(s, 'released', False) for s in self.sims)
        self.ad.group_steps += 1
        super().step(n)

    def close(self):
        assert not self.closed
        self.closed = True


class _LockingToy(ToyAdapter):
    def __init__(self):
        super().__init__()
        self.locks = []
        self.group_steps = 0

    def lockstep(self, sims):
        return _CountingLock(self, sims)

    def release(self, sim):
        sim.released = True


def test_adaptive_dt_batch_reuses_unchanged_groups():
    """The adaptive-dt scheduler keeps a lockstep group while its members are unchanged
    (whatever their step count), builds a new one when a member leaves or is rebuilt, steps
    no group holding a released plan and closes every group once."""
    relax = pd.RelaxSettings(dt=0.1, totalT=1e4, stepT=10.0, divs=10, maxDepth=4, requiredFitness=0.99,
                             minimumA=1e-6, dtMax=1.0)
    points = [(0.1, 0.5, 1.0), (0.1, 0.75, 1.0), (0.1, 0.9, 1.0), (0.1, 0.6, 1.0), (0.1, 0.5, 1.3),
              (0.2, 0.55, 0.98)]
    ad = _LockingToy()
    builds = pd.LOCKSTEP_BUILDS["groups"]
    got = pd.get_f_abc_batch(ad, {}, 'blob', {}, {}, relax, points)
    for g, p in zip(got, points):
        w = pd.get_f_abc(ToyAdapter(), {}, 'blob', {}, {}, relax, *p)
        assert (g.values(), g.stop, g.steps, g.dt_max) == (w.values(), w.stop, w.steps, w.dt_max), p
    assert all(lock.closed for lock in ad.locks)
    assert pd.LOCKSTEP_BUILDS["groups"] - builds == len(ad.locks)
    # (1526 group steps through 306 groups when written)
    assert len(ad.locks) * 3 < ad.group_steps


@pytest.mark.gpu
def test_log_adaptive_dt_batch_on_b200_plans():
    """Adaptive dt on B200 plans: the members ask for different step counts at different
    ping-pong parities, plans rebuilt by a rollback or a dt change join the lockstep
    mid-run, and plans of different dt share a batch launch. The batch returns each
    point's one-point result bit for bit, and no lockstep group ever had to fall back to
    stepping its plans one by one."""
    relax = pd.RelaxSettings(dt=0.1, totalT=2e4, stepT=1e2, divs=10, maxDepth=4, requiredFitness=0.99,
                             minimumA=1e-6, dtMax=0.4)
    ad = pd.LogAdapter()
    points = [(-0.9, 0.63, 0.9638831589013295), (-0.9, 0.63, 0.98), (-0.9, 0.88, 1.0)]
    fallbacks = pd.LOCKSTEP_FALLBACKS["parity"]
    got = pd.get_f_abc_batch(ad, LOG_PARAMS, 'triangle', CELL, ANSATZ, relax, points)
    got += pd.get_f_abc_batch(ad, LOG_PARAMS, 'honeycomb', CELL, ANSATZ, relax, [(-0.9, 1.2, 1.0)])
    assert pd.LOCKSTEP_FALLBACKS["parity"] == fallbacks
    for g, (structure, p) in zip(got, [('triangle', p) for p in points] + [('honeycomb', (-0.9, 1.2, 1.0))]):
        w = pd.get_f_abc(ad, LOG_PARAMS, structure, CELL, ANSATZ, relax, *p)
        assert (g.values(), g.stop, g.steps, g.dt_max) == (w.values(), w.stop, w.steps, w.dt_max), (structure, p)
    assert max(g.dt_max for g in got) > 0.1
