"""The relaxation driver (pfc_models_b200.phase_diagram) on the oracle's CPU stepper: a
logPFC adapter whose simulations are oracle.pfc_oracle.OracleSim (the reference's CPU
step restated in NumPy) and whose diagnose is the oracle's restatement of the adapters'
fitness (diagnose_modes, divided by the mean as logpfc_cpu/phase_diagram.py:211-223
does). Driven by `get_f_abc`, it must reproduce the values the reference's own test pins
for MinimizeFreeEnergy.Get_f_ABC (tests/test_phase_diagram_q0star.py:44-58, 489-510):
the stop and the step count exactly, f within 1e-12 and fitness and amplitudes within
1e-12 (the oracle's FFT is NumPy's, the reference's pyFFTW's, so the converged values
differ by round-off only). This pins the driver's decisions on the real model without a
GPU; the B200 plans are held to the same pins in test_relax.py."""
import numpy as np
import pytest

from oracle import pfc_oracle as orc
from pfc_models_b200 import diagnostics, phase_diagram as pd

from test_relax import ANSATZ, CELL, LOG_PARAMS, PINNED, RELAX, _check_pinned


class _OSim:
    def __init__(self, sim, dt):
        self.o, self.dt = sim, dt

    @property
    def t(self):
        return self.o.t


class OracleLogAdapter(pd.LogAdapter):
    """LogAdapter with the oracle's CPU stepper in place of B200 plans; counts the
    fitness evaluations that took the reference's rescaled branch."""
    rescaled = 0

    def _simulation(self, params, temp, dt, mean, geometry):
        g = orc.build_geometry(geometry.Nx, geometry.Ny, geometry.Lx, geometry.Ly)
        p = orc.Params(Gamma=params['Gamma'], beta=params['beta'], q0=params['q0'], epsilon=temp, g=params['g'],
                       dt=dt)
        return _OSim(orc.OracleSim("log", p, g), dt)

    def build(self, params, structure, cell, ansatz, temp, meanDensity, q00, dt, state=None, nThreads=1):
        params = self.validate_params(params)
        structure = self._structure(structure)
        cell = self.validate_cell(cell)
        ansatz = self.validate_ansatz(ansatz)
        field = self.ansatz_field(structure, cell, ansatz, meanDensity) if state is None else state
        sim = self._simulation(params, temp, dt, meanDensity, self.box(cell, q00))
        sim.o.set_field(field)
        return sim

    def get_state(self, sim):
        return sim.o.n.copy()

    def set_state(self, sim, state):
        sim.o.set_field(state)

    def get_time(self, sim):
        return sim.o.t

    def set_time(self, sim, t):
        sim.o.t = t

    def get_dt(self, sim):
        return sim.dt

    def step(self, sim):
        sim.o.step()

    def step_many(self, sim, n):
        for _ in range(n):
            sim.o.step()

    def snapshot(self, sim, out=None):
        return sim.o.n.copy()

    def release(self, sim):
        pass

    def lockstep(self, sims):
        return pd._LoopLockstep(self, sims)

    def free_energy(self, sim):
        return sim.o.free_energy()

    def diagnose(self, sim, structure, cell):
        st, c = self._structure(structure), self.validate_cell(cell)
        rows, cols, sets = diagnostics.mode_table(st, c)
        mode_sets = [(rows[sets == s], cols[sets == s]) for s in range(3)]
        n = sim.o.n
        fitness, A, B, C, _ = orc.diagnose_modes(n, mode_sets, st.amplitudeSign, c['Mx'] * c['My'])
        mean = np.fft.rfft2(n)[0, 0].real / n.size
        amps = tuple(abs(a / mean) for a in (A, B, C))
        rebuilt = self.three_mode(st, c, mean, *(st.amplitudeSign * a * mean for a in amps))
        low = rebuilt.min()
        if low < 0:   # the reference rescales the rebuilt field towards the mean
            self.rescaled += 1
            # as the B200 adapter does it: from the fitness against the mirrored field
            mirrored = orc.diagnose_modes(n, mode_sets, -st.amplitudeSign, c['Mx'] * c['My'])[0]
            fitness = pd.scaled_fitness(fitness, mirrored, rebuilt - mean, mean / (mean - low))
            direct = 1 - float(np.abs(np.power(n - self._positive(rebuilt, mean), 2).mean()))
            assert abs(fitness - direct) < 1e-13
        return diagnostics.Diagnostics(fitness, amps, {})


@pytest.mark.parametrize('ref', [p for p in PINNED if p[0] != 'honeycomb'], ids=['triangle', 'stripe'])
def test_oracle_relaxation_reproduces_the_reference_pins(ref):
    structure, eps, phi, q00 = ref[:4]
    r = pd.get_f_abc(OracleLogAdapter(), LOG_PARAMS, structure, CELL, ANSATZ, RELAX, eps, phi, q00)
    _check_pinned(r, ref)


def test_oracle_relaxation_rolls_back_the_honeycomb_like_the_reference():
    """dt = 0.1 goes NaN in the honeycomb's first blocks; both are redone at dt 0.01 in ten
    sub-blocks (22000 steps), and f converges to the reference's value within 1e-12. On the
    way the rebuilt 3-mode field goes negative, so the log fitness's rescaled branch
    (logpfc_cpu/phase_diagram.py:196-199) is part of what the pins hold."""
    ref = next(p for p in PINNED if p[0] == 'honeycomb')
    ad = OracleLogAdapter()
    r = pd.get_f_abc(ad, LOG_PARAMS, 'honeycomb', CELL, ANSATZ, RELAX, *ref[1:4])
    _check_pinned(r, ref)
    assert ad.rescaled > 0      # some fitness checks on the way take the rescaled branch


def test_oracle_batch_driver_returns_the_pins():
    """The batched driver over the same adapter (its lockstep is a loop over the CPU
    simulations) returns the pinned triangle and stripe results."""
    for ref in (p for p in PINNED if p[0] != 'honeycomb'):
        got = pd.get_f_abc_batch(OracleLogAdapter(), LOG_PARAMS, ref[0], CELL, ANSATZ, RELAX,
                                 [ref[1:4], (ref[1], ref[2], ref[3] * 1.01)])
        _check_pinned(got[0], ref)
        assert got[1].stop == pd.STOP_CONVERGED


def test_oracle_find_q0star_reproduces_the_reference_pin():
    """Find_q0Star at (eps -0.9, phi 0.63) on the oracle's stepper through
    `find_q0star`: q0* within 1e-8 and fmin within 1e-13 of the reference test's values
    (tests/test_phase_diagram_q0star.py:53, 529-539), in the 392,000 steps the reference
    test records for it (:531-533). About 40 s of one CPU core."""
    from test_relax import QSCAN
    recs = []
    q, f = pd.find_q0star(OracleLogAdapter(), LOG_PARAMS, 'triangle', CELL, ANSATZ, RELAX, QSCAN, -0.9, 0.63,
                          record=recs.append)
    assert abs(q - 0.9638831589507376) < 1e-8
    assert abs(f - (-0.5535949848941145)) < 1e-13
    assert sum(r['steps'] for r in recs) == 392000


def test_oracle_density_scan_reproduces_the_status_points():
    """tests/test_phase_diagram_q0star.py:542-551: (-0.9, 0.51) and (-0.9, 0.52) end with
    no local minimum, the reference's message, in the 66,000 and 56,000 steps its comment
    records; here through `scan_density_batch` (one batched search) on the oracle's
    stepper. About 10 s of one CPU core."""
    from test_relax import QSCAN
    r = pd.scan_density_batch(OracleLogAdapter(), LOG_PARAMS, 'triangle', CELL, ANSATZ, RELAX, QSCAN, -0.9,
                              [0.51, 0.52])
    assert [str(x) for x in r['status']] == [pd.STATUS_NO_LOCAL_MINIMUM] * 2
    assert [str(x) for x in r['message']] == [pd.MSG_NO_LOCAL_MINIMUM] * 2
    assert np.isnan(r['q0star']).all() and np.isnan(r['fmin']).all()
    q = r['qscan']
    assert [int(q['steps'][q['phi_index'] == k].sum()) for k in range(2)] == [66000, 56000]


class OracleFrozenAdapter(OracleLogAdapter):
    """Also the frozen field of the oracle (frozen_moments, logpfc_cpu/phase_diagram.py:
    465-505); no defect screen."""
    defect_diagnostics = None

    def frozen_field(self, state, params, temp, cell):
        A, local = orc.frozen_moments(np.asarray(state), temp, params['g'], 1.0, cell)
        return diagnostics.FrozenField(A, local, params['beta'], params.get('q0', 1.0))


def test_oracle_frozen_q_agrees_with_find_q0star_under_adaptive_dt():
    """tests/test_phase_diagram_frozen_q.py:69-83 on the oracle's stepper: the 14 x 12
    cell (7 x 12, 2 x 1), an H2L ansatz and adaptive dt (0.01 up to 0.1); the frozen-q
    search and Find_q0Star agree within the reference test's bounds (q 1e-5, f 1e-9,
    f_frozen within 1e-10 of f). About 30 s of one CPU core."""
    small = {'uNx': 7, 'uNy': 12, 'Mx': 2, 'My': 1}
    h2l = {'mode': 'H2L', 'A1': 0.9, 'A2': 0.0, 'A3': 0.0}
    relax = pd.RelaxSettings(dt=0.01, dtMax=0.1, dtRate=1e-5, dtGrow=2.0, dtChecks=10, totalT=1e6, stepT=100.0,
                             divs=10, maxDepth=4, requiredFitness=0.99, minimumA=1e-6)
    qs = pd.QScanSettings(passes=3, Deltaq=0.02, q00_Steps=21, Deltaq_Refinement=0.05)
    params = {'beta': 0.5, 'g': -2.0, 'v0': 1.0}
    recs = []
    q_f, f_f = pd.find_q0star(OracleFrozenAdapter(), params, 'triangle', small, h2l, relax, qs, -0.9, 0.62,
                              record=recs.append)
    assert max(r['dt_max'] for r in recs) == pytest.approx(0.1)     # dt grew to dtMax
    r = pd.solve_frozen_q_batch(OracleFrozenAdapter(), params, 'triangle', small, h2l, relax, pd.FrozenQSettings(),
                                -0.9, [0.62])[0]
    assert r['status'] == pd.STATUS_OK
    assert abs(r['q'] - q_f) < 1e-5
    assert abs(r['f'] - f_f) < 1e-9
    assert abs(r['f_frozen'] - r['f']) < 1e-10


class OracleStdAdapter(OracleLogAdapter):
    """stdPFC on the oracle: the std ansatz (absolute amplitudes, no rescale), the std
    stepper and the adapters' absolute-amplitude fitness."""
    STRUCTURES = pd.StdAdapter.STRUCTURES
    ansatz_field = pd.StdAdapter.ansatz_field

    def _simulation(self, params, temp, dt, mean, geometry):
        g = orc.build_geometry(geometry.Nx, geometry.Ny, geometry.Lx, geometry.Ly)
        p = orc.Params(Gamma=params['Gamma'], beta=params['beta'], q0=params['q0'], epsilon=temp, g=params['g'],
                       dt=dt)
        return _OSim(orc.OracleSim("std", p, g), dt)

    def diagnose(self, sim, structure, cell):
        st, c = self._structure(structure), self.validate_cell(cell)
        rows, cols, sets = diagnostics.mode_table(st, c)
        mode_sets = [(rows[sets == s], cols[sets == s]) for s in range(3)]
        fitness, A, B, C, _ = orc.diagnose_modes(sim.o.n, mode_sets, st.amplitudeSign, c['Mx'] * c['My'])
        return diagnostics.Diagnostics(fitness, (A, B, C), {})


def test_oracle_std_relaxation_reproduces_the_recorded_mirror_values():
    """tests/test_phase_diagram_q0star.py:627-643: stdPFC at g = 0, eps -0.25, the triangle at
    nbar -0.25 and the honeycomb at +0.25. Without ansatz noise the reference recorded f
    0.020967377878349205, fitness 0.9999995344356641, A 0.1324548908767042 in 3000 steps
    (:633-634); here within 1e-13 / 1e-12 / 1e-12 and in 3000 steps. The two structures
    mirror each other to round-off (the reference's own FFT makes them bit-identical; the
    oracle's NumPy x**3 is not exactly odd), and f lies below the liquid's."""
    import dataclasses
    params = dict(beta=1.0, g=0.0)
    relax = dataclasses.replace(RELAX, noise=0.0)
    tri = pd.get_f_abc(OracleStdAdapter(), params, 'triangle', CELL, ANSATZ, relax, -0.25, -0.25, 1.0)
    hc = pd.get_f_abc(OracleStdAdapter(), params, 'honeycomb', CELL, ANSATZ, relax, -0.25, 0.25, 1.0)
    assert tri.stop == hc.stop == pd.STOP_CONVERGED and tri.steps == hc.steps == 3000
    assert abs(tri.f - 0.020967377878349205) < 1e-13
    assert abs(tri.fitness - 0.9999995344356641) < 1e-12 and abs(tri.amplitudes[0] - 0.1324548908767042) < 1e-12
    assert hc.values() == pytest.approx(tri.values(), abs=1e-14)
    liquid = (1.0 - 0.25) / 2 * 0.25 ** 2 + 0.25 ** 4 / 4
    assert tri.f < liquid


def test_oracle_adaptive_dt_batch_equals_one_point_runs():
    """Adaptive dt (0.01 up to 0.1) on the oracle's logPFC stepper, the 14 x 12 cell: three
    q00 points as one batch equal the one-point runs bit for bit."""
    small = {'uNx': 7, 'uNy': 12, 'Mx': 2, 'My': 1}
    h2l = {'mode': 'H2L', 'A1': 0.9, 'A2': 0.0, 'A3': 0.0}
    relax = pd.RelaxSettings(dt=0.01, dtMax=0.1, dtRate=1e-5, dtGrow=2.0, dtChecks=10, totalT=1e6, stepT=100.0,
                             divs=10, maxDepth=4, requiredFitness=0.99, minimumA=1e-6)
    params = {'beta': 0.5, 'g': -2.0, 'v0': 1.0}
    points = [(-0.9, 0.62, 0.94), (-0.9, 0.62, 0.96), (-0.9, 0.62, 1.0)]
    got = pd.get_f_abc_batch(OracleLogAdapter(), params, 'triangle', small, h2l, relax, points)
    for g, p in zip(got, points):
        w = pd.get_f_abc(OracleLogAdapter(), params, 'triangle', small, h2l, relax, *p)
        assert (g.values(), g.stop, g.steps, g.dt_max) == (w.values(), w.stop, w.steps, w.dt_max), p
    assert all(g.dt_max == pytest.approx(0.1) for g in got)
