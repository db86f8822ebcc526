"""Generate tests/golden/frozen.npz from the reference's logPFC `frozen_field`.

Run in a container where the reference checkout exists (it is not needed, and not
present, where the tests run):

    NUMBA_CACHE_DIR=<scratch dir> PYTHONPYCACHEPREFIX=<scratch dir> \
        python tests/golden/make_frozen_golden.py <reference checkout>

For the three parameter sets of the reference's own test
(tests/test_phase_diagram_frozen_q.py:22-37: a 'triangle' H2L ansatz in the
{'uNx': 14, 'uNy': 24, 'Mx': 2, 'My': 1} cell at mean 0.7, q00 = 1, scaled by
1 + 0.05 N(0, 1) noise from default_rng(1)), records the field, the reference's
FrozenField moments A = (A0, A1, A2), its local term, q_opt and f(q) at five q, plus the
adapter's free energy of the same field in the box rescaled by each q (the reference
test's consistency check), and the reference's `defect_diagnostics` (peak spread, sub-q
ratio, peak count, flag) of those fields and of the clean ansatz with and without one
vacancy. The adapter runs the reference's logpfc_cpu simulation with the pyFFTW
stand-in of `pyfftw_standin/`.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CELL = {'uNx': 14, 'uNy': 24, 'Mx': 2, 'My': 1}
H2L = {'mode': 'H2L', 'A1': 0.9, 'A2': 0.0, 'A3': 0.0}
PARAMS = [(0.5, -2.0, -0.9), (0.25, 1.0, -3.0), (1.0, 0.0, -2.0)]
QS = (0.7, 0.93, 1.0, 1.08, 1.3)


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, "pyfftw_standin"))
    sys.path.insert(0, os.path.join(ref_root, "src"))
    from pfc_models.models.logpfc_cpu import phase_diagram as ad

    out = {"qs": np.array(QS), "params": np.array(PARAMS), "cell": np.array([14, 24, 2, 1])}
    for k, (beta, g, temp) in enumerate(PARAMS):
        params = {'beta': beta, 'g': g, 'v0': 1.0}
        rng = np.random.default_rng(1)
        sim = ad.build(params, 'triangle', CELL, H2L, temp, 0.7, 1.0, 0.01)
        phi = ad.get_state(sim) * (1 + 0.05 * rng.standard_normal(ad.get_state(sim).shape))
        ff = ad.frozen_field(phi, params, temp, CELL)
        f_adapter = []
        for q in QS:
            s = ad.build(params, 'triangle', CELL, H2L, temp, float(phi.mean()), q, 0.01, state=np.array(phi))
            f_adapter.append(float(ad.free_energy(s)))
        out[f"phi_{k}"] = np.ascontiguousarray(phi, dtype=np.float64)
        out[f"A_{k}"] = np.array(ff.A, dtype=np.float64)
        out[f"local_{k}"] = np.array([ff.local])
        out[f"qopt_{k}"] = np.array([ff.q_opt()])
        out[f"f_{k}"] = np.array([float(ff.f(q)) for q in QS])
        out[f"f_adapter_{k}"] = np.array(f_adapter)
        dd = ad.defect_diagnostics(phi, CELL)
        out[f"defect_{k}"] = np.array([dd["peak_spread"], dd["subq_ratio"], dd["n_peaks"], float(dd["defect_flag"])])
        print(k, ff.A.tolist(), ff.local, ff.q_opt(), dd)
    # defect screen on the clean ansatz and on the ansatz with one vacancy
    params = {'beta': 0.5, 'g': -2.0, 'v0': 1.0}
    sim = ad.build(params, 'triangle', CELL, H2L, -0.9, 0.7, 1.0, 0.01)
    clean = np.ascontiguousarray(ad.get_state(sim), dtype=np.float64)
    vac = clean.copy()
    ny, nx = vac.shape
    iy, ix = np.unravel_index(np.argmax(clean[ny // 4: 3 * ny // 4, nx // 4: 3 * nx // 4]), (ny // 2, nx // 2))
    iy, ix = iy + ny // 4, ix + nx // 4
    yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    vac = vac - 0.6 * (clean[iy, ix] - clean.mean()) * np.exp(-((yy - iy) ** 2 + (xx - ix) ** 2) / 4.0)
    for name, field in (("clean", clean), ("vacancy", vac)):
        dd = ad.defect_diagnostics(field, CELL)
        out[f"dfield_{name}"] = field
        out[f"dres_{name}"] = np.array([dd["peak_spread"], dd["subq_ratio"], dd["n_peaks"], float(dd["defect_flag"])])
        print(name, dd)
    np.savez_compressed(os.path.join(HERE, "frozen.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
