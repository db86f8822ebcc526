"""Generate tests/golden/diagnose.npz from the reference's phase-diagram `diagnose`.

Run in a container where the reference checkout exists (it is not needed, and not
present, where the tests run):

    NUMBA_CACHE_DIR=<scratch dir> PYTHONPYCACHEPREFIX=<scratch dir> \
        python tests/golden/make_diagnose_golden.py <reference checkout>

`diagnose(sim, structure, cell)` (src/pfc_models/models/stdpfc_cpu/phase_diagram.py:
178-215) needs from `sim` only `n`, `State.n`, `State.n_hat`, `fft_fwd` and `Geometry`;
a small stand-in object supplies them (`fft_fwd` = NumPy's rfft2, as the pyFFTW
stand-in in `pyfftw_standin/` computes it), so the reference's own fitness, amplitude
and maxima code runs unmodified. Each field is the reference's `_build3Mode` ansatz in
the reference's `_box` (q00 = 1), plus seeded noise and a Gaussian dip. A cell whose
3-mode indices fall outside the half spectrum records that the reference raised.
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, structure, cell, mean, (A1, A2, A3) before the structure's sign and scale
    ("tri_small", "triangle", dict(uNx=16, uNy=28, Mx=2, My=1), -0.30, (0.40, 0.08, 0.03)),
    ("hc", "honeycomb", dict(uNx=14, uNy=24, Mx=2, My=2), 0.25, (0.35, 0.05, 0.02)),
    ("stripe", "stripe", dict(uNx=12, uNy=10, Mx=3, My=1), -0.10, (0.50, 0.06, 0.01)),
    ("tri_box", "triangle", dict(uNx=16, uNy=28, Mx=4, My=2), -0.25, (0.45, 0.10, 0.04)),
    ("tri_too_coarse", "triangle", dict(uNx=2, uNy=8, Mx=2, My=1), -0.30, (0.40, 0.08, 0.03)),
]


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, "pyfftw_standin"))
    sys.path.insert(0, os.path.join(ref_root, "src"))
    from pfc_models.models.stdpfc_cpu import phase_diagram as pd

    out = {}
    names = []
    for k, (name, sname, cell, mean, amps) in enumerate(CASES):
        st = pd.STRUCTURES[sname]
        geom = pd._box(cell, 1.0)
        nx, ny = cell["uNx"] * cell["Mx"], cell["uNy"] * cell["My"]
        rng = np.random.default_rng(100 + k)
        try:
            n = pd._build3Mode(geom, st, cell, mean, *(st.amplitudeSign * st.amplitudeScale * a for a in amps))
        except IndexError:
            n = mean + 0.3 * np.cos(2 * np.pi * np.arange(nx) / nx)[None, :] * np.ones((ny, 1))
        n = n + 0.004 * rng.uniform(-1, 1, n.shape)
        X, Y = geom.X, geom.Y
        cx, cy = 0.37 * geom.Lx, 0.61 * geom.Ly
        n = n - 0.05 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * (2.0 * geom.dx) ** 2))
        n = np.ascontiguousarray(n, dtype=np.float64)
        sim = types.SimpleNamespace(
            n=n, State=types.SimpleNamespace(n=n, n_hat=np.zeros((ny, nx // 2 + 1), dtype=complex)),
            Geometry=geom, fft_fwd=lambda a, o: o.__setitem__(Ellipsis, np.fft.rfft2(a)))
        try:
            d = pd.diagnose(sim, sname, cell)
            res = [d.fitness, *d.amplitudes, d.details["maxima_per_cell"], 0.0]
        except IndexError:
            res = [np.nan] * 5 + [2.0]
        out["field_" + name] = n
        out["result_" + name] = np.array(res, dtype=np.float64)
        out["cell_" + name] = np.array([cell["uNx"], cell["uNy"], cell["Mx"], cell["My"]], dtype=np.int64)
        out["geom_" + name] = np.array([geom.Lx, geom.Ly])
        names.append((name, sname))
    out["names"] = np.array([n for n, _ in names])
    out["structures"] = np.array([s for _, s in names])
    np.savez_compressed(os.path.join(HERE, "diagnose.npz"), **out)
    for name, _ in names:
        print(name, out["result_" + name].tolist())


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
