"""Generate tests/golden/vacancy.npz from the reference's own vacancy tracker.

Run in a container where the reference checkout exists (it is not needed, and not
present, where the tests run):

    PYTHONPYCACHEPREFIX=<scratch dir> python tests/golden/make_vacancy_golden.py <reference checkout>

`_VacancyTracker` (src/pfc_models/analysis/vacancy_tracker.py) is plain NumPy, so its
module is loaded by file path and run unmodified. The fields are seeded synthetic
local densities:

* `crystal`, `crystal_moved`, `crystal_moved2` (96 x 80, dx = 0.7, dy = 0.65): a
  one-mode triangular profile with six Gaussian dips (the vacancies) at non-integer
  positions, smoothed in Fourier space; the two later fields move every dip by less
  than a pixel. The tracker adds the six vacancies on `crystal` and tracks them over
  the two later fields (`traj`, 3 positions per vacancy).
* `special` (40 x 32, dx = 0.5, dy = 0.25, so that x0 / dx is exact): patches built for
  the rules the reference's arithmetic implies: a 3 x 3 plateau (np.argmin takes the
  first minimum in row-major order), a cross with a zero denominator (no sub-pixel
  shift), half-integer pixel positions (np.round rounds half to even), a neighbourhood
  cut by the last row or column, an index of -1 that wraps, and the starts for which
  the reference raises (an empty neighbourhood at row or column 0, a cross neighbour
  past the last row or column, a NaN position).

`cases` rows: field id, x0, y0, expected x, expected y, and what the reference did:
0 returned, 1 raised ValueError, 2 raised IndexError.
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ["crystal", "crystal_moved", "crystal_moved2", "special"]


def load_tracker(ref_root):
    path = os.path.join(ref_root, "src", "pfc_models", "analysis", "vacancy_tracker.py")
    spec = importlib.util.spec_from_file_location("ref_vacancy_tracker", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod._VacancyTracker


def crystal_field(nx, ny, dx, dy, dips, rng):
    x = np.arange(nx) * dx
    y = np.arange(ny) * dy
    X, Y = np.meshgrid(x, y)
    q = 2 * np.pi / (9 * dx)
    f = np.cos(q * X) * np.cos(q * Y / np.sqrt(3)) - 0.5 * np.cos(2 * q * Y / np.sqrt(3))
    for (cx, cy) in dips:
        f -= 3.0 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * (1.6 * dx) ** 2))
    f += 1e-3 * rng.uniform(-1, 1, f.shape)
    kx = 2 * np.pi * np.fft.rfftfreq(nx, dx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, dy)
    KX, KY = np.meshgrid(kx, ky)
    return np.fft.irfft2(np.fft.rfft2(f) * np.exp(-(KX ** 2 + KY ** 2) * (0.8 * dx) ** 2 / 2), s=f.shape)


def special_field():
    ny, nx = 32, 40
    f = np.full((ny, nx), 1.0)
    starts = []
    # 3 x 3 plateau around (py, px) = (8, 8): the first minimum is the window's corner
    f[7:10, 7:10] = -5.0
    f[6, 7:10] = -1.0
    starts.append((8, 8))
    # zero denominator along x: window row [m, m, m] at py = 16 moves to px - 1, whose
    # cross has left = mid = right
    f[16, 17:22] = -7.0
    f[15, 17:22] = 0.5
    f[17, 17:22] = 0.25
    starts.append((16, 20))
    # a sloped dip for half-integer starts (x0 / dx = 24.5 and 25.5)
    f[20, 22:30] = [0.3, 0.1, -0.4, -0.9, -1.2, -0.8, -0.2, 0.2]
    f[19, 22:30] = 0.2
    f[21, 22:30] = 0.6
    starts += [(20, 24.5), (20, 25.5)]
    # last row: minimum one row in (valid) and on the last row (cross below is past the end)
    f[ny - 2, 4] = -3.0
    starts.append((ny - 1, 4))
    f[ny - 1, 12] = -3.5
    starts.append((ny - 1, 12))
    # last column: minimum on the last column (cross right is past the end)
    f[10, nx - 1] = -2.5
    starts.append((10, nx - 1))
    # column 1 with the minimum on column 0: the cross left index -1 wraps
    f[24, 0] = -2.2
    f[24, nx - 1] = -0.5
    starts.append((24, 1))
    # row 0 and column 0 starts: the neighbourhood slice is empty
    starts += [(0, 20), (12, 0)]
    return f, starts


def main(ref_root):
    Tracker = load_tracker(ref_root)
    rng = np.random.default_rng(17)
    nx, ny, dx, dy = 96, 80, 0.7, 0.65
    dips = [(rng.uniform(6, nx - 6) * dx, rng.uniform(6, ny - 6) * dy) for _ in range(6)]
    fields = {"crystal": crystal_field(nx, ny, dx, dy, dips, rng)}
    moved = [(cx + rng.uniform(-0.4, 0.4) * dx, cy + rng.uniform(-0.4, 0.4) * dy) for cx, cy in dips]
    fields["crystal_moved"] = crystal_field(nx, ny, dx, dy, moved, rng)
    moved2 = [(cx + rng.uniform(-0.4, 0.4) * dx, cy + rng.uniform(-0.4, 0.4) * dy) for cx, cy in moved]
    fields["crystal_moved2"] = crystal_field(nx, ny, dx, dy, moved2, rng)
    special, starts = special_field()
    fields["special"] = special
    geoms = {"crystal": (dx, dy), "crystal_moved": (dx, dy), "crystal_moved2": (dx, dy), "special": (0.5, 0.25)}

    cases = []

    def locate(fid, x0, y0):
        name = FIELDS[fid]
        t = Tracker(types.SimpleNamespace(dx=geoms[name][0], dy=geoms[name][1]))
        try:
            x, y = t.LocateVacancy(fields[name], x0, y0)
            cases.append((fid, x0, y0, float(x), float(y), 0))
        except ValueError:
            cases.append((fid, x0, y0, np.nan, np.nan, 1))
        except IndexError:
            cases.append((fid, x0, y0, np.nan, np.nan, 2))

    # single locates: from the nearest pixel of each dip and from points around it
    for (cx, cy) in dips:
        for ox, oy in ((0, 0), (0.6, -0.3), (-1.2, 0.9)):
            locate(0, cx + ox * dx, cy + oy * dy)
    for (py, px) in starts:
        locate(3, px * 0.5, py * 0.25)
    locate(3, float("nan"), 2.0)

    # tracking: add on the first field at the dips' nearest pixels, then track twice
    t = Tracker(types.SimpleNamespace(dx=dx, dy=dy))
    add_px = [(int(round(cx / dx)), int(round(cy / dy))) for cx, cy in dips]
    for (px, py) in add_px:
        t.AddVacancy(fields["crystal"], px, py)
    t.TrackVacancies(fields["crystal_moved"])
    t.TrackVacancies(fields["crystal_moved2"])
    traj = np.array(t.vacancyTrajectories, dtype=np.float64)   # (vacancies, 3, 2)

    out = dict(cases=np.array(cases, dtype=np.float64), traj=traj, add_px=np.array(add_px, dtype=np.int64),
               geom_crystal=np.array([dx, dy]), geom_special=np.array([0.5, 0.25]),
               field_names=np.array(FIELDS))
    for k, v in fields.items():
        out["field_" + k] = v
    np.savez_compressed(os.path.join(HERE, "vacancy.npz"), **out)
    raised = int(sum(1 for c in cases if c[5]))
    print(f"{len(cases)} locate cases ({raised} raising), {traj.shape[0]} tracked vacancies")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
