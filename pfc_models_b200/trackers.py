"""Vacancy tracking on the device.

`VacancyTracker` has the interface of the reference's `_VacancyTracker`
(src/pfc_models/analysis/vacancy_tracker.py:15-77): `LocateVacancy(local_phi, x0, y0)`,
`AddVacancy(local_phi, nx, ny)`, `TrackVacancies(local_phi)` and the lists
`vacancyCoords` / `vacancyTrajectories`. Every vacancy is located in one launch of
`pfc_locate_vacancies` on a device copy of the local field, with the reference's FP64
arithmetic and NumPy's index rules, so positions are bit-identical to the reference's.

`local_phi` may be what the reference passes (a host array, e.g. `Get_local_n()`), a
CUDA float64 tensor of shape (Ny, Nx), or a `Simulation`, whose coarse-grained density
(the field `Get_local_n` / `Get_local_phi` return) is then computed on the device and
never copied to the host: per tracking call only the positions (16 bytes per vacancy)
cross PCIe.

Where the reference raises (a non-finite position, an empty 3 x 3 neighbourhood: ValueError;
a cross neighbour past the last row or column: IndexError), so does this class, after
updating the vacancies before the failing one, as the reference's loop does.

    python -m pfc_models_b200.trackers [--n 2048] [--vacancies 256]

times one tracking call on the device (the local field, the launch and the copy of the
positions to the host) against the copy of the local field to the host that the
reference makes for each call before its Python loop over the vacancies.
"""
from __future__ import annotations

import ctypes
import math

from . import _lib


class VacancyTracker:
    """analysis/vacancy_tracker.py:15-77, located on the device."""

    def __init__(self, geometry, device=None):
        import torch
        self.torch = torch
        self.Geometry = geometry
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.lib = _lib.load()
        self.vacancyCoords = []
        self.vacancyTrajectories = []

    # -- the local field on the device
    def _field(self, local_phi):
        t = self.torch
        plan = getattr(local_phi, "plan", None)
        if plan is not None and hasattr(plan, "get_field"):
            return plan.get_field(_lib.FIELD_LOCAL_N, 2 * math.pi)
        f = t.as_tensor(local_phi, dtype=t.float64, device=self.device)
        if f.dim() != 2:
            raise ValueError(f"local_phi must be 2-D (Ny, Nx), got shape {tuple(f.shape)}")
        return f.contiguous()

    def _locate(self, field, coords):
        """New positions of `coords` (list of (x, y)) and the index of the first vacancy
        the reference would raise on (None if none), with that error."""
        t = self.torch
        n = len(coords)
        if n == 0:
            return [], None, None
        xy = t.tensor([c for p in coords for c in p], dtype=t.float64).to(self.device)
        status = t.empty(n, dtype=t.int32, device=self.device)
        ny, nx = field.shape
        stream = ctypes.c_void_p(t.cuda.current_stream(self.device).cuda_stream)
        _lib.check(self.lib.pfc_locate_vacancies(ctypes.c_void_p(field.data_ptr()), int(nx), int(ny),
                                                 float(self.Geometry.dx), float(self.Geometry.dy),
                                                 ctypes.c_void_p(xy.data_ptr()), n,
                                                 ctypes.c_void_p(status.data_ptr()), stream))
        out = xy.cpu().view(n, 2).tolist()
        st = status.cpu().tolist()
        for i, s in enumerate(st):
            if s:
                x0, y0 = coords[i]
                err = (ValueError(f"vacancy {i} at ({x0}, {y0}): empty 3x3 neighbourhood or non-finite position")
                       if s == 1 else
                       IndexError(f"vacancy {i} at ({x0}, {y0}): a cross neighbour lies past the grid"))
                return [tuple(p) for p in out], i, err
        return [tuple(p) for p in out], None, None

    # -- the reference's interface
    def LocateVacancy(self, local_phi, x0, y0):
        """Sub-pixel position of the local-density minimum next to (x0, y0)."""
        pos, bad, err = self._locate(self._field(local_phi), [(float(x0), float(y0))])
        if bad is not None:
            raise err
        return pos[0]

    def AddVacancy(self, local_phi, nx, ny):
        x, y = self.LocateVacancy(local_phi, nx * self.Geometry.dx, ny * self.Geometry.dy)
        self.vacancyCoords.append((x, y))
        self.vacancyTrajectories.append([(x, y)])

    def TrackVacancies(self, local_phi):
        """Moves every vacancy to the minimum next to its last position (one launch)."""
        pos, bad, err = self._locate(self._field(local_phi), self.vacancyCoords)
        upto = len(pos) if bad is None else bad
        for i in range(upto):
            self.vacancyCoords[i] = pos[i]
            self.vacancyTrajectories[i].append(pos[i])
        if bad is not None:
            raise err


def main():
    import argparse
    import json

    import numpy as np
    import torch

    from . import fields, stdpfc
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--vacancies", type=int, default=256)
    ap.add_argument("--repeat", type=int, default=20)
    a = ap.parse_args()
    dx = math.pi / 4
    geom = stdpfc.Build2DGeometry(a.n, a.n, a.n * dx, a.n * dx)
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
    sim = stdpfc.BuildB200_Simulation(prm, geom, precision="fp32")
    sim.State.n[...] = fields.GeneratePolycrystalInitialConditions(geom, -0.3, 0.01, nSeeds=64, radius=12 * dx,
                                                                   noise_seed=0, seed=1)
    sim.TimeSteps(200)
    rng = np.random.default_rng(3)
    tracker = VacancyTracker(geom)
    px = rng.integers(2, a.n - 2, size=(a.vacancies, 2))
    for x, y in px:
        tracker.AddVacancy(sim, int(x), int(y))

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.repeat):
            fn()
        e1.record()
        e1.synchronize()
        return 1e3 * e0.elapsed_time(e1) / a.repeat

    # one tracking call from the same positions each time (repeated tracking on one
    # field would walk starts that are not minima off flat regions)
    coords = list(tracker.vacancyCoords)
    track_us = timed(lambda: tracker._locate(tracker._field(sim), coords))
    host_copy_us = timed(lambda: sim.Get_local_n())
    print(json.dumps({"n": a.n, "vacancies": a.vacancies, "device_track_us": track_us,
                      "reference_field_to_host_us": host_copy_us,
                      "field_bytes": a.n * a.n * 8}))


if __name__ == "__main__":
    main()
