"""Vacancy tracking (analysis/vacancy_tracker.py:15-77): the oracle's restatement and
the device kernel (pfc_locate_vacancies through trackers.VacancyTracker) against the
reference's own outputs (tests/golden/vacancy.npz, made by make_vacancy_golden.py).

Index and position work: the bar is bit-identical positions and the same exception
(ValueError / IndexError) wherever the reference raises.
"""
import ctypes
import math
import types

import numpy as np
import pytest

from oracle import pfc_oracle as orc
from pfc_models_b200 import _lib

RAISES = {1: ValueError, 2: IndexError}


def _cases(golden):
    d = golden("vacancy")
    names = [str(n) for n in d["field_names"]]
    out = []
    for fid, x0, y0, ex, ey, code in d["cases"]:
        name = names[int(fid)]
        dx, dy = d["geom_special"] if name == "special" else d["geom_crystal"]
        out.append((d["field_" + name], float(x0), float(y0), float(dx), float(dy), float(ex), float(ey), int(code)))
    return d, out


def test_fixture_covers_the_index_rules(golden):
    d, cases = _cases(golden)
    codes = [c[-1] for c in cases]
    assert codes.count(1) >= 3 and codes.count(2) >= 2 and codes.count(0) >= 20
    assert d["traj"].shape == (6, 3, 2)


def test_oracle_matches_reference_tracker(golden):
    d, cases = _cases(golden)
    for field, x0, y0, dx, dy, ex, ey, code in cases:
        if code:
            with pytest.raises(RAISES[code]):
                orc.locate_vacancy(field, x0, y0, dx, dy)
        else:
            assert orc.locate_vacancy(field, x0, y0, dx, dy) == (ex, ey)
    # AddVacancy on the first field, TrackVacancies on the two later ones
    dx, dy = (float(v) for v in d["geom_crystal"])
    for v, (px, py) in enumerate(d["add_px"]):
        pos = orc.locate_vacancy(d["field_crystal"], px * dx, py * dy, dx, dy)
        traj = [pos]
        for name in ("crystal_moved", "crystal_moved2"):
            pos = orc.locate_vacancy(d["field_" + name], pos[0], pos[1], dx, dy)
            traj.append(pos)
        assert np.array_equal(np.array(traj), d["traj"][v])


def test_entry_point_checks_arguments_without_touching_the_device(built_lib):
    lib = _lib.load()
    f = ctypes.c_void_p(0)
    assert lib.pfc_locate_vacancies(f, 8, 8, 0.5, 0.5, f, 0, f, f) == _lib.PFC_OK    # nothing to do
    assert lib.pfc_locate_vacancies(f, 8, 8, 0.0, 0.5, f, 1, f, f) == _lib.PFC_E_ARG
    assert lib.pfc_locate_vacancies(f, 8, 8, 0.5, float("nan"), f, 1, f, f) == _lib.PFC_E_ARG
    assert lib.pfc_locate_vacancies(f, 0, 8, 0.5, 0.5, f, 1, f, f) == _lib.PFC_E_ARG
    assert lib.pfc_locate_vacancies(f, 8, 8, 0.5, 0.5, f, -1, f, f) == _lib.PFC_E_ARG
    assert lib.pfc_locate_vacancies(f, 8, 8, 0.5, 0.5, f, 1, f, f) == _lib.PFC_E_ARG  # null pointers
    assert "null pointer" in _lib.last_error()


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_device_locate_matches_reference(golden):
    from pfc_models_b200.trackers import VacancyTracker
    d, cases = _cases(golden)
    for field, x0, y0, dx, dy, ex, ey, code in cases:
        tr = VacancyTracker(types.SimpleNamespace(dx=dx, dy=dy))
        if code:
            with pytest.raises(RAISES[code]):
                tr.LocateVacancy(field, x0, y0)
        else:
            assert tr.LocateVacancy(field, x0, y0) == (ex, ey)


@pytest.mark.gpu
def test_device_tracking_matches_reference_trajectories(golden):
    import torch
    from pfc_models_b200.trackers import VacancyTracker
    d = golden("vacancy")
    dx, dy = (float(v) for v in d["geom_crystal"])
    tr = VacancyTracker(types.SimpleNamespace(dx=dx, dy=dy))
    for px, py in d["add_px"]:
        tr.AddVacancy(d["field_crystal"], int(px), int(py))
    # a device tensor is used in place
    tr.TrackVacancies(torch.as_tensor(d["field_crystal_moved"], device="cuda"))
    tr.TrackVacancies(d["field_crystal_moved2"])
    assert np.array_equal(np.array(tr.vacancyTrajectories), d["traj"])
    assert tr.vacancyCoords == [tuple(t[-1]) for t in d["traj"].tolist()]


@pytest.mark.gpu
def test_device_tracker_matches_oracle_on_a_simulation_field():
    """The coarse-grained density of a stepped 256^2 crystal, located on the device from
    the simulation itself, against the oracle on the host copy of the same field, for
    starts all over the grid, the edges included."""
    from pfc_models_b200 import fields, stdpfc
    from pfc_models_b200.trackers import VacancyTracker
    dx = math.pi / 4
    geom = stdpfc.Build2DGeometry(256, 256, 256 * dx, 256 * dx)
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
    sim = stdpfc.BuildB200_Simulation(prm, geom, precision="fp64")
    sim.State.n[...] = fields.GeneratePolycrystalInitialConditions(geom, -0.3, 0.01, nSeeds=4, radius=30 * dx,
                                                                   noise_seed=0, seed=1)
    sim.TimeSteps(50)
    local = sim.Get_local_n()
    rng = np.random.default_rng(5)
    starts = [(float(x), float(y)) for x, y in rng.uniform(-1.5, 257.5, (200, 2)) * dx]
    starts += [(0.0, 5.0), (255 * dx, 5.0), (5.0, 255 * dx), (1 * dx, 1 * dx), (-1 * dx, 10.0)]
    tr = VacancyTracker(geom)
    n_ok = 0
    for x0, y0 in starts:
        try:
            want = orc.locate_vacancy(local, x0, y0, geom.dx, geom.dy)
        except (ValueError, IndexError) as e:
            with pytest.raises(type(e)):
                tr.LocateVacancy(sim, x0, y0)
            continue
        assert tr.LocateVacancy(sim, x0, y0) == want
        n_ok += 1
    assert n_ok > 150


@pytest.mark.gpu
def test_track_updates_the_vacancies_before_one_that_raises(golden):
    """The reference's loop moves the vacancies before the one that raises and leaves it
    and the later ones where they were; one launch for all keeps that behaviour."""
    from pfc_models_b200.trackers import VacancyTracker
    d = golden("vacancy")
    field = d["field_special"]
    tr = VacancyTracker(types.SimpleNamespace(dx=0.5, dy=0.25))
    tr.vacancyCoords = [(8 * 0.5, 8 * 0.25), (12 * 0.5, 31 * 0.25), (24.5 * 0.5, 20 * 0.25)]
    tr.vacancyTrajectories = [[c] for c in tr.vacancyCoords]
    before = list(tr.vacancyCoords)
    with pytest.raises(IndexError):
        tr.TrackVacancies(field)
    assert tr.vacancyCoords[0] == orc.locate_vacancy(field, before[0][0], before[0][1], 0.5, 0.25)
    assert tr.vacancyCoords[1:] == before[1:]
    assert [len(t) for t in tr.vacancyTrajectories] == [2, 1, 1]
