"""Host side of the phase-diagram sweep: points, initial states, sharding across
ranks (gloo, world size 2) and the common-tangent consumer. No GPU."""
import json
import math
import os
import socket

import numpy as np
import pytest

from pfc_models_b200 import sweep, tangent
from tests.conftest import GOLDEN


def test_points_layout():
    pts = sweep.sweep_points()
    assert len(pts) == 512
    assert [p.index for p in pts] == list(range(512))
    assert pts[0].r == -0.6 and pts[-1].r == pytest.approx(-0.05) and pts[31].psi == 0.0
    assert all((p.start == "crystal") == (p.index % 2 == 0) for p in pts)
    assert {(p.n, p.mx, p.my) for p in pts} == set(sweep.BOXES)
    assert [p.n for p in pts] == [p.n for p in sweep.sweep_points()]   # seeded
    for p in pts[:6]:
        assert p.lx / p.n == pytest.approx(p.ly / p.n, rel=0.02)       # near-square cells


@pytest.mark.parametrize("k", [0, 1])
def test_initial_fields(k):
    p = sweep.sweep_points()[k]
    f = sweep.initial_field(p)
    assert f.shape == (p.n, p.n)
    assert f.mean() == pytest.approx(p.psi, abs=1e-3 if k else 1e-12)
    if p.start == "crystal":
        # whole periods: the profile continues smoothly across the boundary
        q = sweep.Q_ONE_MODE
        prof = lambda x, y: np.cos(q * x) * np.cos(q * y / math.sqrt(3)) - 0.5 * np.cos(2 * q * y / math.sqrt(3))
        assert prof(p.lx, 0.3) == pytest.approx(prof(0.0, 0.3), abs=1e-12)
        assert prof(0.2, p.ly) == pytest.approx(prof(0.2, 0.0), abs=1e-12)


def test_shard_is_a_partition():
    pts = sweep.sweep_points()
    parts = [sweep.shard(pts, r, 3) for r in range(3)]
    assert sorted(p.index for part in parts for p in part) == list(range(512))
    sizes = [sum(p.n * p.n for p in part) for part in parts]
    assert max(sizes) / min(sizes) < 1.3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pts = sweep.shard(sweep.sweep_points(), rank, world)
    res = [dict(index=p.index, r=p.r, F=float(p.index), mu=0.0, mean=p.psi) for p in pts]
    timing = {"steps": 10, "ms": 100.0 + rank, "sites": sum(p.n * p.n for p in pts), "launches": 60, "points": len(pts)}
    merged, t = sweep.gather_results(res, timing, world)
    if rank == 0:
        json.dump({"indices": sorted(d["index"] for d in merged), "timing": t}, open(out_path, "w"))
    dist.barrier()
    dist.destroy_process_group()


def test_gather_across_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    out = tmp_path / "g.json"
    mp.spawn(_gather_worker, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    d = json.load(open(out))
    assert d["indices"] == list(range(512))
    assert d["timing"]["ms"] == 101.0                     # the slowest rank
    assert d["timing"]["sites"] == sum(p.n * p.n for p in sweep.sweep_points())
    assert d["timing"]["ranks"] == 2 and d["timing"]["points"] == 512


def test_tangent_reproduces_the_reference_logpfc_coexistence():
    """eps = -0.9 logPFC: analytic liquid against the reference's triangle table."""
    g = json.load(open(os.path.join(GOLDEN, "tangent_logpfc_eps-0.9.json")))
    B, G, E = g["beta"], g["g"], g["eps"]
    f = lambda p: p * np.log(p) + 0.5 * (B + E) * p ** 2 + G / 3 * p ** 3 + 0.25 * p ** 4  # noqa: E731
    mu = lambda p: 1 + np.log(p) + (B + E) * p + G * p ** 2 + p ** 3  # noqa: E731
    d2 = lambda p: 1 / p + (B + E) + 2 * G * p + 3 * p ** 2  # noqa: E731
    liq = tangent.analytic_branch("liquid", f, mu, 0.05, 0.9, d2f=d2)
    tri = np.array(g["triangle"])
    t = tangent.common_tangent(liq, tangent.tabulated_branch("triangle", tri[:, 0], tri[:, 1]))
    assert t.phi_a == pytest.approx(g["phi_l_analytic"], abs=2e-12)
    assert t.phi_b == pytest.approx(g["phi_s_analytic"], abs=2e-12)
    assert t.phi_a == pytest.approx(g["fsolve"]["phi_l"], abs=1e-10)
    assert t.phi_b == pytest.approx(g["fsolve"]["phi_s"], abs=1e-10)
    assert t.mu == pytest.approx(g["mu"], abs=1e-6) and t.omega == pytest.approx(g["omega"], abs=1e-6)


def test_tangent_between_parabolas_is_exact():
    k1, c1, e1, k2, c2, e2 = 2.0, -0.5, 0.1, 5.0, 0.3, -0.05
    a = tangent.analytic_branch("a", lambda p: 0.5 * k1 * (p - c1) ** 2 + e1, lambda p: k1 * (p - c1), -2, 2,
                                d2f=lambda p: np.full(np.shape(p), k1))
    x = np.linspace(-1, 1.5, 60)
    b = tangent.tabulated_branch("b", x, 0.5 * k2 * (x - c2) ** 2 + e2, mu=k2 * (x - c2))
    t = tangent.common_tangent(a, b)
    # omega(mu) = -mu^2/(2k) - c mu + e on each side
    qa, qb = -1 / (2 * k1) + 1 / (2 * k2), -c1 + c2
    m = [(-qb + s * math.sqrt(qb * qb - 4 * qa * (e1 - e2))) / (2 * qa) for s in (1, -1)]
    m = [v for v in m if -2 * k1 < v < 2 * k1]
    mu = min(m, key=lambda v: -v * v / (2 * k1) - c1 * v + e1)
    assert t.mu == pytest.approx(mu, abs=1e-10)
    assert t.phi_a == pytest.approx(c1 + mu / k1, abs=1e-10) and t.phi_b == pytest.approx(c2 + mu / k2, abs=1e-10)


def _synthetic(r, psis, fsol, musol, start="crystal"):
    return [dict(index=i, r=r, psi=p, mean=p, F=float(fsol(p)), mu=float(musol(p)), F_prev=float(fsol(p)),
                 start=start) for i, p in enumerate(psis)]


def test_coexistence_feed_matches_direct_tangent():
    r = -0.4
    k, c, e = 3.0, -0.2, -0.03      # a convex "solid" branch below the liquid
    fs = lambda p: 0.5 * k * (p - c) ** 2 + e  # noqa: E731
    ms = lambda p: k * (p - c)  # noqa: E731
    res = _synthetic(r, np.linspace(-0.40, -0.05, 10), fs, ms)
    row = sweep.coexistence(res)[0]
    x = np.array([d["mean"] for d in res])
    t = tangent.common_tangent(tangent.std_liquid_branch(r, -1.0, 0.5),
                               tangent.tabulated_branch("s", x, fs(x), mu=ms(x), extend_lo=0.5 * (x[1] - x[0])))
    assert row["solid_points"] == 10
    assert row["psi_l"] == pytest.approx(t.phi_a, abs=1e-12) and row["psi_s"] == pytest.approx(t.phi_b, abs=1e-12)


def test_solid_run_stops_where_f_and_mu_disagree():
    fs = lambda p: 2.0 * p ** 2  # noqa: E731
    ms = lambda p: 4.0 * p  # noqa: E731
    pts = _synthetic(-0.3, np.linspace(-0.4, 0.0, 9), fs, ms)
    assert len(sweep.solid_run(pts)) == 9
    pts[5]["F"] += 0.01                      # one bad point is skipped
    assert [d["index"] for d in sweep.solid_run(pts)] == [0, 1, 2, 3, 4, 6, 7, 8]
    pts[6]["F"] += 0.01                      # two in a row end the run
    assert [d["index"] for d in sweep.solid_run(pts)] == [0, 1, 2, 3, 4]
