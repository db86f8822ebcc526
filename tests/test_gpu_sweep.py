"""The batched phase-diagram sweep on the GPU: 512 points, 5000 steps, FP32-mixed
against FP64 plain. Coexistence densities from the common tangent agree within
1e-4; the settled crystals the tangents rest on agree in F per site within 1e-6."""
import numpy as np
import pytest

from pfc_models_b200 import sweep

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def both():
    out = {}
    for precision in ("fp32", "fp64"):
        res, timing = sweep.run_sweep(5000, precision)
        out[precision] = (res, timing, sweep.coexistence(res))
    return out


def test_sweep_runs_every_point_in_one_batch(both):
    for precision, (res, timing, _) in both.items():
        assert len(res) == 512 and [d["index"] for d in res] == list(range(512))
        assert timing["classes"] == 3
        assert timing["launches"] == 2 * 3 * 5000
        assert all(np.isfinite(d["F"]) and np.isfinite(d["mu"]) for d in res)
        # mass is conserved by every simulation
        assert max(abs(d["mean"] - np.mean(sweep.initial_field(sweep.sweep_points()[d["index"]])))
                   for d in res) < 1e-12


def test_coexistence_fp32_mixed_matches_fp64(both):
    c32, c64 = both["fp32"][2], both["fp64"][2]
    found = [(a, b) for a, b in zip(c32, c64) if np.isfinite(a["psi_s"]) and np.isfinite(b["psi_s"])]
    assert len(found) >= 4
    for a, b in found:
        assert abs(a["psi_l"] - b["psi_l"]) < 1e-4 and abs(a["psi_s"] - b["psi_s"]) < 1e-4, (a, b)
        assert a["psi_l"] < a["psi_s"] < 0


def test_points_next_to_the_tangent_agree(both):
    """The settled crystals nearest each coexistence density (the ones the tangent
    rests on) have the same F and mu per site in both forms."""
    def runs(res):
        return {r: sweep.solid_run([d for d in res if d["r"] == r and d["start"] == "crystal"
                                    and sweep.is_crystal(d) and sweep.is_settled(d)])
                for r in sorted({d["r"] for d in res})}
    a, b = runs(both["fp32"][0]), runs(both["fp64"][0])
    n = 0
    for x, y in zip(both["fp32"][2], both["fp64"][2]):
        if not (np.isfinite(x["psi_s"]) and np.isfinite(y["psi_s"])):
            continue
        near = sorted(b[y["r"]], key=lambda p: abs(p["mean"] - y["psi_s"]))[:2]
        mine = {p["index"]: p for p in a[x["r"]]}
        for p in near:
            q = mine.get(p["index"])
            if q is not None:
                assert abs(q["F"] - p["F"]) < 1e-6 and abs(q["mu"] - p["mu"]) < 1e-5, p["index"]
                n += 1
    assert n >= 6
