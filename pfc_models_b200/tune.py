"""Autotuner of the power-of-two step kernels, with an on-disk cache.

    python -m pfc_models_b200.tune --sizes 256,2048 --precision fp32,fp64 [--model std] [--save]

For one grid, precision and model it times every built variant of the two step
kernels (complex values per thread of the row and the column kernel, rows per
CTA of the row kernel; in FP32 also the two-lane packed kernels of either pass, and
the packed row kernel's TMA-staged tile) with CUDA events on a seeded noisy-liquid
state, and keeps the fastest row and the fastest column variant. A second stage times that choice
with 1, 2 and 4 columns per CTA of the column kernel, with and without programmatic
dependent launch, over whole steps replayed from CUDA graphs, and keeps a change only
where it is at least 1 % faster (`--refine` runs this stage alone on the entries the
package or the cache already holds). Results are cached as JSON, keyed
by GPU name, grid, precision and model, in the file named by $PFC_TUNE_CACHE
(default ~/.cache/pfc_models_b200/tune.json). `Simulation(kernels="auto")` looks
a grid up there first, then in the table measured on B200 that ships with the
package (tuned_b200.json), and otherwise uses the precision's defaults.
"""
from __future__ import annotations

import argparse
import itertools
import json
import math
import os
import threading

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGED = os.path.join(HERE, "tuned_b200.json")
EE_CHOICES = {_lib.FP32_MIXED: (8, 16, 32), _lib.FP64_PLAIN: (8, 16)}
TILE_CHOICES = (1, 2, 4, 8, 16)
COL_CTA_CHOICES = (1, 2, 4)
VARIANT_KEYS = ("ee_row", "ee_col", "row_tile", "col_cta", "pdl", "packed", "tma", "generic")
PACKED_EE = (8, 16)                 # values per lane of the two-lane packed FP32 kernels
PACKED_TILES = (2, 4, 8, 16)
_lock = threading.Lock()
_memo: dict = {}


def cache_path() -> str:
    return os.environ.get("PFC_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "pfc_models_b200",
                                                           "tune.json")


def _key(device_name, nx, ny, precision, model, batched=False):
    prec = "fp32" if precision == _lib.FP32_MIXED else "fp64"
    mod = "log" if model == _lib.MODEL_LOG else "std"
    return f"{device_name}|{nx}x{ny}|{prec}|{mod}" + ("|batch" if batched else "")


def _load(path):
    with _lock:
        if path in _memo:
            return _memo[path]
        try:
            with open(path) as f:
                d = json.load(f)
        except (OSError, ValueError):
            d = {}
        _memo[path] = d
        return d


def _device_name():
    import torch
    return torch.cuda.get_device_name()


def lookup(nx, ny, precision, model, device_name=None, batched=False):
    """The cached variant {"ee_row", "ee_col", "row_tile", "col_cta", "pdl"} for this
    grid, or None.
    `batched`: prefer the variant measured for many plans stepped as one batch (the
    single-plan choice favours latency, a batch is throughput-bound)."""
    if device_name is None:
        try:
            device_name = _device_name()
        except Exception:
            return None
    keys = ([_key(device_name, nx, ny, precision, model, True)] if batched else []) + \
        [_key(device_name, nx, ny, precision, model)]
    for key in keys:
        for path in (cache_path(), PACKAGED):
            e = _load(path).get(key)
            if e:
                return {k: int(e.get(k) or 0) for k in VARIANT_KEYS}
    return None


def _store(path, key, entry):
    d = dict(_load(path))
    d[key] = entry
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
    with _lock:
        _memo[path] = d


def balanced_tiles(ny, sms=None):
    """Row-tile heights other than powers of two that spread ny rows evenly over the SMs at
    two and four CTAs per SM (2048 rows: 7, 293 tiles, two per SM, where 8-row tiles leave 40
    of 148 SMs with one). The plan takes a height only where its CTA is whole multiples of
    it."""
    if sms is None:
        import torch
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    out = []
    for per_sm in (2, 4):
        t = -(-ny // (per_sm * sms))
        if 2 < t < 16 and t & (t - 1) and t not in out:
            out.append(t)
    return tuple(out)


def tune(nx, ny, precision="fp32", model="std", steps=20, warmup=3, save=True, path=None, batch=1):
    """Times the variants for one grid; returns the chosen entry (and caches it).
    With batch > 1 every variant steps `batch` plans together through a `Batch` and the
    fastest whole step wins (cached under the grid's batch key)."""
    if batch > 1:
        return _tune_batch(nx, ny, precision, model, steps, warmup, save, path, batch)
    import numpy as np
    import torch

    from . import fields, logpfc, stdpfc
    from .simulation import _PRECISIONS
    prec = _PRECISIONS[precision]
    mod = logpfc if model == "log" else stdpfc
    geom = mod.Build2DGeometry(nx, ny, nx * math.pi / 4, ny * math.pi / 4)
    if model == "log":
        prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.1)
        mean = 0.55
    else:
        prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
        mean = -0.3
    f0 = fields.GenerateNoisyLiquid(geom, mean, 0.01, seed=0)
    ees = EE_CHOICES[prec]
    # row candidates (packed?, values per thread or lane, tile, TMA) and column candidates
    # (packed?, values); each row candidate is timed beside the column candidates in turn
    row_c = [(False, e, t, 0) for e, t in itertools.product(ees, TILE_CHOICES + balanced_tiles(ny))]
    col_c = [(False, e) for e in ees]
    if prec == _lib.FP32_MIXED:
        row_c += [(True, e, t, m) for e, t, m in itertools.product(PACKED_EE, PACKED_TILES, (0, 1))]
        col_c += [(True, e) for e in PACKED_EE]
    rows, cols = {}, {}
    for i, (rp, ee_r, tile, tma) in enumerate(row_c):
        cp, ee_c = col_c[i % len(col_c)]
        packed = {(False, False): 0, (True, True): 1, (True, False): 2, (False, True): 3}[(rp, cp)]
        variant = {"ee_row": ee_r, "ee_col": ee_c, "row_tile": tile, "packed": packed, "tma": tma}
        try:
            sim = mod.BuildB200_Simulation(prm, geom, precision=precision, kernels=variant)
        except _lib.PfcError:
            continue     # a candidate this grid cannot take
        v = sim.plan.variant()
        if not v["fast"]:
            sim.plan.close()
            continue
        field = sim.State.phi if model == "log" else sim.State.n
        field[...] = f0
        sim.plan.step_timed(warmup)
        ms_r, ms_c = sim.plan.step_timed(steps)
        torch.cuda.synchronize()
        ok = np.isfinite(sim.CalculateFreeEnergy())
        sim.plan.close()
        if not ok:
            continue
        # a side with an odd factor holds a fixed number of values per thread (e.g. 28):
        # recorded as 0, the plan's own choice, which is what a request gets there
        er = v["ee_row"] if v["ee_row"] in (PACKED_EE if rp else ees) else 0
        ec = v["ee_col"] if v["ee_col"] in (PACKED_EE if cp else ees) else 0
        rk = (rp, er, v["row_tile"], tma)
        rows[rk] = min(rows.get(rk, math.inf), 1e3 * ms_r / steps)
        cols.setdefault((cp, ec), []).append(1e3 * ms_c / steps)
    if not rows or not cols:
        return None
    (rp, ee_r, tile, tma), row_us = min(rows.items(), key=lambda kv: kv[1])
    col_avg = {k: sum(v) / len(v) for k, v in cols.items()}
    (cp, ee_c), col_us = min(col_avg.items(), key=lambda kv: kv[1])
    packed = {(False, False): 0, (True, True): 1, (True, False): 2, (False, True): 3}[(rp, cp)]
    tag = lambda pk: "p" if pk else "s"  # noqa: E731
    entry = {"ee_row": ee_r, "ee_col": ee_c, "row_tile": tile, "packed": packed, "tma": tma if rp else 0,
             "row_us": row_us, "col_us": col_us,
             "rows_us": {f"{tag(a)}{b}/{c}/{d}": u for (a, b, c, d), u in sorted(rows.items())},
             "cols_us": {f"{tag(a)}{b}": u for (a, b), u in sorted(col_avg.items())}}
    entry.update(refine(nx, ny, precision, model, entry))
    if save:
        _store(path or cache_path(), _key(_device_name(), nx, ny, prec,
                                          _lib.MODEL_LOG if model == "log" else _lib.MODEL_STD), entry)
    return entry


def _setup(nx, ny, precision, model):
    from . import fields, logpfc, stdpfc
    mod = logpfc if model == "log" else stdpfc
    geom = mod.Build2DGeometry(nx, ny, nx * math.pi / 4, ny * math.pi / 4)
    if model == "log":
        prm = logpfc.BuildLogPFCModelParameters(Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.1)
        mean = 0.55
    else:
        prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
        mean = -0.3
    return mod, geom, prm, fields.GenerateNoisyLiquid(geom, mean, 0.01, seed=0)


def _tune_batch(nx, ny, precision, model, steps, warmup, save, path, batch):
    import torch

    from .simulation import _PRECISIONS, Batch
    prec = _PRECISIONS[precision]
    mod, geom, prm, f0 = _setup(nx, ny, precision, model)
    ees = EE_CHOICES[prec]
    timed = {}
    for ee_r, tile, ee_c in itertools.product(ees, TILE_CHOICES, ees):
        variant = {"ee_row": ee_r, "ee_col": ee_c, "row_tile": tile}
        sims = []
        try:
            for _ in range(batch):
                sims.append(mod.BuildB200_Simulation(prm, geom, precision=precision, kernels=variant))
        except _lib.PfcError:
            for s in sims:
                s.plan.close()
            continue
        v = sims[0].plan.variant()
        key = (v["ee_row"] if v["ee_row"] in ees else 0, v["row_tile"], v["ee_col"] if v["ee_col"] in ees else 0)
        if not v["fast"] or key in timed:
            for s in sims:
                s.plan.close()
            continue
        for s in sims:
            (s.State.phi if model == "log" else s.State.n)[...] = f0
        b = Batch(sims)
        b.step(max(warmup, 16))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.step(steps)
        e1.record()
        e1.synchronize()
        timed[key] = 1e3 * e0.elapsed_time(e1) / steps
        b.close()
        for s in sims:
            s.plan.close()
    if not timed:
        return None
    (ee_r, tile, ee_c), us = min(timed.items(), key=lambda kv: kv[1])
    entry = {"ee_row": ee_r, "ee_col": ee_c, "row_tile": tile, "batch": batch, "step_us": us,
             "row_us": None, "col_us": None,
             "steps_us": {f"{a}/{b}/{c}": u for (a, b, c), u in sorted(timed.items())}}
    entry.update(refine(nx, ny, precision, model, entry, batch=batch))
    if save:
        _store(path or cache_path(), _key(_device_name(), nx, ny, prec,
                                          _lib.MODEL_LOG if model == "log" else _lib.MODEL_STD, True), entry)
    return entry


def _time_blocks(nx, ny, precision, model, variant, batch, steps=320, skip=None, fast=True):
    """(us per whole step, column-kernel threads per CTA) of `batch` plans (1: one plan)
    with this variant, replayed from 16-step graphs after a warm-up that records them.
    (None, None) if the variant cannot be built or (with `fast`) the fast kernels do not
    apply; (None, threads) without timing when skip(threads) is true (a launch equal to one
    timed already). `fast=False` times whatever kernels the variant selects."""
    import torch

    from .simulation import Batch
    mod, geom, prm, f0 = _setup(nx, ny, precision, model)
    sims = []
    try:
        for _ in range(batch):
            sims.append(mod.BuildB200_Simulation(prm, geom, precision=precision, kernels=variant))
    except _lib.PfcError:
        for s in sims:
            s.plan.close()
        return None, None
    b = None
    try:
        if fast and not sims[0].plan.variant()["fast"]:
            return None, None
        threads = sims[0].plan.info()["fast_col_threads"]
        if skip is not None and skip(threads):
            return None, threads
        for s in sims:
            (s.State.phi if model == "log" else s.State.n)[...] = f0
        b = Batch(sims) if batch > 1 else None
        stepper = b if b is not None else sims[0].plan
        stepper.step(32)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        stepper.step(steps)
        e1.record()
        e1.synchronize()
        return 1e3 * e0.elapsed_time(e1) / steps, threads
    finally:
        if b is not None:
            b.close()
        for s in sims:
            s.plan.close()


def refine(nx, ny, precision, model, base, batch=1, min_gain=0.01):
    """Second stage: columns per CTA of the column kernel and programmatic dependent
    launch for the row/column variant in `base`, timed over whole steps. Returns
    {"col_cta", "pdl", "refine_us"}; keeps the defaults (0, 0) unless a choice is at
    least `min_gain` faster than they are."""
    v0 = {k: int(base.get(k) or 0) for k in ("ee_row", "ee_col", "row_tile", "packed", "tma")}
    timed, seen = {}, set()
    # sides with an odd factor: the register-resident kernels hold a fixed number of values
    # per thread, and on small or skinny grids the run-time mixed-radix kernels can be faster
    generic_us = None
    if nx & (nx - 1) or ny & (ny - 1):
        generic_us, _ = _time_blocks(nx, ny, precision, model, {"generic": 1}, batch, fast=False)
    for cc in (0,) + COL_CTA_CHOICES:
        for pdl in (0, 1, 2):   # 2: the column kernel only
            us, threads = _time_blocks(nx, ny, precision, model, dict(v0, col_cta=cc, pdl=pdl), batch,
                                       skip=lambda th: (th, pdl) in seen)
            if threads is None:
                return {"col_cta": 0, "pdl": 0}
            if us is None:
                continue     # the same launch as a choice timed already
            seen.add((threads, pdl))
            timed[(cc, pdl)] = us
    best = min(timed.items(), key=lambda kv: kv[1])
    if best[1] > (1 - min_gain) * timed[(0, 0)]:
        best = ((0, 0), timed[(0, 0)])
    (cc, pdl), best_us = best
    out = {"col_cta": cc, "pdl": pdl, "refine_us": {f"{a}/{b}": u for (a, b), u in sorted(timed.items())}}
    if generic_us is not None:
        out["generic_us"] = generic_us
        out["generic"] = 1 if generic_us < (1 - min_gain) * best_us else 0
    return out


def refine_table(path_in, device_name, steps=320):
    """Runs the second stage on every entry of `path_in` for this GPU; returns the
    updated table."""
    d = dict(_load(path_in))
    for key, e in sorted(d.items()):
        parts = key.split("|")
        if parts[0] != device_name:
            continue
        nx, ny = (int(v) for v in parts[1].split("x"))
        batch = int(e.get("batch") or 1) if len(parts) > 4 and parts[4] == "batch" else 1
        e = dict(e)
        e.update(refine(nx, ny, parts[2], parts[3], e, batch=batch))
        d[key] = e
        print(json.dumps({key: {k: e.get(k) for k in VARIANT_KEYS + ("refine_us",)}}), flush=True)
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="2048", help="comma list of n (n x n grids) or nx x ny items like 512x256")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--model", default="std")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--save", action="store_true", help="write the user cache")
    ap.add_argument("--batch", type=int, default=1, help="time this many plans stepped as one batch")
    ap.add_argument("--out", default=None, help="also write all entries to this JSON file")
    ap.add_argument("--refine", default=None, metavar="TABLE",
                    help="run only the second stage on every entry of TABLE ('packaged' for the shipped "
                         "table) and write the result to --out")
    a = ap.parse_args()
    if a.refine:
        d = refine_table(PACKAGED if a.refine == "packaged" else a.refine, _device_name())
        if a.out:
            with open(a.out, "w") as f:
                json.dump(d, f, indent=1, sort_keys=True)
        return
    allres = {}
    for s in a.sizes.split(","):
        nx, ny = (int(v) for v in s.split("x")) if "x" in s else (int(s), int(s))
        for precision in a.precision.split(","):
            for model in a.model.split(","):
                e = tune(nx, ny, precision, model, steps=a.steps, save=a.save, batch=a.batch)
                key = _key(_device_name(), nx, ny, _lib.FP32_MIXED if precision == "fp32" else _lib.FP64_PLAIN,
                           _lib.MODEL_LOG if model == "log" else _lib.MODEL_STD, a.batch > 1)
                allres[key] = e
                print(json.dumps({key: e}), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(allres, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
