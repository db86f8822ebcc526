#!/usr/bin/env python
"""PFC site-steps/s on B200: the fused ETD1 stepper on the 2048^2 stdPFC polycrystal.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (stdPFC polycrystal, 2048^2): dx = dy = pi/4, dt = 0.5, r = epsilon = -0.3,
Gamma = beta = q0 = 1, g = 0; mean psi = -0.3 plus 0.01 U[-1,1] noise (seed 0) and
64 seeds of radius 12 dx with the rotated one-mode profile (seed 1). Synthetic,
seeded; no dataset is involved.

One bench step = one ETD1 time step (row kernel + column kernel). `value` is the
FP32-mixed form with the state resident in HBM, each step timed with a pair of CUDA
events on the launching stream and L2 flushed (a 256 MiB write) between steps, so
every step starts from HBM. The per-kernel durations behind `roofline` come from a
second pass of the same number of steps with events around each launch. The FP64 plain form is timed the same way (`fp64_plain`).
`e2e` is the same metric through the public Python API (`State.n[...] = host`,
`TimeStep()` x 100, `CalculateFreeEnergy()`), the host field pinned, both copies
(the field in, F/mu/mean out) inside the timed region. Under torchrun with N > 1 every rank runs an
independent replica (a single simulation does not shard profitably over NVLink);
timings are the max over ranks.

`--impl reference` times the reference's CPU algorithm (the oracle port of
stdpfc_cpu, threaded pocketfft through scipy.fft with every host core) on the
same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "PFC site-steps/s (stdPFC 2048^2 polycrystal, FP32-mixed ETD1 step)"
UNIT = "site-steps/s"
NX = NY = 2048
DX = math.pi / 4
PARAMS = dict(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.3, g=0.0, dt=0.5)
E2E_STEPS = 100
FLUSH_BYTES = 256 << 20


def workload_config(extra=None):
    c = {"workload": "stdPFC polycrystal 2048x2048, dx=pi/4, dt=0.5, r=-0.3, 64 seeds r=12dx, FP32-mixed",
         "nx": NX, "ny": NY, "model": "stdPFC", "precision": "fp32_mixed",
         "l2": "flushed between steps (256 MiB write)"}
    if extra:
        c.update(extra)
    return c


def initial_field():
    from pfc_models_b200 import fields, spectral
    g = spectral.Build2DGeometry(NX, NY, NX * DX, NY * DX)
    return g, fields.GeneratePolycrystalInitialConditions(g, -0.3, 0.01, nSeeds=64, radius=12 * DX,
                                                          A=0.5, q=math.sqrt(3) / 2, noise_seed=0, seed=1)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples SM clock and clock-event reasons of one GPU during the timed region
    through NVML (read-only queries), polled every 2 ms from a thread."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.reasons = 0
        self.thread = None

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            uuid = None
            try:
                import torch
                uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            except Exception:
                pass
            h = None
            if uuid:
                try:
                    h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
                except Exception:
                    h = None
            if h is None:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.h, self.nv = h, pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            get_r = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        except Exception:
            self.h = None
            return
        self.stop_flag = False

        def loop():
            while not self.stop_flag:
                try:
                    self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                    self.reasons |= int(get_r(self.h))
                except Exception:
                    pass
                time.sleep(0.002)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return None
        self.stop_flag = True
        self.thread.join(timeout=2)
        if not self.samples:
            return None
        names = sorted(n for bit, n in self.REASONS.items() if self.reasons & bit)
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz, "reasons": names,
                "samples": len(self.samples), "source": "nvml"}


# ------------------------------------------------------------------ CPU baseline (oracle port)
def cpu_baseline(max_seconds=20.0, max_steps=20):
    """Reference CPU algorithm (oracle port of stdpfc_cpu) on this host, all cores."""
    from oracle import pfc_oracle as orc
    geom_h, f0 = initial_field()
    geom = orc.build_geometry(NX, NY, NX * DX, NY * DX)
    cores = os.cpu_count() or 1
    sim = orc.OracleSim("std", orc.Params(**PARAMS), geom, fft="scipy", workers=cores)
    sim.set_field(f0)
    sim.step()  # warm-up (plan caches)
    times = []
    t_start = time.perf_counter()
    while len(times) < max_steps and (time.perf_counter() - t_start) < max_seconds:
        t0 = time.perf_counter()
        sim.step()
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": NX * NY / med, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(times)} ETD1 steps of the same 2048^2 workload, median step "
                      f"{med * 1e3:.1f} ms (numpy/scipy pocketfft, {cores} threads)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import pfc_oracle as orc
    _, f0 = initial_field()
    geom = orc.build_geometry(NX, NY, NX * DX, NY * DX)
    cores = os.cpu_count() or 1
    sim = orc.OracleSim("std", orc.Params(**PARAMS), geom, fft="scipy", workers=cores)
    sim.set_field(f0)
    for _ in range(max(args.warmup, 1)):
        sim.step()
    budget_s = 150.0
    times = []
    t_all = time.perf_counter()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sim.step()
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget_s:
            break
    total = sum(times)
    value = NX * NY * len(times) / total
    sample = (f"{len(times)} of {args.steps} requested ETD1 steps at 2048^2 "
              f"(stopped at the {budget_s:.0f} s budget)" if len(times) < args.steps else
              f"{len(times)} ETD1 steps at 2048^2")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded polycrystal)",
            "config": workload_config({"precision": "fp64 (reference CPU algorithm)", "l2": "n/a (CPU)"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample + f", numpy/scipy pocketfft, {cores} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    distributed = world > 1
    if distributed:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    def barrier():
        if distributed:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not distributed:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from pfc_models_b200 import stdpfc

    geom, f0 = initial_field()
    flush_buf = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def flush():
        flush_buf.zero_()

    def build(precision):
        sim = stdpfc.BuildB200_Simulation(stdpfc.BuildStdPFCModelParameters(**PARAMS), geom, precision=precision)
        sim.State.n[...] = f0
        return sim

    def time_steps(sim, k, sampler=None):
        """The timed region: k steps, each bracketed by its own pair of CUDA events on the
        launching stream (nothing recorded between the two kernels of a step), L2 flushed
        between steps outside the events."""
        s = torch.cuda.current_stream(dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        launches0 = sim.plan.launches()
        barrier()
        if sampler:
            sampler.start()
        for a, b in evs:
            a.record(s)
            sim.plan.step(1)
            b.record(s)
            flush()
        barrier()
        clocks = sampler.stop() if sampler else None
        return [a.elapsed_time(b) for a, b in evs], sim.plan.launches() - launches0, clocks

    def time_kernels(sim, k):
        """Per-kernel durations for the roofline: k more steps with events around each of
        the two launches (an event between the kernels adds a few us, so this pass is kept
        apart from the timed region above), L2 flushed between steps."""
        ms_r, ms_c = [], []
        barrier()
        for _ in range(k):
            r, c = sim.plan.step_timed(1)
            ms_r.append(r)
            ms_c.append(c)
            flush()
        barrier()
        return ms_r, ms_c

    sites = NX * NY
    results = {}
    for precision in ("fp32", "fp64"):
        sim = build(precision)
        # warm-up through the timed path: records the one-step graph of each parity
        for _ in range(max(args.warmup, 3)):
            sim.plan.step(1)
            flush()
        sampler = ClockSampler(local) if precision == "fp32" else None
        ms_step, launches, clocks = time_steps(sim, args.steps, sampler)
        total_ms = max_over_ranks(sum(ms_step))
        ms_r, ms_c = time_kernels(sim, args.steps)
        results[precision] = dict(sim=sim, ms_r=ms_r, ms_c=ms_c, total_ms=total_ms, launches=launches,
                                  clocks=clocks, value=world * sites * args.steps / (total_ms / 1e3))
    # F agreement of the two forms after the same number of steps from the same field
    F32 = results["fp32"]["sim"].Reduce()
    F64 = results["fp64"]["sim"].Reduce()
    dF = abs(F32[0] / F64[0] - 1)
    mass_drift = abs(F32[2] - float(np.mean(f0)))

    # ---- end to end through the public API, host buffers pinned
    sim = results["fp32"]["sim"]
    host_in = torch.from_numpy(f0).pin_memory()
    e2e_frames = max(2, min(args.steps // 20, 10))
    sim.State.n[...] = host_in
    sim.TimeSteps(E2E_STEPS)
    sim.CalculateFreeEnergy()
    barrier()
    s = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(s)
    for _ in range(e2e_frames):
        sim.State.n[...] = host_in
        for _ in range(E2E_STEPS):
            sim.TimeStep()
        sim.CalculateFreeEnergy()
    ev1.record(s)
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1))
    e2e_value = world * sites * E2E_STEPS * e2e_frames / (e2e_ms / 1e3)

    # ---- roofline of the dominant kernel (column pass: reads V and n_hat, writes n_hat' and W)
    hbm, peak_kind = peaks()
    r32 = results["fp32"]
    col_ms = statistics.mean(r32["ms_c"])
    row_ms = statistics.mean(r32["ms_r"])
    elt = 8  # complex64
    spec = (NX // 2) * NY * elt
    col_bytes, row_bytes = 4 * spec, 2 * spec
    dominant = "column" if col_ms >= row_ms else "row"
    dom_bytes, dom_ms = (col_bytes, col_ms) if dominant == "column" else (row_bytes, row_ms)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    # the whole step from the timed region (whole-step events), the kernels from their pass
    step_achieved = (col_bytes + row_bytes) / ((r32["total_ms"] / args.steps) / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get(f"fp32_{dominant}")
        except Exception:
            traffic = None

    if rank == 0:
        ms_per_step = r32["total_ms"] / args.steps
        line = {
            "metric": METRIC, "value": r32["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 mean, ETD coefficients and reductions)",
            "data": "synthetic (seeded polycrystal)",
            "config": workload_config({"parallelism": "replicas" if world > 1 else "single GPU"}),
            "gpu_launches": r32["launches"],
            "fp64_plain": {"value": results["fp64"]["value"], "ms_per_step": results["fp64"]["total_ms"] / args.steps,
                           "fp32_over_fp64": r32["value"] / results["fp64"]["value"]},
            "accuracy": {"dF_over_F_fp32_vs_fp64": dF, "mass_drift_fp32": mass_drift,
                         "after_steps": max(args.warmup, 3) + 2 * args.steps},
            "roofline": {"bound": "hbm", "kernel": f"{dominant} pass (FP32)", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": dom_bytes,
                         "step": {"achieved": step_achieved, "frac": step_achieved / hbm,
                                  "bytes_per_site": (col_bytes + row_bytes) / sites,
                                  "row_ms": row_ms, "col_ms": col_ms,
                                  "kernel_timing": "separate pass of the same number of steps, CUDA events "
                                                   "around each launch"}},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": sites * 8,
                    "d2h_bytes_per_step": 24,
                    "note": f"one e2e step = State.n[...] = pinned host field (FP64), {E2E_STEPS} "
                            "TimeStep() calls, CalculateFreeEnergy() (F, mu, mean to the host)"},
            "clocks": r32["clocks"],
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line))
    for r in results.values():
        r["sim"].plan.close()
    if distributed:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
