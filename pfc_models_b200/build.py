"""Build ``libpfc_b200.so`` in-tree for sm_100a (B200).

    python -m pfc_models_b200.build [--force] [--verbose] [--jobs N]

nvcc cross-compiles without a GPU. Each .cu file (the plan code and one file
per precision and kernel variant) compiles to an object under ``_build/`` in
parallel; the objects link into the library, written next to this file so that
it travels with the source tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libpfc_b200.so")
SOURCES = ["pfc_plan.cu", "pfc_generic_f32.cu", "pfc_generic_f64.cu",
           "pfc_fast_f32_e8.cu", "pfc_fast_f32_e16.cu", "pfc_fast_f32_e32.cu", "pfc_fast_f64_e8.cu",
           "pfc_fast_f64_e16.cu", "pfc_track.cu", "pfc_diag.cu", "pfc_onecta.cu", "pfc_pack_inst.cu", "pfc_extv.cu",
           "pfc_fastmix_f32.cu", "pfc_fastmix_f64.cu", "pfc_queue_f32.cu", "pfc_queue_f64.cu"]
HEADERS = ["pfc_fft.cuh", "pfc_kernels.cuh", "pfc_fast.cuh", "pfc_small.cuh", "pfc_registry.h",
           "pfc_fast_inst.cuh", "pfc_generic_inst.cuh", "pfc_pack.cuh", "pfc_pack_step.cuh", "pfc_fastmix_inst.cuh",
           "pfc_queue.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC"]


def nvcc_path() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else None


def _obj(src):
    return os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")


def _stale_objects(force):
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "pfc_b200.h")]
    newest_dep = max(_mtime(d) or 0 for d in deps)
    out = []
    for s in SOURCES:
        o = _mtime(_obj(s))
        if force or o is None or o < max(newest_dep, _mtime(os.path.join(CSRC, s)) or 0):
            out.append(s)
    return out


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    todo = _stale_objects(force)
    lib_t = _mtime(OUT)
    if not todo and lib_t is not None and lib_t >= max(_mtime(_obj(s)) for s in SOURCES):
        return OUT
    nvcc = nvcc_path()

    def compile_one(src):
        cmd = [nvcc, *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src),
               "-o", _obj(src) + ".tmp"]
        if verbose:
            cmd += ["-Xptxas", "-v"]
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        os.replace(_obj(src) + ".tmp", _obj(src))

    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(compile_one, todo))
    cmd = [nvcc, "-shared", *ARCH, "-o", OUT + ".tmp", *[_obj(s) for s in SOURCES]]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, jobs=a.jobs))
