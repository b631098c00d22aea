"""Build libkiddo_gpu.so in-tree: nvcc for sm_100a, g++ for the host builder.

Run ``python -m kiddo_b200.build`` (or call ``build()``).  Objects go to
``kiddo_b200/_build/``; the shared library lands next to this file so it
travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkiddo_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread"]

CU_SOURCES = ["kgpu_api.cu", "kgpu_scan.cu", "kgpu_noalloc.cu", "kgpu_forest.cu",
              "kgpu_periodic_fast.cu",
              "kgpu_build.cu",
              "kgpu_chamfer.cu",
              "kgpu_points.cu",
              "kernels_f32_warp.cu",
              "kernels_f32_thread.cu",
              "kernels_f32_donnelly.cu",
              "kernels_f64_donnelly.cu",
              "kernels_f32_radius.cu",
              "kernels_f64_warp.cu",
              "kernels_f64_thread.cu",
              "kernels_f64_radius.cu",
              "kernels_f32_rows.cu",
              "kernels_f64_rows.cu",
              ]
CXX_SOURCES = ["layout_build.cpp", "archive.cpp"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build(force: bool = False, verbose: bool = False, extra_nvcc=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "kiddo_gpu.h")]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([nvcc] + ARCH + NVCC_FLAGS + list(extra_nvcc) + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([os.environ.get("CXX", "g++")] + CXX_FLAGS + ["-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for out in ex.map(_run, jobs):
                if verbose and out:
                    sys.stderr.write(out)
    if force or jobs or _newer(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
