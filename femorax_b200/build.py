"""Builds the product library femorax_b200/libfemorax_b200.so in the source tree (sm_100a).

    python -m femorax_b200.build [--force]

Host C++ (compile step, C ABI) is compiled by g++ without fused multiply-adds; the CUDA kernels
by nvcc for sm_100a. The Gauss-point path (general.cu) is compiled with --fmad=false so that its
arithmetic is the reference host build's; the box, vector and solver kernels use fused
multiply-adds. Objects go to femorax_b200/_build/ (ignored by git); rebuilds are incremental.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfemorax_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                      "-I" + os.path.join(ROOT, "include")]
CXX_COMMON = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-I" + os.path.join(CUDA, "include"),
              "-I" + os.path.join(ROOT, "include")]

# (source, extra flags)
CUDA_SOURCES = [
    ("general.cu", ["--fmad=false"]),
    ("general_fast.cu", []),
    ("box.cu", []),
    ("box_f64_apply.cu", []),
    ("box_f64_force.cu", []),
    ("box_f32_apply.cu", []),
    ("box_f32_force.cu", []),
    ("box_f64_forcew.cu", []),
    ("box_f32_forcew.cu", []),
    ("vector.cu", []),
    ("solve.cu", []),
    ("stepping.cu", []),
    ("batch.cu", []),
    ("nbatch.cu", []),
    ("serve.cu", []),
    ("pimy.cu", ["--fmad=false"]),
    ("pdmy.cu", ["--fmad=false"]),
]
CXX_SOURCES = ["api.cpp", "compile.cpp"]


def _deps() -> float:
    """Newest modification time among the headers (a header change rebuilds everything)."""
    t = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".hpp", ".cuh")):
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _deps()
    jobs = []
    objs = []
    for src, extra in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            jobs.append([NVCC] + NVCC_COMMON + extra + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            jobs.append([GXX] + CXX_COMMON + ["-c", s, "-o", o])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for cmd, _ in zip(jobs, ex.map(_run, jobs)):
                if verbose:
                    print(" ".join(cmd))
    if jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-ldl", "-lrt", "-lpthread"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
