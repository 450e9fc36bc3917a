"""Builds libpms_b200.so in-tree with nvcc for sm_100a (B200).

    python -m pmsim_b200.build          # or pmsim_b200.build.build()

The library is plain C ABI (include/pms.h); Python binds it with ctypes (pmsim_b200/_lib.py).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpms_b200.so")
SOURCES = ["pms_material.cu", "pms_plasticity.cu", "pms_elements.cu", "pms_solver.cu", "pms_dpcg.cu", "pms_shapes.cpp", "pms_pattern.cpp"]
HEADERS = ["pms_device.cuh", "pms_shapes.h", "pms_pattern.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def sources():
    return [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in sources() + HEADERS] + [os.path.join(ROOT, "include", "pms.h")]
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC,-fopenmp",
           "-ccbin", "/usr/bin/g++", "-o", LIB + ".tmp"]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in sources()]
    cmd += ["-lgomp"]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose or ptxas_info:
        print(res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
