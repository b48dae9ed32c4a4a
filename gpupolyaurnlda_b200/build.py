"""Builds libGPUPolyaUrnLDA.so (sm_100a) and the C++ host driver in-tree.

The reference builds its library with nvcc from src/cu/*.cu into
target/cuda/libGPUPolyaUrnLDA.so (Makefile:1-53, build.rs:1-8); this script
produces the same library name next to this file, compiled for sm_100a only.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libGPUPolyaUrnLDA.so")
TRAIN_BIN = os.path.join(HERE, "gpulda_train")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false and -ffp-contract=off keep every double operation a separately
# rounded IEEE operation on both the device and the host.
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-Xptxas", "-v",
]
LIB_SOURCES = ["gpulda.cu", "kernels.cu", "zsweep.cu", "zsweep_map.cu", "batch.cu", "serve.cu", "zsweep_pairs.cu"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    out = []
    for d in (CSRC, os.path.join(CSRC, "host"), os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                out.append(os.path.join(d, f))
    return out


def build_library(force: bool = False, verbose: bool = False) -> str:
    deps = _deps()
    if force or _stale(LIB, deps):
        cmd = [NVCC] + NVCC_FLAGS + ["-shared", "-o", LIB] + [os.path.join(CSRC, s) for s in LIB_SOURCES]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed building libGPUPolyaUrnLDA.so")
        if verbose:
            sys.stderr.write(r.stderr)
        with open(os.path.join(HERE, "ptxas_info.txt"), "w") as f:
            f.write(r.stderr)
    if force or _stale(TRAIN_BIN, deps + [LIB]):
        cmd = ["g++", "-O2", "-std=c++17", "-o", TRAIN_BIN, os.path.join(CSRC, "host", "gpulda_train.cpp"),
               "-I", os.path.join(ROOT, "include"), "-L", HERE, "-lGPUPolyaUrnLDA", f"-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("g++ failed building gpulda_train")
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    print(LIB)
