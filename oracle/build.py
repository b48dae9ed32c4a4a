"""Builds the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

Plain x86-64 code (no -march=native: the library travels to other hosts),
-ffp-contract=off so every double operation is separately rounded, matching
the CUDA library's explicit round-to-nearest intrinsics.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SRC = os.path.join(HERE, "oracle.cpp")


def build_oracle(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(SRC) > os.path.getmtime(LIB):
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
               "-pthread", "-o", LIB, SRC]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("g++ failed building the oracle")
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
