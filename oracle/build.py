"""Builds the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

Plain x86-64 code (no -march=native: this build travels to other hosts),
-ffp-contract=off so every double operation is separately rounded, matching
the CUDA library's explicit round-to-nearest intrinsics.

build_oracle_native() builds a second copy with -march=native on the host
that runs it (oracle/_build/liboracle_native_<cpu>.so): the timed CPU baseline uses
it.  Its results are the same bit for bit: contraction stays off and no
flag reorders floating-point operations.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SRC = os.path.join(HERE, "oracle.cpp")
FLAGS = ["-O3", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-pthread"]


def build_oracle(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(SRC) > os.path.getmtime(LIB):
        _compile(FLAGS + ["-o", LIB, SRC])
    return LIB


def _cpu_signature() -> str:
    """Digest of the host CPU's model and instruction-set flags."""
    import hashlib
    try:
        with open("/proc/cpuinfo") as f:
            lines = [l for l in f if l.startswith(("model name", "flags"))][:2]
    except OSError:
        lines = []
    return hashlib.sha256("".join(lines).encode()).hexdigest()[:12]


def build_oracle_native(force: bool = False) -> str:
    """-march=native build for the host that runs it, named by that host's
    CPU signature, so a copy built on another host is never loaded here."""
    os.makedirs(OUT_DIR, exist_ok=True)
    lib = os.path.join(OUT_DIR, f"liboracle_native_{_cpu_signature()}.so")
    if force or not os.path.exists(lib) or os.path.getmtime(SRC) > os.path.getmtime(lib):
        _compile(FLAGS + ["-march=native", "-o", lib, SRC])
    return lib


def _compile(args: list[str]) -> None:
    r = subprocess.run(["g++"] + args, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("g++ failed building the oracle")


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
