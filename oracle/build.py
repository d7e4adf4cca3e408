"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/iblbm_oracle.c`` into ``oracle/_build/liboracle.so`` with gcc.
``-ffp-contract=off`` keeps every multiply and add separately rounded, matching
the reference's numba/numpy arithmetic; OpenMP only parallelises per-node loops,
so results do not depend on the thread count.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "iblbm_oracle.c")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")


def build_oracle(force: bool = False) -> str:
    """Compile the oracle shared library if it is missing or stale; return its path."""
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = [
        "gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp",
        "-ffp-contract=off", "-fno-fast-math", "-Wall",
        SRC, "-o", LIB, "-lm",
    ]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force=True))
