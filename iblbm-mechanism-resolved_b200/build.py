"""Build ``libiblbm_b200.so`` (the C-ABI library) in-tree with nvcc for sm_100a.

FP64 translation units that must reproduce the reference's arithmetic bit for
bit are compiled with ``-fmad=false`` (no multiply-add contraction); FP32
units use the default contraction.  Objects go to ``_build/``; the library is
written next to this file so it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libiblbm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
          "-I", CSRC, "-I", INCLUDE]
# unit -> extra flags
UNITS = {
    "dense_f64.cu": ["-fmad=false"],
    "ibm_f64.cu": ["-fmad=false"],
    "ops_f64.cu": ["-fmad=false"],
    "particles_f64.cu": ["-fmad=false"],
    "batch_f64.cu": ["-fmad=false"],
    "diag.cu": ["-fmad=false"],
    "dense_f32.cu": [],
    "pipe_f32.cu": [],
    "batch_f32.cu": [],
    "ibm_f32.cu": [],
    "mlp_f32.cu": [],
}


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA unit for sm_100a and link the shared library."""
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "iblbm_b200.h"))
    objs, cmds = [], []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src, *headers]):
            cmd = [nvcc, *ARCH, *COMMON, *flags, "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), file=sys.stderr)
            cmds.append(cmd)
    # the units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for _ in pool.map(subprocess.check_call, cmds):
            pass
    if force or _stale(LIB, objs):
        subprocess.check_call([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
