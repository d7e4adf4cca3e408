"""Digests of long FP64 runs of the CPU oracle at the benchmark configurations.

The oracle (``oracle/``) is pinned bit for bit to the reference's own outputs
(tests/test_oracle_golden.py).  Running it for thousands of steps at full
lattice size takes minutes to half an hour on the host, too long for a test,
so this script runs it once and records, per configuration, the SHA-256 of the
final rho / U / f* / fib / feq arrays, the Cd / Cl histories and the particle
states.  ``tests/test_gpu_long_windows.py`` runs the FP64 form on the GPU for
the same steps and compares bit for bit against these digests, without
running the oracle there.

Windows: configuration 2 (1601 x 641, MDF + Peskin-4, TRT and CM-MRT) for
2 000 steps, configuration 3 (1281 x 1281 oscillating DFC) for one period of
10 000 steps, configuration 5 (321 x 1281, two settling discs) for 5 000 steps.

Usage:  python tests/golden/make_golden_long.py [--only NAME] [--threads N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.make_golden import INIT_CASES, _sha  # noqa: E402

LONG_CASES = {
    "C2_trt_2000": dict(INIT_CASES["C2"], max_steps=2000, check_interval=500, use_convergence=False,
                        mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6),
    "C2_cmmrt_2000": dict(INIT_CASES["C2"], collision_model="CM_MRT", max_steps=2000, check_interval=500,
                          use_convergence=False, mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6),
    "C5_5000": dict(INIT_CASES["C5"], max_steps=5000, check_interval=500, use_convergence=False),
    "C3_10000": dict(INIT_CASES["C3"], max_steps=10000, check_interval=1000, use_convergence=False),
}


def _cfg(kw):
    from iblbm_b200.config import SimConfig
    kw = dict(kw)
    kw["cylinder_center"] = tuple(kw["cylinder_center"])
    if kw.get("particles_config"):
        kw["particles_config"] = [dict(p, center=tuple(p["center"])) for p in kw["particles_config"]]
    return SimConfig(**kw)


def make_long(name, kw, out_dir):
    from oracle import harness as H
    t0 = time.time()
    res = H.run(_cfg(kw))
    st = res["state"]
    d = {"config_json": np.frombuffer(json.dumps(kw).encode(), dtype=np.uint8)}
    for k in ("ro", "U", "fib", "fstar", "feq"):
        d[f"sha_{k}"] = np.frombuffer(bytes.fromhex(_sha(getattr(st, k))), dtype=np.uint8)
    d["Cd_history"] = np.asarray(res["Cd_history"], dtype=np.float64)
    d["Cl_history"] = np.asarray(res["Cl_history"], dtype=np.float64)
    d["final_step"] = np.array([res["final_step"]])
    if st.particles:
        d["particles"] = np.array([[*p.pos, *p.vel, *p.force] for p in st.particles])
    d["seconds"] = np.array([time.time() - t0])
    np.savez_compressed(os.path.join(out_dir, f"long_{name}.npz"), **d)
    return time.time() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    args = ap.parse_args()
    os.environ["OMP_NUM_THREADS"] = str(args.threads)
    from oracle.build import build_oracle
    build_oracle()
    for name, kw in LONG_CASES.items():
        if args.only not in (None, name):
            continue
        dt = make_long(name, kw, HERE)
        print(f"long_{name}.npz written ({dt:.0f} s)", flush=True)


if __name__ == "__main__":
    main()
