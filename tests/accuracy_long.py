"""The FP32 form against the FP64 form at the benchmark configurations' own
step counts, on the GPU.

The FP64 form reproduces the reference's arithmetic bit for bit (the parity
tests, and tests/test_gpu_long_windows.py over 2 000 - 10 000 steps at full
size), so it stands in for the reference over runs far too long for the CPU
oracle.  Each configuration runs through the public run() in both forms:

* configuration 2 (1601 x 641, Re 100, MDF + Peskin-4), TRT and CM-MRT,
  200 000 steps: Cd / Cl over the last 20 % of the run (mean, standard
  deviation, peak-to-peak amplitude), the Strouhal number (the reference's FFT
  estimate and the mean period between interpolated upward zero crossings of
  Cl), and the largest pointwise Cd difference;
* configuration 3 (1281 x 1281 oscillating cylinder, DFC, BGK), 10 periods
  (100 000 steps): the same force statistics;
* configuration 5 (two settling discs, coupled MDF, CM-MRT, Velocity-Verlet),
  300 000 steps or until a stop rule ends the run, density ratios 1.5 and
  1.01: positions (lattice units), velocities and particle Reynolds numbers
  over every recorded step both runs share.

The configuration 4 sweep (72 cases, 50 000 steps) is checked by bench.py
itself (`sweep.accuracy_vs_f64`).  Usage on a GPU host:

    python tests/accuracy_long.py --out accuracy_long.json [--only NAME]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _cases():
    import bench
    return {
        "C2_trt_200k": (bench.workload_config("TRT", max_steps=200_000), "fixed"),
        "C2_cmmrt_200k": (bench.workload_config("CM_MRT", max_steps=200_000), "fixed"),
        "C3_dfc_100k": (bench.config3(max_steps=100_000), "fixed"),
        "C5_rho1.5_300k": (bench.config5(max_steps=300_000, rho_ratio=1.5), "particles"),
        "C5_rho1.01_300k": (bench.config5(max_steps=300_000, rho_ratio=1.01), "particles"),
    }


def upward_crossing_period(cl, every):
    """Mean period (steps) between interpolated upward zero crossings of Cl
    minus its mean, over the series given."""
    x = np.asarray(cl, dtype=float)
    x = x - x.mean()
    t = []
    for i in range(len(x) - 1):
        if x[i] < 0.0 <= x[i + 1]:
            t.append((i + x[i] / (x[i] - x[i + 1])) * every)
    return float(np.mean(np.diff(t))) if len(t) >= 3 else float("nan")


def force_stats(r64, r32, cfg, tail=0.2):
    from iblbm_b200.diagnostics import compute_strouhal
    cd64, cd32 = np.asarray(r64["Cd_history"]), np.asarray(r32["Cd_history"])
    cl64, cl32 = np.asarray(r64["Cl_history"]), np.asarray(r32["Cl_history"])
    n = min(len(cd64), len(cd32))
    cd64, cd32, cl64, cl32 = cd64[:n], cd32[:n], cl64[:n], cl32[:n]
    ci = int(cfg.check_interval)
    bad = {}
    for name, cd, cl in (("f64", cd64, cl64), ("f32", cd32, cl32)):
        idx = np.nonzero(~(np.isfinite(cd) & np.isfinite(cl)))[0]
        bad[name] = int((idx[0] + 1) * ci) if len(idx) else None
    if bad["f64"] is not None or bad["f32"] is not None:
        # a run that diverges: compare the samples before either form does
        first = min(v for v in bad.values() if v is not None) // ci - 1
        out = {"samples": n, "every": ci, "first_nonfinite_check_step": bad,
               "cd_max_pointwise_rel_err_before": float(np.max(np.abs(cd32[:first] - cd64[:first])
                                                               / np.abs(cd64[:first]))) if first > 0 else None}
        return out
    k0 = int(n * (1.0 - tail))
    ref = abs(float(np.mean(cd64[k0:])))
    st = r64["state"]
    u_ref = cfg.lattice_u if cfg.motion_type == "oscillating" else st.in_u
    D = 2.0 * st.lattice_r
    out = {"samples": n, "every": ci,
           "cd_tail_mean_f64": float(np.mean(cd64[k0:])), "cl_tail_std_f64": float(np.std(cl64[k0:])),
           "cd_tail_mean_rel_err": abs(float(np.mean(cd32[k0:]) - np.mean(cd64[k0:]))) / ref,
           "cl_tail_mean_err_rel_cd": abs(float(np.mean(cl32[k0:]) - np.mean(cl64[k0:]))) / ref,
           "cl_tail_std_err_rel_cd": abs(float(np.std(cl32[k0:]) - np.std(cl64[k0:]))) / ref,
           "cl_tail_amplitude_rel_err": abs(float(np.ptp(cl32[k0:]) - np.ptp(cl64[k0:])))
                                        / max(float(np.ptp(cl64[k0:])), 1e-300),
           "cd_max_pointwise_rel_err": float(np.max(np.abs(cd32 - cd64))) / ref,
           "cd_last_rel_err": abs(float(cd32[-1] - cd64[-1])) / abs(float(cd64[-1]))}
    if cfg.motion_type is None:
        st64 = compute_strouhal(cl64, n * ci, D, u_ref, ci)
        st32 = compute_strouhal(cl32, n * ci, D, u_ref, ci)
        p64 = upward_crossing_period(cl64[n // 2:], ci)
        p32 = upward_crossing_period(cl32[n // 2:], ci)
        out.update({"strouhal_fft_f64": st64, "strouhal_fft_f32": st32,
                    "strouhal_fft_rel_err": abs(st32 - st64) / abs(st64),
                    "strouhal_period_f64": D / (u_ref * p64), "strouhal_period_f32": D / (u_ref * p32),
                    "strouhal_period_rel_err": abs(p32 - p64) / p64})
    return out


def particle_stats(r64, r32, cfg):
    h64, h32 = r64["sedimentation_history"], r32["sedimentation_history"]
    s64 = {rec["step"]: rec for rec in h64}
    common = [rec for rec in h32 if rec["step"] in s64]
    st = r64["state"]
    dx = st.dx
    D = 2.0 * st.lattice_r
    nu = (st.tau - 0.5) / 3.0
    dpos, dvel, dre, vmax = 0.0, 0.0, 0.0, 0.0
    for rec in common:
        for p32, p64 in zip(rec["particles"], s64[rec["step"]]["particles"]):
            dpos = max(dpos, abs(p32["x"] - p64["x"]) / dx, abs(p32["y"] - p64["y"]) / dx)
            dvel = max(dvel, abs(p32["vx"] - p64["vx"]), abs(p32["vy"] - p64["vy"]))
            v64, v32 = np.hypot(p64["vx"], p64["vy"]), np.hypot(p32["vx"], p32["vy"])
            vmax = max(vmax, v64)
            if v64 > 0:
                dre = max(dre, abs(v32 - v64) * D / nu)
    last64 = h64[-1]["particles"]
    re_last = [float(np.hypot(p["vx"], p["vy"]) * D / nu) for p in last64]
    return {"records_compared": len(common), "final_step_f64": r64["final_step"], "final_step_f32": r32["final_step"],
            "termination_f64": r64["termination_reason"], "termination_f32": r32["termination_reason"],
            "max_position_err_lattice": dpos, "max_velocity_err_rel_vmax": dvel / vmax if vmax else 0.0,
            "max_particle_re_err": dre, "particle_re_last_f64": re_last,
            "final_positions_f64_lattice": [[p["x"] / dx, p["y"] / dx] for p in last64]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    import torch
    from iblbm_b200 import run
    from iblbm_b200.engine import Engine
    res = {}
    for name, (cfg, kind) in _cases().items():
        if args.only not in (None, name):
            continue
        t0 = time.time()
        runs = {p: run(cfg, verbose=False, engine=Engine(cfg, precision=p)) for p in ("f64", "f32")}
        torch.cuda.synchronize()
        for r in runs.values():
            r.pop("engine", None)
        stats = force_stats(runs["f64"], runs["f32"], cfg) if kind == "fixed" else \
            particle_stats(runs["f64"], runs["f32"], cfg)
        stats["seconds"] = time.time() - t0
        stats["steps"] = int(cfg.max_steps)
        res[name] = stats
        print(name, json.dumps(stats), flush=True)
        del runs
        torch.cuda.empty_cache()
    with open(args.out, "w") as fh:
        json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
