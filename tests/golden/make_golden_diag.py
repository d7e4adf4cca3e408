"""Fixtures for the diagnostics (tests/test_diagnostics.py), made by running the
reference's own functions: iblbm.diagnostics.compute_strouhal on seeded
synthetic Cl series (signed, and rectified |Cl| on both sides of the aliasing
threshold), and iblbm.diagnostics.compute_slip_error and
iblbm.diagnostics.ibm_quality.compute_leakage_flux on a seeded velocity field,
with the reference's post-processing statistics and internal-flow sums on the
same series and fields.

Usage:  python tests/golden/make_golden_diag.py --reference /path/to/reference
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IBLBM_REFERENCE"),
                    required="IBLBM_REFERENCE" not in os.environ,
                    help="reference checkout (or set IBLBM_REFERENCE)")
    args = ap.parse_args()
    os.environ["IBLBM_GPU"] = "0"
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/iblbm_numba_cache")
    sys.path.insert(0, args.reference)
    from iblbm.diagnostics import compute_slip_error, compute_strouhal
    from iblbm.diagnostics.ibm_quality import compute_leakage_flux
    from iblbm.diagnostics import core
    from iblbm.diagnostics import internal_flow as inf
    from iblbm.diagnostics import surface
    from iblbm.lbm import make_d2q9
    rng = np.random.default_rng(11)
    out = {}
    ci, D, u = 50, 20.0, 0.05
    n = 400
    steps = np.arange(1, n + 1) * ci
    series = {
        "signed": 0.3 * np.sin(2 * np.pi * 0.17 * u / D * steps) + 1e-3 * rng.standard_normal(n),
        "rect_low": np.abs(0.3 * np.sin(2 * np.pi * 0.15 * u / D * steps)) + 1e-4 * rng.random(n),
        "rect_high": np.abs(0.3 * np.sin(2 * np.pi * 0.2 * (u * 8) / D * steps)) + 1e-4 * rng.random(n),
    }
    for k, cl in series.items():
        out[f"st_{k}_cl"] = cl
        out[f"st_{k}"] = np.array([compute_strouhal(cl, steps, D, u * (8 if k == "rect_high" else 1), ci)])
    out["st_ci"] = np.array([ci])
    out["st_D"] = np.array([D])
    out["st_u"] = np.array([u])
    ny, nx, NN = 81, 161, 81
    dx = dy = 1.0 / (NN - 1)
    Eux = 0.05 + 0.01 * rng.standard_normal((ny, nx))
    Euy = 0.01 * rng.standard_normal((ny, nx))
    for delta in ("hat", "peskin4pt"):
        r = compute_slip_error(Eux, Euy, dx, dy, 0.5, 0.5, 0.25, NN, delta, u_ref=0.05)
        out[f"slip_{delta}_mean"] = np.array([r["mean"]])
        out[f"slip_{delta}_max"] = np.array([r["max"]])
        out[f"slip_{delta}_per_marker"] = r["per_marker"]
        q = compute_leakage_flux(Eux, Euy, dx, dy, 0.5, 0.5, 0.25, NN, delta, u_ref=0.05)
        out[f"leak_{delta}_total"] = np.array([q["total"], q["total_raw"]])
        out[f"leak_{delta}_per_marker"] = q["per_marker"]
    out["slip_Eux"], out["slip_Euy"] = Eux, Euy
    # post-processing statistics on the same series and fields
    for k in series:
        cl = out[f"st_{k}_cl"]
        out[f"tail_{k}"] = np.array([core.tail_start_index(len(cl)), core.tail_mean(cl),
                                     core.tail_peak_to_peak_amp(cl), core.tail_mean(cl, 0.5),
                                     core.compute_cl_amplitude(cl)])
    Eold = 0.05 + 0.01 * rng.standard_normal((ny, nx))
    out["conv_old"] = Eold
    out["conv"] = np.array([core.check_convergence(Eux, Euy, Eold, Euy * 0.5)])
    # a wake: reverse flow behind a body at (0.5, 0.5), D = 0.25, ending at x = 0.9
    xs = np.arange(nx) * dx
    wake = np.tile(np.where((xs > 0.62) & (xs < 0.9), -0.01 * np.sin(np.pi * (xs - 0.62) / 0.28), 0.02), (ny, 1))
    out["recirc_field"] = wake
    # flow inside a disc at (0.5, 0.5), D = 0.25, on the seeded field
    ro = 1.0 + 0.01 * rng.standard_normal((ny, nx))
    out["inside_ro"] = ro
    res = inf.compute_inside_residual(Eux, Euy, dx, dy, 0.5, 0.5, 0.25, kappa=2.0, u_ref=0.05)
    out["inside_residual"] = np.array([res["mean"], res["max"], res["n_points"], res["mean_normalized"],
                                       res["max_normalized"]])
    out["internal_momentum"] = np.array(inf.compute_internal_momentum(Eux, Euy, ro, dx, dy, 0.5, 0.5, 0.125))
    out["internal_angular_momentum"] = np.array([inf.compute_internal_angular_momentum(Eux, Euy, ro, dx, dy,
                                                                                        0.5, 0.5, 0.125)])
    # stress of a seeded D2Q9 state and the force it puts on a cylinder (the circle
    # near the lattice edge exercises the clamped cells)
    # (populations from their own seed, 12, so the test makes them again instead of loading them)
    rng12 = np.random.default_rng(12)
    fst = (1.0 / 9.0) + 0.01 * rng12.standard_normal((nx * ny, 9))
    feq_s = (1.0 / 9.0) + 0.01 * rng12.standard_normal((nx * ny, 9))
    sig = surface.compute_stress_tensor(fst, feq_s, ro.ravel(), 0.8, make_d2q9(), ny, nx)
    out["stress_sha"] = np.frombuffer(hashlib.sha256(np.ascontiguousarray(sig).tobytes()).digest(), dtype=np.uint8)
    out["stress_sample"] = sig.reshape(-1, 4)[::97]
    out["surface_force"] = np.stack([surface.integrate_surface_force(sig, 0.5, 0.5, 0.125, dx, dy, nx, ny),
                                     surface.integrate_surface_force(sig, 0.05, 0.5, 0.125, dx, dy, nx, ny, 100)])
    U = np.stack([Eux.ravel(), Euy.ravel()], axis=1)
    out["l_int_z"] = np.array([inf.compute_l_int_z(U, ro.ravel(), nx, ny, dx, 0.5, 0.5, 0.125),
                               inf.compute_l_int_z(U, ro.ravel(), nx, ny, dx, 0.02, 0.97, 0.125)])
    out["recirc"] = np.array([core.compute_recirculation_length(wake, dx, dy, 0.5, 0.5, 0.25),
                              core.compute_recirculation_length(np.abs(wake), dx, dy, 0.5, 0.5, 0.25)])
    np.savez_compressed(os.path.join(HERE, "diag.npz"), **out)
    print("wrote", os.path.join(HERE, "diag.npz"))


if __name__ == "__main__":
    main()
