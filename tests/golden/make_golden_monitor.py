"""Fixtures for the sedimentation output files (tests/test_monitor.py), made by
running the reference's own monitor callback (monitor/sedimentation.py
create_sedimentation_callback) over a seeded synthetic sequence of states.
Its plotting module needs matplotlib, which is not installed here, so a stub
module with no-op plot functions stands in for ``monitor.plots``; the JSON and
.npz outputs do not depend on it.

Usage:  python tests/golden/make_golden_monitor.py --reference /path/to/reference
"""
from __future__ import annotations

import argparse
import os
import shutil
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KINDS = ("multi", "single")
CALLS = 12
PLOT_EVERY = 5
SNAPSHOT_EVERY = 4


def config_kwargs(kind):
    """SimConfig arguments of each synthetic run (same names in both packages)."""
    base = dict(Re=20, NN=33, xmax=1, ymax=2, cylinder_D_ratio=0.125, ibm_method="MDF", delta_type="peskin4pt",
                collision_model="CM_MRT", max_steps=1200, check_interval=100, gravity=2e-5,
                settling_inertia_model="none")
    if kind == "multi":
        return dict(base, cylinder_center=(0.5, 1.6),
                    particles_config=[{"center": (0.5, 1.6), "rho_ratio": 1.5},
                                      {"center": (0.52, 1.4), "rho_ratio": 1.2}])
    return dict(base, cylinder_center=(0.3, 1.0), rho_ratio=1.5, gravity_direction="right",
                particles_config=[{"center": (0.3, 1.0), "rho_ratio": 1.5}])


def sequence(kind):
    """[(step, state, elapsed)] for CALLS callbacks: positions, velocities,
    forces, a small velocity field and MDF statistics from a seeded generator.
    The states carry both this package's attributes and the reference's."""
    rng = np.random.default_rng(17 if kind == "multi" else 23)
    ny, nx = 6, 8
    n_p = 2 if kind == "multi" else 1
    out = []
    pos = np.array([[0.5, 1.6], [0.52, 1.4]])[:n_p].copy()
    for k in range(1, CALLS + 1):
        vel = 1e-3 * rng.standard_normal((n_p, 2))
        pos = pos + vel * 10.0
        force = 1e-4 * rng.standard_normal((n_p, 2))
        parts = [types.SimpleNamespace(pos=pos[i].copy(), vel=vel[i].copy(), fib_force=force[i].copy(),
                                       rho_ratio=(1.5, 1.2)[i]) for i in range(n_p)]
        stats = {"iter_count": int(rng.integers(3, 21)), "last_residual": float(rng.random() * 1e-4),
                 "diverged": bool(k % 5 == 0), "converged": bool(k % 3 == 0)}
        if k == 7:
            stats["last_residual"] = float("inf")
        st = types.SimpleNamespace(
            particles=parts, particle_pos=pos[0].copy(), particle_vel=vel[0].copy(), particle_force=force[0].copy(),
            p_int=None, _mdf_iter_stats=stats, mdf_iter_stats=stats, ny=ny, nx=nx, dx=1.0 / 32, dy=1.0 / 32,
            tau=0.62, U=1e-2 * rng.standard_normal((ny * nx, 2)))
        out.append((100 * k, st, 3.25 * k + 0.375 * (k % 4)))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IBLBM_REFERENCE"),
                    required="IBLBM_REFERENCE" not in os.environ,
                    help="reference checkout (or set IBLBM_REFERENCE)")
    args = ap.parse_args()
    os.environ["IBLBM_GPU"] = "0"
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/iblbm_numba_cache")
    sys.path.insert(0, args.reference)
    stub = types.ModuleType("monitor.plots")
    for name in ("plot_sedimentation_particle", "plot_sedimentation_summary", "plot_sedimentation_trajectory",
                 "plot_sedimentation_velocity"):
        setattr(stub, name, lambda *a, **k: None)
    sys.modules["monitor.plots"] = stub
    from iblbm import SimConfig
    from monitor.sedimentation import create_sedimentation_callback
    for kind in KINDS:
        out = os.path.join(HERE, f"monitor_{kind}")
        if os.path.isdir(out):
            shutil.rmtree(out)
        cfg = SimConfig(**config_kwargs(kind))
        cb = create_sedimentation_callback(out, cfg, plot_every=PLOT_EVERY, snapshot_every=SNAPSHOT_EVERY)
        seq = sequence(kind)
        for step, st, elapsed in seq:
            cb(step=step, Cd=0.0, Cl=0.0, error=1.0, state=st, elapsed=elapsed, converged=False)
        cb.finalize(converged=False, final_state=seq[-1][1], final_step=seq[-1][0], termination_reason="max_steps")
        print(kind, sorted(os.listdir(out)))


if __name__ == "__main__":
    main()
