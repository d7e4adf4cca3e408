"""Fixture for the Taylor-Green convergence study (tests/test_tg_convergence.py).

The reference ships the results of its spatial convergence study of the
decaying Taylor-Green vortex (data/taylor_green/{df,mdf,dfc}/convergence.npz:
the relative L2 velocity error after one convective time at D = 10, 20, 40, 80
lattice nodes per half-width, pure LBM and with each IB method).  This script
copies those tables, records the configurations that the reference's scenario
builder (scenarios/taylor_green.py:16-85, make_tg_config) makes for each
resolution, and runs the reference itself (iblbm.run, CPU path) at every
resolution of every column, measuring the error with the reference's
own iblbm.diagnostics.tg_analytical_velocity_field and compute_l2_error.

The IB columns of the stored tables were made with a Lagrangian marker spacing
of 0.5 dx (the configuration default, iblbm/config.py:99) rather than the 1.0
that make_tg_config now sets; the runs below use 0.5 for the IB columns.

Usage:  python tests/golden/make_golden_tg_convergence.py --reference /path/to/reference
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESOLUTIONS = (10, 20, 40, 80)
IB_SPACING = 0.5


def _error(st, cfg, diag):
    """Relative L2 error of the final velocity against the vortex at t = max_steps
    (coordinates centred on the lattice, half-width (NN - 1) / 2)."""
    L = 0.5 * (cfg.NN - 1)
    nu = cfg.lattice_u * (cfg.cylinder_D_ratio * (cfg.NN - 1)) / cfg.Re
    X, Y = np.meshgrid(np.arange(st.nx) - (st.nx - 1) / 2.0, np.arange(st.ny) - (st.ny - 1) / 2.0)
    ux, uy = diag.tg_analytical_velocity_field(X.ravel(), Y.ravel(), float(cfg.max_steps), cfg.tg_u0, L, nu)
    return diag.compute_l2_error(np.asarray(st.U), np.stack([ux, uy], axis=1))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IBLBM_REFERENCE"),
                    required="IBLBM_REFERENCE" not in os.environ,
                    help="reference checkout (or set IBLBM_REFERENCE)")
    args = ap.parse_args()
    os.environ["IBLBM_GPU"] = "0"
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/iblbm_numba_cache")
    sys.dont_write_bytecode = True
    sys.path.insert(0, args.reference)
    import iblbm.diagnostics as diag
    from iblbm import run
    from scenarios.taylor_green import make_tg_config

    out = {"resolutions": np.array(RESOLUTIONS), "ib_marker_spacing": np.array([IB_SPACING])}
    stored = {m: np.load(os.path.join(args.reference, "data", "taylor_green", m, "convergence.npz"))
              for m in ("df", "mdf", "dfc")}
    for m in ("df", "mdf", "dfc"):
        assert list(stored[m]["resolutions"]) == list(RESOLUTIONS)
    out["stored_lbm"] = stored["df"]["errors_lbm"]
    out["stored_DF"] = stored["df"]["errors_ibm"]
    out["stored_MDF"] = stored["mdf"]["errors"]
    out["stored_DFC"] = stored["dfc"]["errors"]
    out["stored_mdf_iterations"] = np.array([int(stored["mdf"]["mdf_iterations"])])

    configs = {}
    for D in RESOLUTIONS:
        cfg = make_tg_config(D, use_ibm=False)
        configs[str(D)] = {k: v for k, v in dataclasses.asdict(cfg).items()
                           if isinstance(v, (int, float, str, bool, type(None), tuple, list))}
    out["configs_json"] = np.frombuffer(json.dumps(configs).encode(), dtype=np.uint8)

    for col in ("lbm", "DF", "MDF", "DFC"):
        errs = []
        for D in RESOLUTIONS:
            if col == "lbm":
                cfg = make_tg_config(D, use_ibm=False)
            else:
                cfg = dataclasses.replace(make_tg_config(D, use_ibm=True, ibm_method=col),
                                          marker_spacing_factor=IB_SPACING)
            st = run(cfg, verbose=False)["state"]
            errs.append(_error(st, cfg, diag))
            print(col, D, repr(errs[-1]), flush=True)
        out[f"ref_run_{col}"] = np.array(errs)
    np.savez_compressed(os.path.join(HERE, "tg_convergence.npz"), **out)
    print("wrote", os.path.join(HERE, "tg_convergence.npz"))


if __name__ == "__main__":
    main()
