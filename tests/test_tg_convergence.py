"""The reference's Taylor-Green spatial convergence study (D = 10, 20, 40, 80
nodes per half-width, one convective time, relative L2 velocity error; pure
LBM and with DF / MDF / DFC markers carrying the analytic velocity).

Fixture ``tests/golden/tg_convergence.npz`` (made by make_golden_tg_convergence.py):
the reference's stored tables (data/taylor_green/*/convergence.npz), the
configurations its scenario builder makes, and the errors of the reference
itself run at every resolution.  The current reference reproduces the stored
pure-LBM, DF and DFC columns to 1e-13 (with the IB columns' marker spacing of
0.5 dx) but not the stored MDF column (0.06-0.22 % apart: an MDF iteration other
than the present one made it), so MDF is pinned on the reference's own runs.
At D = 80 the IB band's lists exceed shared memory and the band step keeps them
in global memory.
"""
import json
import os

import numpy as np
import pytest

from iblbm_b200.diagnostics import tg_l2_error
from iblbm_b200.scenarios import make_tg_config

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "tg_convergence.npz"))
RES = [int(d) for d in G["resolutions"]]
COLS = ("lbm", "DF", "MDF", "DFC")


def _cfg(col, D):
    import dataclasses
    if col == "lbm":
        return make_tg_config(D, use_ibm=False)
    cfg = make_tg_config(D, use_ibm=True, ibm_method=col)
    return dataclasses.replace(cfg, marker_spacing_factor=float(G["ib_marker_spacing"][0]))


def _slope(errs):
    dx = 1.0 / np.asarray(RES, dtype=float)
    return np.polyfit(np.log(dx), np.log(errs), 1)[0]


def test_config_builder_matches_the_reference():
    """make_tg_config makes the reference's configuration at every resolution."""
    ref = json.loads(bytes(G["configs_json"]).decode())
    for D in RES:
        cfg = make_tg_config(D)
        for k, v in ref[str(D)].items():
            if hasattr(cfg, k):
                got = getattr(cfg, k)
                assert (list(got) if isinstance(got, tuple) else got) == v, (D, k)


def test_stored_table_is_the_reference_run_for_lbm_df_dfc():
    """The reference's stored tables against the reference run now."""
    for col, key in (("lbm", "stored_lbm"), ("DF", "stored_DF"), ("DFC", "stored_DFC")):
        np.testing.assert_allclose(G[f"ref_run_{col}"], G[key], rtol=1e-11, atol=0, err_msg=col)
    mdf = np.abs(G["ref_run_MDF"] / G["stored_MDF"] - 1)
    assert mdf.max() < 3e-3 and mdf.min() > 1e-5


@pytest.mark.parametrize("col", COLS)
def test_oracle_reproduces_the_reference_runs(col):
    """The oracle's error at D = 10, 20, 40 equals the reference's to 1e-12
    (D = 80 runs in the GPU test)."""
    from oracle import harness as H
    for D, want in zip(RES[:3], G[f"ref_run_{col}"][:3]):
        cfg = _cfg(col, D)
        s = H.run(cfg)["state"]
        got = tg_l2_error(s.U, cfg, s.nx, s.ny)
        assert abs(got / want - 1) < 1e-12, (col, D, got, want)


def test_convergence_orders():
    """Second-order convergence of every column (the reference's stored orders:
    1.92 pure LBM, 1.99 DF, 1.96 MDF, 2.16 DFC)."""
    for col in COLS:
        assert 1.85 < _slope(G[f"ref_run_{col}"]) < 2.25, col
    assert abs(_slope(G["stored_lbm"]) - 1.9202376588638084) < 1e-9


def _ana_norm(cfg, nx, ny):
    from iblbm_b200.diagnostics import tg_analytical_velocity_field
    from iblbm_b200.physics import tg_params
    L, nu = tg_params(cfg)
    X, Y = np.meshgrid(np.arange(nx) - (nx - 1) / 2.0, np.arange(ny) - (ny - 1) / 2.0)
    ux, uy = tg_analytical_velocity_field(X.ravel(), Y.ravel(), float(cfg.max_steps), cfg.tg_u0, L, nu)
    return np.sqrt(np.sum(ux ** 2 + uy ** 2))


@pytest.mark.gpu
@pytest.mark.parametrize("col", COLS)
def test_gpu_convergence_study(col):
    """Every resolution on the GPU.  FP64 form: the error equals the reference's
    run to 1e-12.  FP32 shifted form: its velocity field stays within 5e-5 of
    the FP64 field (L2, relative to the vortex's norm; measured 0.4e-6 to
    1.6e-5), so its error is the FP64 error to within that (the D = 80 errors
    are 3e-4 to 7e-4)."""
    import torch
    assert torch.cuda.is_available()
    from iblbm_b200 import run
    from iblbm_b200.engine import Engine
    for D, want in zip(RES, G[f"ref_run_{col}"]):
        cfg = _cfg(col, D)
        s64 = run(cfg, verbose=False, engine=Engine(cfg, precision="f64"))["state"]
        got = tg_l2_error(s64.U, cfg, s64.nx, s64.ny)
        assert abs(got / want - 1) < 1e-12, (col, D, got, want)
        s32 = run(cfg, verbose=False, engine=Engine(cfg, precision="f32"))["state"]
        dev = np.sqrt(np.sum((s32.U - s64.U) ** 2)) / _ana_norm(cfg, s64.nx, s64.ny)
        e32 = tg_l2_error(s32.U, cfg, s32.nx, s32.ny)
        print(f"{col} D={D} err64={got:.6e} err32={e32:.6e} fp32_dev={dev:.3e}")
        assert dev < 5e-5, (col, D, dev)
        assert abs(e32 - got) <= dev * (1 + 1e-9)
