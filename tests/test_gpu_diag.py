"""GPU: diagnostics reduced on the device (iblbm_force_coeffs, iblbm_velocity_change).

Cd / Cl of an output step equal the reference's formula evaluated on the host
from the same fields (numpy sums: 1e-12 relative); the ring-buffered run (many
checks queued, one read) gives the same histories as checks read one at a
time; the convergence error equals the reference's on two output steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _cfg(**kw):
    from iblbm_b200.config import SimConfig
    base = dict(Re=40, NN=49, xmax=2, ymax=1, cylinder_center=(0.45, 0.5), cylinder_D_ratio=0.25, lattice_u=0.05,
                inflow_u=0.05, bc_type="dirichlet_neumann", delta_type="peskin4pt", ibm_method="MDF",
                collision_model="TRT", trt_magic_param=0.1875, mdf_iterations=20, mdf_min_iterations=5,
                mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                check_interval=20)
    base.update(kw)
    return SimConfig(**base)


def _host_cd_cl(eng):
    """iblbm/diagnostics/core.py:53-113 on the host from the engine's fields."""
    st = eng.read_state()
    cfg = eng.cfg
    u_ref = cfg.lattice_u if cfg.motion_type == "oscillating" else st.in_u
    if eng.method == "DFC":
        f = np.asarray(st.dfc_force_lagr).sum(axis=0)
    else:
        f = st.fib.sum(axis=0)
    denom = float(np.mean(st.ro)) * u_ref ** 2 * st.lattice_r
    return abs(float(f[0])) / denom, float(f[1]) / denom


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("method", ["DF", "MDF", "DFC"])
def test_force_coefficients_match_host_formula(torch, precision, method):
    from iblbm_b200.engine import Engine
    e = Engine(_cfg(ibm_method=method), precision=precision)
    e.advance(120, outputs_last=True)
    cd, cl = e.cd_cl()
    hcd, hcl = _host_cd_cl(e)
    assert cd == pytest.approx(hcd, rel=1e-12, abs=0)
    assert cl == pytest.approx(hcl, rel=1e-9, abs=1e-13 * abs(hcd))


def test_ring_buffered_run_equals_per_check_reads(torch):
    """run() with nothing to stop on queues its checks into the device ring
    (one read at the end); with a callback every check is read at once: both
    give the same Cd / Cl histories, bit for bit."""
    from iblbm_b200 import run
    cfg = _cfg(max_steps=400)
    a = run(cfg, verbose=False)
    b = run(cfg, verbose=False, callback=lambda **kw: None)
    assert len(a["Cd_history"]) == 400 // 20
    np.testing.assert_array_equal(a["Cd_history"], b["Cd_history"])
    np.testing.assert_array_equal(a["Cl_history"], b["Cl_history"])


def test_velocity_change_matches_reference_formula(torch):
    from iblbm_b200.engine import Engine
    e = Engine(_cfg(), precision="f64")
    e.advance(40, outputs_last=True)
    U0 = e.read_state().U.copy()
    first = e.velocity_change()
    assert float(first[2].item()) == 1.0  # first call: reference field of zeros
    e.advance(20, outputs_last=True)
    U1 = e.read_state().U.copy()
    got = e.velocity_change().cpu().numpy()
    num, den = float(np.sum((U1 - U0) ** 2)), float(np.sum(U0 ** 2))
    assert got[0] == pytest.approx(num, rel=1e-12)
    assert got[1] == pytest.approx(den, rel=1e-12)
    assert got[2] == pytest.approx(np.sqrt(num / den), rel=1e-12)


def test_convergence_stop_rule_on_device(torch):
    """The velocity-convergence stop rule (iblbm/runtime/loop.py:118-126),
    its error reduced on the device: the run stops at the first check whose
    error, evaluated on the host from the fields the callback receives, is
    below the threshold, and every reported error equals the host's."""
    from iblbm_b200 import run
    cfg = _cfg(max_steps=4000, use_convergence=True, convergence_start=100, convergence_threshold=2e-3,
               check_interval=50, NN=33)
    seen = []
    run_res = run(cfg, verbose=False, callback=lambda **kw: seen.append((kw["step"], kw["state"].U.copy())))
    prev, stop, errs = None, None, {}
    for step, U in seen:
        if step == cfg.convergence_start:
            prev = U
        elif step > cfg.convergence_start and prev is not None:
            err = float(np.sqrt(np.sum((U - prev) ** 2) / np.sum(prev ** 2)))
            errs[step] = err
            prev = U
            if err < cfg.convergence_threshold and stop is None:
                stop = step
    assert stop is not None and run_res["converged"]
    assert run_res["final_step"] == stop
