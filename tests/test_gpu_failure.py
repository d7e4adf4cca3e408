"""GPU: the failure paths of the band kernel and the pipelined pass report a
status instead of hanging or faulting, and leave the device usable.

Nothing here faults, traps or hangs the GPU: every wait that is made to run
out is a bounded wait on a copy that was never issued (a test switch in the
argument block), with a limit of a few hundred polls, so no copy is in flight
when the kernel returns; the other failures are host-side inputs that the
kernel's own checks turn into a status (a fixed body moved by three nodes in
one step; an oscillation table shorter than the run)."""
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
                mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=100, use_convergence=False,
                check_interval=20)
    base.update(kw)
    return SimConfig(**base)


def _device_still_exact(torch):
    """A fresh run after the failure matches the oracle bit for bit."""
    from iblbm_b200 import run
    from oracle import harness as H
    cfg = _cfg(max_steps=40)
    res, ref = run(cfg, verbose=False), H.run(cfg)
    assert res["engine"].status() == 0
    for k in ("ro", "U", "fstar", "fib"):
        np.testing.assert_array_equal(getattr(res["state"], k), getattr(ref["state"], k), err_msg=k)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_band_copy_wait_runs_out_and_reports(torch, precision):
    """The fixed body's restore copy is not issued while the band kernel waits
    for it with a 256-poll limit: the step reports status 6; the next normal
    step reports 0, and the device still computes bit-exact results.  (The
    single-CTA step: the cluster form of the FP64 step restores nothing by bulk
    copy.)"""
    from iblbm_b200.engine import Engine
    e = Engine(_cfg(), precision=precision, cluster=0)
    e.advance(5, outputs_last=False)  # the band is built and cached; later steps restore it by a bulk copy
    torch.cuda.synchronize()
    assert e.status() == 0
    for a in e.ibm_args:
        a.wait_limit, a.test_skip_copy = 256, 1
    e._step_serial(False)
    e.fence()
    torch.cuda.synchronize()
    assert e.status() == 6
    for a in e.ibm_args:
        a.wait_limit, a.test_skip_copy = 0, 0
    e._step_serial(False)
    e.fence()
    torch.cuda.synchronize()
    assert e.status() == 0
    _device_still_exact(torch)


def test_pipeline_wait_runs_out_and_reports(torch):
    """The pipelined FP32 pass with a producer that issues no copy: every
    consumer wait runs out after 256 polls, the pass reports status 1 (the
    engine's status 101) and returns; the next normal pass runs clean."""
    from iblbm_b200.engine import Engine
    e = Engine(_cfg(NN=97), precision="f32")
    e.set_tile("pipe4x2")
    e.advance(3, outputs_last=False)
    torch.cuda.synchronize()
    assert e.status() == 0
    for per_parity in e.dense_full:
        for a in per_parity:
            a.wait_limit, a.test_skip_copy = 256, 1
    e._step_serial(False)
    e.fence()
    torch.cuda.synchronize()
    assert e.status() == 101
    e.d_pipe_status.zero_()
    e.set_tile("pipe4x2")  # fresh argument blocks: default limit, copies issued
    e._step_serial(False)
    e.fence()
    torch.cuda.synchronize()
    assert e.status() == 0
    _device_still_exact(torch)


def test_fixed_body_moved_past_the_exclusion_box_reports(torch):
    """Markers of a fixed body moved three nodes between steps: the band of
    the overlapped step no longer lies inside the box that the concurrent bulk
    pass left out, and the band kernel reports status 5."""
    from iblbm_b200.engine import Engine
    e = Engine(_cfg(), precision="f64")
    e.advance(6, outputs_last=False)
    torch.cuda.synchronize()
    assert e.status() == 0
    e.d_Lx.add_(3.0 * e.st.dx)
    e.rebuild_next = True
    e._step_overlapped(False)
    e.join()
    torch.cuda.synchronize()
    assert e.status() == 5


def test_oscillation_table_exhausted_reports(torch):
    """An oscillating body whose motion table covers its configured run
    (entry t is the displacement of step t): stepping past the table reports
    status 4 (the kernel reads no entry beyond it)."""
    from iblbm_b200.engine import Engine
    kw = dict(NN=97, xmax=1, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.125, lattice_u=0.02,
              inflow_u=0.0, bc_type="open_boundary", ibm_method="DFC", motion_type="oscillating", KC=5.0,
              nx_formula="simple", Re=20, collision_model="BGK", max_steps=10)
    e = Engine(_cfg(**kw), precision="f64")
    n = int(e.xt.numel())  # steps 1 .. n - 1 have an entry
    e.advance(n - 1, outputs_last=False)
    torch.cuda.synchronize()
    assert e.status() == 0
    e.advance(1, outputs_last=False)
    torch.cuda.synchronize()
    assert e.status() == 4
