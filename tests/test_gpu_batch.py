"""GPU: the batched multi-case path against the same cases run one at a time.

A batch runs every case's band step in one launch (one CTA per case) and the
collide-stream pass of all cases of a kind in one launch; each case's result
must equal that of its own single-case FP32 engine with the same tile shape
(the kernels share every device function)."""
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
                inflow_u=0.05, bc_type="dirichlet_neumann", delta_type="hat", ibm_method="DF",
                collision_model="BGK", trt_magic_param=0.1875, mdf_iterations=20, mdf_min_iterations=5,
                mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=200, use_convergence=False,
                check_interval=50)
    base.update(kw)
    return SimConfig(**base)


CASES = [
    dict(),
    dict(NN=65, ibm_method="MDF", delta_type="peskin4pt", collision_model="TRT"),
    dict(NN=41, Re=20, ibm_method="DFC", delta_type="peskin4pt", collision_model="CM_MRT"),
    dict(NN=81, ibm_method="MDF", delta_type="hat", collision_model="CM_MRT", cylinder_D_ratio=0.2),
    dict(NN=49, ibm_method="DF", delta_type="peskin4pt", collision_model="BGK", Re=60),
    dict(NN=97, xmax=1, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.125, lattice_u=0.02, inflow_u=0.0,
         bc_type="open_boundary", ibm_method="DFC", delta_type="peskin4pt", motion_type="oscillating", KC=5.0,
         nx_formula="simple", Re=20),
]


@pytest.mark.parametrize("tile,merged", [("rows2", False), ("node", False), ("rows2", True), ("rows4", True)])
def test_batch_matches_single_cases(torch, tile, merged):
    from iblbm_b200.batch import Batch
    from iblbm_b200.engine import Engine
    cfgs = [_cfg(**kw) for kw in CASES]
    b = Batch(cfgs, tile=tile)
    b.set_tile_all(tile, merged=merged)
    b.advance(61, outputs_last=True)
    torch.cuda.synchronize()
    assert b.status() == [0] * len(cfgs)
    for cfg, eb in zip(cfgs, b.engines):
        es = Engine(cfg, precision="f32")
        es.set_tile(tile)
        es.advance(61, outputs_last=True)
        torch.cuda.synchronize()
        assert es.status() == 0
        sb, ss = eb.read_state(), es.read_state()
        for k in ("ro", "U", "fstar", "fib"):
            np.testing.assert_array_equal(getattr(sb, k), getattr(ss, k), err_msg=f"{cfg.ibm_method} {k}")
        np.testing.assert_array_equal(eb.fpost_aos(), es.fpost_aos())
        assert eb.cd_cl() == es.cd_cl()


def test_step_io_matches_plain_steps(torch):
    """A step driven with host I/O (markers in from pinned memory, forces out,
    one graph per parity) computes the same bits as plain eager steps."""
    from iblbm_b200.batch import Batch
    cfgs = [_cfg(**kw) for kw in CASES]
    a, b = Batch(cfgs), Batch(cfgs)
    a.advance(5, outputs_last=False)
    b.advance(5, outputs_last=False)
    host_in = torch.empty(a.marker_in.numel(), dtype=torch.float64).pin_memory()
    host_in.copy_(a.marker_in.cpu())
    host_out = torch.empty(a.marker_out.numel(), dtype=torch.float64).pin_memory()
    for _ in range(6):
        a.step_io(host_in, host_out)
    b.advance(6, outputs_last=False, use_graph=False)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host_out.numpy(), b.marker_out.cpu().numpy())
    for ea, eb in zip(a.engines, b.engines):
        np.testing.assert_array_equal(ea.fpost_aos(), eb.fpost_aos())
    # one step ahead with two alternating buffer pairs
    ins = [host_in, torch.empty_like(host_in).pin_memory()]
    ins[1].copy_(host_in)
    outs = [host_out, torch.empty_like(host_out).pin_memory()]
    evs = [a.step_io(ins[k % 2], outs[k % 2], wait=False) for k in range(5)]
    evs[-1].synchronize()
    b.advance(5, outputs_last=False, use_graph=False)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(outs[0].numpy(), b.marker_out.cpu().numpy())  # the fifth step used outs[0]
    for ea, eb in zip(a.engines, b.engines):
        np.testing.assert_array_equal(ea.fpost_aos(), eb.fpost_aos())


def test_fp64_batch_matches_single_cases(torch):
    """The FP64 batch (plain form): every case bit for bit equal to its own
    FP64 engine, whose arithmetic is the reference's (moving and fixed bodies,
    every band method and collision model of CASES)."""
    from iblbm_b200.batch import Batch
    from iblbm_b200.engine import Engine
    cfgs = [_cfg(**kw) for kw in CASES]
    b = Batch(cfgs, precision="f64")
    b.advance(61, outputs_last=True)
    torch.cuda.synchronize()
    assert b.status() == [0] * len(cfgs)
    for cfg, eb in zip(cfgs, b.engines):
        es = Engine(cfg, precision="f64")
        es.advance(61, outputs_last=True)
        torch.cuda.synchronize()
        assert es.status() == 0
        sb, ss = eb.read_state(), es.read_state()
        for k in ("ro", "U", "fstar", "fib", "feq"):
            np.testing.assert_array_equal(getattr(sb, k), getattr(ss, k), err_msg=f"{cfg.ibm_method} {k}")
        np.testing.assert_array_equal(eb.fpost_aos(), es.fpost_aos())
        assert eb.cd_cl() == es.cd_cl()
