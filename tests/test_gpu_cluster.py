"""The FP64 MDF band step of one fixed body on a thread-block cluster against
the single-CTA step: same operations in the same order, so the same bits.

The single-CTA step is itself bit-exact against the oracle (test_gpu_parity.py,
whose MDF cases now run on the cluster by default), so these tests pin the
cluster form to it on more shapes: both delta kernels, dense marker sets, every
cluster size, the three collision models and the device fallback."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _cfg(**over):
    from iblbm_b200.config import SimConfig
    kw = dict(Re=100, NN=161, xmax=2.5, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.0625,
              lattice_u=0.04, inflow_u=0.04, bc_type="dirichlet_neumann", delta_type="peskin4pt",
              ibm_method="MDF", collision_model="TRT", trt_magic_param=0.1875, mdf_iterations=20,
              mdf_min_iterations=5, mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=60,
              use_convergence=False, check_interval=50)
    kw.update(over)
    return SimConfig(**kw)


def _pair(torch, cfg, size, steps=60, graph=True):
    from iblbm_b200.engine import Engine
    a, b = Engine(cfg, cluster=size), Engine(cfg, cluster=0)
    assert a.cluster == size and b.cluster == 0
    for e in (a, b):
        e.advance(steps, outputs_last=True, use_graph=graph)
    torch.cuda.synchronize()
    assert a.status() == 0 and b.status() == 0
    return a, b


def _same(a, b):
    s1, s2 = a.read_state(), b.read_state()
    for k in ("fstar", "U", "ro", "fib"):
        np.testing.assert_array_equal(getattr(s1, k), getattr(s2, k), err_msg=k)
    np.testing.assert_array_equal(a.fpost_aos(), b.fpost_aos())
    for k in ("d_Lux", "d_Luy", "d_Lfx", "d_Lfy", "d_dstats"):
        np.testing.assert_array_equal(getattr(a, k).cpu().numpy(), getattr(b, k).cpu().numpy(), err_msg=k)
    np.testing.assert_array_equal(a.d_stats[:3].cpu().numpy(), b.d_stats[:3].cpu().numpy())


@pytest.mark.parametrize("size", [2, 4, 8])
@pytest.mark.parametrize("delta", ["peskin4pt", "hat"])
def test_cluster_matches_single_cta(torch, size, delta):
    a, b = _pair(torch, _cfg(delta_type=delta), size)
    assert a.mdf_stats()["cluster"]
    assert not b.mdf_stats()["cluster"]
    _same(a, b)


@pytest.mark.parametrize("collision", ["BGK", "CM_MRT"])
def test_cluster_collision_models(torch, collision):
    a, b = _pair(torch, _cfg(collision_model=collision), 8)
    assert a.mdf_stats()["cluster"]
    _same(a, b)


def test_cluster_dense_markers_eager(torch):
    """Markers every 0.3 dx (105 markers, lists of up to 23 entries), eager launches."""
    a, b = _pair(torch, _cfg(marker_spacing_factor=0.3), 8, steps=30, graph=False)
    assert a.Lb == 105 and a.mdf_stats()["cluster"]
    _same(a, b)


def test_cluster_falls_back_when_lists_exceed_the_stencil(torch):
    """Markers every 0.25 dx: a node's list reaches 28 entries, more than the 25
    a node holds in registers, so the plan does not hold and the cluster's first
    CTA runs the single-CTA step (stats[3] is not -3); the bits stay the same."""
    a, b = _pair(torch, _cfg(marker_spacing_factor=0.25), 8, steps=20)
    assert a.Lb == 126
    assert not a.mdf_stats()["cluster"]
    assert a.d_plan[8:16].cpu().numpy().min() == 0  # some rank found a long list
    _same(a, b)


def test_cluster_full_size_config2(torch):
    """Configuration 2 (1601 x 641, 126 markers, Peskin-4, TRT) for 100 steps on
    8 CTAs against the single-CTA step."""
    import bench
    cfg = bench.workload_config(max_steps=100)
    a, b = _pair(torch, cfg, 8, steps=100)
    assert a.mdf_stats()["cluster"] and a.Lb == 126
    _same(a, b)



def test_cluster_falls_back_when_nodes_exceed_the_threads(torch):
    """A body of 251 markers (D = 80) on 2 CTAs: each rank's markers cover more
    band nodes than a CTA has threads after its marker warps, so the plan does
    not hold and the single-CTA step runs in the launch; the bits stay the same."""
    a, b = _pair(torch, _cfg(cylinder_D_ratio=0.5), 2, steps=20)
    assert a.Lb == 251
    assert not a.mdf_stats()["cluster"]
    assert a.d_plan[8:10].cpu().numpy().min() == 0
    _same(a, b)


@pytest.mark.parametrize("size", [2, 4])
def test_cluster_sizes_full_size_config2(torch, size):
    """Configuration 2 on 2 and 4 CTAs (63 and 32 markers per CTA)."""
    import bench
    cfg = bench.workload_config(max_steps=40)
    a, b = _pair(torch, cfg, size, steps=40)
    assert a.mdf_stats()["cluster"]
    _same(a, b)
