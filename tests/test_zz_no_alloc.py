"""The band step that allocates nothing (iblbm_ibm_step_f64_noalloc).

Some callers cannot allocate device memory when they call this library — a host
framework that owns every device allocation and gives plugins only the buffers
they declared, or a service that forbids cudaMalloc after start-up because it
can synchronize the device.  The no-allocation entry point serves them by
taking the band kernel's per-launch scratch from a fixed array compiled into
the library.  These tests call it through the C ABI and check that it produces
exactly what the allocating entry point produces (bit for bit, the tolerance of
every FP64 parity test here), on two calls in a row, and that it refuses sizes
beyond its fixed capacity.

This file is named to be collected last: its first GPU call resolves the
array's device address, and it must pass both alone and after the other tests.
"""
import ctypes

import numpy as np
import pytest


def _cfg(kw):
    from iblbm_b200.config import SimConfig
    kw = dict(kw)
    kw["cylinder_center"] = tuple(kw["cylinder_center"])
    return SimConfig(**kw)


def test_noalloc_rejects_sizes_beyond_its_capacity():
    """Host-side check: no launch, no device call needed."""
    from iblbm_b200 import _lib
    L = _lib.lib()
    a = _lib.IbmArgs()
    a.lb_total = 1025
    a.band_capacity = 100
    assert L.iblbm_ibm_step_f64_noalloc(ctypes.byref(a), None) == -3
    a.lb_total = 10
    a.band_capacity = 4097
    assert L.iblbm_ibm_step_f64_noalloc(ctypes.byref(a), None) == -3
    a.band_capacity = 2049  # above the band kernel's own limit
    assert L.iblbm_ibm_step_f64_noalloc(ctypes.byref(a), None) == -3
    assert L.iblbm_ibm_step_f64_noalloc(None, None) == -1


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_mdf_trt_p4", "c3_dfc_bgk_p4_osc", "dfc_trt_hat_fixed"])
def test_noalloc_band_step_matches_allocating_entry(name):
    """Two identical engines: one band step through each entry point, twice in a
    row (rebuild, then cached lists / next oscillation phase); every band output
    must agree bit for bit."""
    import torch
    from iblbm_b200 import _lib
    from iblbm_b200.engine import Engine
    from tests.golden.make_golden import RUN_CASES
    L = _lib.lib()
    kw = dict(RUN_CASES[name], max_steps=20)
    e1, e2 = Engine(_cfg(kw)), Engine(_cfg(kw))
    stream = torch.cuda.current_stream().cuda_stream
    outputs = ("d_fib", "d_df", "d_stats", "d_dstats", "d_Lux", "d_Luy", "d_Lfx", "d_Lfy", "d_dfc_force",
               "d_lambda", "d_count", "d_nodes", "d_box", "d_map", "d_excl")
    for call in range(2):
        for eng, fn in ((e1, L.iblbm_ibm_step_f64), (e2, L.iblbm_ibm_step_f64_noalloc)):
            a = eng.ibm_args[eng.parity]
            a.rebuild = 1 if (call == 0 or eng.moving) else 0
            a.excl_cur = 0
            assert fn(ctypes.byref(a), stream) == 0
        torch.cuda.synchronize()
        assert int(e1.d_stats[4].item()) == 0 and int(e2.d_stats[4].item()) == 0
        for k in outputs:
            x, y = getattr(e1, k), getattr(e2, k)
            assert torch.equal(x, y), (name, call, k)
        nb = int(e1.d_count.item())
        assert nb > 0
        if e1.method in ("DF", "MDF"):
            assert float(e1.d_fib[: 2 * nb].abs().sum()) > 0.0
        else:
            # a body at rest in a fluid at rest needs no correction (zero Delta f)
            # on the first steps; its lambda(k) is non-trivial
            assert bool((e1.d_lambda[: e1.Lb] > 0.0).all())
    np.testing.assert_array_equal(e1.d_fib.cpu().numpy(), e2.d_fib.cpu().numpy())
