"""Drop-in for iblbm/gpu_kernels.py's dense wrappers, over torch CUDA tensors.

Same names, arguments and return conventions as the reference (each returns
new arrays, except ``velocity_correction_gpu`` which updates U in place);
arrays use the reference's shapes: populations (N, 9), U and fib (N, 2), ro (N,).
Every call launches this package's sm_100a kernels through the C ABI; inputs
must be float64 CUDA tensors.
"""
from __future__ import annotations

import ctypes

from ._lib import check, lib, ptr


def _t():
    import torch
    return torch


def _dev(x, name):
    torch = _t()
    if not isinstance(x, torch.Tensor) or not x.is_cuda or x.dtype != torch.float64:
        raise TypeError(f"{name} must be a float64 CUDA tensor")
    return x.contiguous()


def _stream(x):
    return _t().cuda.current_stream(x.device).cuda_stream


def collision_gpu(fstar, feq, U, fib, tau, dt):
    """BGK + Guo forcing — replaces gpu_kernels.py:760-784."""
    fstar, feq, U, fib = (_dev(a, n) for a, n in ((fstar, "fstar"), (feq, "feq"), (U, "U"), (fib, "fib")))
    f = _t().empty_like(fstar)
    check(lib().iblbm_collision_bgk(ptr(fstar), ptr(feq), ptr(U), ptr(fib), fstar.shape[0], float(tau),
                                    float(dt), ptr(f), _stream(f)), "collision_gpu")
    return f


def collision_trt_gpu(fstar, feq, U, fib, tau, tau_minus, dt):
    """TRT + Guo forcing — replaces gpu_kernels.py:787-812."""
    fstar, feq, U, fib = (_dev(a, n) for a, n in ((fstar, "fstar"), (feq, "feq"), (U, "U"), (fib, "fib")))
    f = _t().empty_like(fstar)
    check(lib().iblbm_collision_trt(ptr(fstar), ptr(feq), ptr(U), ptr(fib), fstar.shape[0], float(tau),
                                    float(tau_minus), float(dt), ptr(f), _stream(f)), "collision_trt_gpu")
    return f


def collision_cm_mrt_gpu(fstar, feq, U, fib, S_diag, dt):
    """Central-moment MRT + Guo forcing — replaces gpu_kernels.py:815-843 (feq is unused, as there)."""
    fstar, U, fib = (_dev(a, n) for a, n in ((fstar, "fstar"), (U, "U"), (fib, "fib")))
    f = _t().empty_like(fstar)
    S = (ctypes.c_double * 9)(*[float(v) for v in S_diag])
    check(lib().iblbm_collision_cm_mrt(ptr(fstar), ptr(U), ptr(fib), fstar.shape[0], S, float(dt), ptr(f),
                                       _stream(f)), "collision_cm_mrt_gpu")
    return f


def streaming_gpu(fstar_old, f, nx, ny):
    """D2Q9 streaming; out-of-lattice sources keep fstar_old — replaces gpu_kernels.py:846-875."""
    fstar_old, f = _dev(fstar_old, "fstar_old"), _dev(f, "f")
    out = _t().empty_like(fstar_old)
    check(lib().iblbm_streaming(ptr(fstar_old), ptr(f), int(nx), int(ny), ptr(out), _stream(out)), "streaming_gpu")
    return out


def macroscopic_gpu(fstar, incompressible=False):
    """(ro, U) from the populations — replaces gpu_kernels.py:878-903."""
    torch = _t()
    fstar = _dev(fstar, "fstar")
    N = fstar.shape[0]
    ro = torch.empty(N, dtype=torch.float64, device=fstar.device)
    U = torch.empty((N, 2), dtype=torch.float64, device=fstar.device)
    check(lib().iblbm_macroscopic(ptr(fstar), N, int(bool(incompressible)), ptr(ro), ptr(U), _stream(ro)),
          "macroscopic_gpu")
    return ro, U


def feq_gpu(ro, U, incompressible=False):
    """Equilibrium populations (N, 9) — replaces gpu_kernels.py:906-927."""
    torch = _t()
    ro, U = _dev(ro, "ro"), _dev(U, "U")
    N = ro.shape[0]
    feq = torch.empty((N, 9), dtype=torch.float64, device=ro.device)
    check(lib().iblbm_feq(ptr(ro), ptr(U), N, int(bool(incompressible)), ptr(feq), _stream(feq)), "feq_gpu")
    return feq


def velocity_correction_gpu(U, fib, ro, dt, incompressible=False):
    """u += fib dt / (2 ro) in place (incompressible: u += fib dt / 2) — replaces gpu_kernels.py:930-948."""
    if not U.is_contiguous():
        raise ValueError("U must be contiguous (updated in place)")
    _dev(U, "U")
    fib, ro = _dev(fib, "fib"), _dev(ro, "ro")
    check(lib().iblbm_velocity_correction(ptr(U), ptr(fib), ptr(ro), U.shape[0], float(dt),
                                          int(bool(incompressible)), _stream(U)), "velocity_correction_gpu")
