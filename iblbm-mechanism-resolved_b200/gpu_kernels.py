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


# ---- immersed boundary: reference-shaped wrappers over the band kernel ---------
_DELTA_TYPE_IDS = {"peskin4pt": 0, "hat": 1}
_DELTA_STENCIL_A = {"peskin4pt": 2, "hat": 1}
_BLOCK = 256


def _grid(n):
    """Launch grid of the reference's raw DF kernels (one thread per marker)."""
    return ((int(n) + _BLOCK - 1) // _BLOCK,)


class _RawKernel:
    """The reference's raw-kernel call convention, kern(grid, block, args):
    iblbm/gpu_kernels.py `_ibm_interp_force_kern` / `_ibm_spread_kern`, as
    launched by iblbm/ibm/forcing.py:185-231 (the GPU branch of the per-particle
    DF closure).  grid and block are accepted and ignored: the band step sizes
    its own launch."""

    def __init__(self, fn):
        self._fn = fn

    def __call__(self, grid, block, args):
        return self._fn(*args)


def _delta_name(delta_type_id):
    return {v: k for k, v in _DELTA_TYPE_IDS.items()}[int(delta_type_id)]


def _interp_force(Lx, Ly, desired_vel, Eux, Euy, Ro, dx, dy, dt, nx, ny, Lb, delta_type_id, stencil_a,
                  incompressible, Lfx, Lfy, Lux, Luy):
    """Per marker: interpolated velocity (Lux, Luy) and force
    F = 2 rho (U_d - U) / dt (or 2 (U_d - U) / dt incompressible), written into
    the given arrays; the DF band step on the given fields, bit for bit the
    reference's CPU ibm_direct_forcing (iblbm/ibm/df.py:93-126)."""
    nx, ny = int(nx), int(ny)
    k = _band_call("DF", Lx, Ly, desired_vel, float(dx), float(dy), float(dt), 1.0, ny, nx,
                   _delta_name(delta_type_id), bool(int(incompressible)), ro=_dev(Ro, "Ro").reshape(-1),
                   ux=_dev(Eux, "Eux").reshape(-1), uy=_dev(Euy, "Euy").reshape(-1))
    for dst, src in ((Lfx, "Lfx"), (Lfy, "Lfy"), (Lux, "Lux"), (Luy, "Luy")):
        dst.reshape(-1).copy_(k[src][: int(Lb)])


def _spread(Lfx, Lfy, Lx, Ly, dx, dy, Larea, nx, ny, Lb, delta_type_id, stencil_a, Efx, Efy):
    """Add each marker's force, spread by its stencil weights times Larea, into
    Efx / Efy ((ny, nx) fields; iblbm/ibm/df.py:128-154 order: stencil slot,
    then marker)."""
    torch = _t()
    nx, ny = int(nx), int(ny)
    dev = _dev(Lx, "Lx").device
    N = nx * ny
    ones = torch.ones(N, dtype=torch.float64, device=dev)
    zeros = torch.zeros(N, dtype=torch.float64, device=dev)
    k = _band_call("DF", Lx, Ly, None, float(dx), float(dy), 1.0, float(Larea), ny, nx, _delta_name(delta_type_id),
                   False, ro=ones, ux=zeros, uy=zeros, given_force=(Lfx, Lfy))
    nb = k["nb"]
    f = k["fib"][: 2 * nb].reshape(nb, 2)
    Efx.reshape(-1).index_add_(0, k["nodes_l"], f[:, 0])
    Efy.reshape(-1).index_add_(0, k["nodes_l"], f[:, 1])


_ibm_interp_force_kern = _RawKernel(_interp_force)
_ibm_spread_kern = _RawKernel(_spread)


def _band_call(method, Lx, Ly, desired_vel, dx, dy, dt, Larea, ny, nx, delta_type, incompressible,
               ro=None, ux=None, uy=None, ustride=1, fstar=None, lambda_k=None, rho_f=1.0, given_force=None):
    """One band-kernel launch on caller-given fields (iblbm_ibm_step_f64 with
    field_*): returns the band's node list and outputs."""
    import numpy as np
    from ._lib import DELTA_IDS, IBM_IDS, Case, Geom, IbmArgs
    from .engine import band_capacity
    torch = _t()
    L = lib()
    Lx, Ly = _dev(Lx, "Lx"), _dev(Ly, "Ly")
    dev = Lx.device
    Lb = int(Lx.numel())
    N = nx * ny
    B = band_capacity(Lx.cpu().numpy(), Ly.cpu().numpy(), dx, dy, nx, ny, delta_type)
    i32, f64 = torch.int32, torch.float64
    z = lambda n, dt=f64: torch.zeros(max(int(n), 1), dtype=dt, device=dev)
    dv = _dev(desired_vel, "desired_vel").reshape(-1) if desired_vel is not None else z(2 * Lb)
    delta = DELTA_IDS[delta_type]
    c = Case()
    c.collision, c.bc, c.incompressible, c.tau, c.dt, c.dens = 0, 0, int(bool(incompressible)), 1.0, float(dt), 1.0
    a = IbmArgs()
    a.g = Geom(nx, ny, (nx + 31) // 32 * 32, ((nx + 31) // 32 * 32) * ny)
    a.c = c
    a.method, a.delta_type, a.rebuild, a.n_particles, a.lb_total = IBM_IDS[method], delta, 1, 1, Lb
    keep = {}
    keep["moff"] = torch.tensor([0, Lb], dtype=i32, device=dev)
    keep["larea"] = torch.tensor([float(Larea)], dtype=f64, device=dev)
    keep["map"] = torch.full((N,), -1, dtype=i32, device=dev)
    for k, n, dt_ in (("box", 4, i32), ("nodes", B, i32), ("count", 1, i32), ("stats", 5, i32), ("dstats", 2, f64),
                      ("fib", 2 * B, f64), ("df", 9 * B, f64), ("Lux", Lb, f64), ("Luy", Lb, f64),
                      ("Lfx", Lb, f64), ("Lfy", Lb, f64), ("force", 2 * Lb, f64), ("valid", 1, i32)):
        keep[k] = z(n, dt_)
    keep["lam"] = _dev(lambda_k, "lambda_k").clone() if lambda_k is not None else z(Lb)
    keep["scr"] = z(L.iblbm_ibm_scratch_doubles(Lb, B, 1))
    keep["iscr"] = z(L.iblbm_ibm_scratch_ints(Lb, B, delta), i32)
    keep["lists"] = z(L.iblbm_ibm_list_cache_ints(Lb, B, delta), i32)
    a.moff, a.Lx, a.Ly, a.dvel, a.larea = (ptr(x) for x in (keep["moff"], Lx, Ly, dv, keep["larea"]))
    a.dx, a.dy = float(dx), float(dy)
    a.lambda_, a.lambda_valid = ptr(keep["lam"]), ptr(keep["valid"])
    a.dfc_rho_f = float(rho_f)
    if lambda_k is not None:
        keep["valid"].fill_(1)
        a.dfc_cache_lambda = 1
    a.correction_scale = 1.0
    a.box, a.map, a.band_nodes, a.band_count = (ptr(keep[k]) for k in ("box", "map", "nodes", "count"))
    a.list_cache = ptr(keep["lists"])
    a.band_capacity, a.box_capacity = B, N
    a.band_fib, a.band_df, a.scratch, a.iscratch = (ptr(keep[k]) for k in ("fib", "df", "scr", "iscr"))
    if given_force is not None:  # spread the given marker forces (DF)
        keep["Lfx"], keep["Lfy"] = (_dev(f, "Lf").reshape(-1).contiguous().clone() for f in given_force)
        a.df_given_force = 1
    a.Lux, a.Luy, a.Lfx, a.Lfy, a.dfc_force = (ptr(keep[k]) for k in ("Lux", "Luy", "Lfx", "Lfy", "force"))
    a.stats, a.dstats = ptr(keep["stats"]), ptr(keep["dstats"])
    if fstar is not None:
        keep["fstar"] = _dev(fstar, "fstar")
        a.field_fstar = ptr(keep["fstar"])
    else:
        keep["ro"], keep["ux"], keep["uy"] = ro, ux, uy
        a.field_ro, a.field_ux, a.field_uy, a.field_ustride = ptr(ro), ptr(ux), ptr(uy), int(ustride)
    check(L.iblbm_ibm_step_f64(ctypes.byref(a), _stream(Lx)), "iblbm_ibm_step_f64")
    st = int(keep["stats"][4].item())
    if st != 0:
        raise RuntimeError(f"band kernel status {st}")
    nb = int(keep["count"].item())
    keep["nb"] = nb
    keep["nodes_l"] = keep["nodes"][:nb].long()
    return keep


def ibm_direct_forcing_gpu(Lx, Ly, desired_vel, Eux, Euy, Ro, dx, dy, dt, Larea, ny, nx, delta_type="peskin4pt",
                           return_interp_vel=False, incompressible=False):
    """Direct forcing — replaces gpu_kernels.py:956-1042 (<- ibm/df.py:37-154).
    Eux, Euy, Ro: (ny, nx) or (N,); returns fib (N, 2) [, Lux, Luy].  Sums run
    in the reference CPU path's order, so results are bit-identical to it."""
    Eux, Euy, Ro = (_dev(x, n).reshape(-1) for x, n in ((Eux, "Eux"), (Euy, "Euy"), (Ro, "Ro")))
    k = _band_call("DF", Lx, Ly, desired_vel, dx, dy, dt, Larea, ny, nx, delta_type, incompressible,
                   ro=Ro, ux=Eux, uy=Euy)
    torch = _t()
    fib = torch.zeros(ny * nx, 2, dtype=torch.float64, device=Eux.device)
    nb = k["nb"]
    fib[k["nodes_l"]] = k["fib"][: 2 * nb].reshape(nb, 2)
    if return_interp_vel:
        return fib, k["Lux"], k["Luy"]
    return fib


def ibm_direct_forcing_fields_gpu(Lx, Ly, desired_vel, Eux, Euy, Ro, dx, dy, dt, Larea, ny, nx,
                                  delta_type="peskin4pt", incompressible=False):
    """Direct forcing returning the unpacked force fields — replaces
    gpu_kernels.py:1045-1088: (Efx, Efy) as (ny, nx), Lux, Luy."""
    fib, Lux, Luy = ibm_direct_forcing_gpu(Lx, Ly, desired_vel, Eux, Euy, Ro, dx, dy, dt, Larea, ny, nx, delta_type,
                                           True, incompressible)
    return fib[:, 0].reshape(ny, nx).contiguous(), fib[:, 1].reshape(ny, nx).contiguous(), Lux, Luy


def compute_lambda_gpu(Lx, Ly, rho_f, Larea, dx, dy, ny, nx, delta_type):
    """DFC lambda(k) = 1 / (2 rho_f ds W_sum(k)) — replaces gpu_kernels.py:1091-1141
    (<- ibm/dfc.py:126-186), bit-identical to the reference for every fluid
    density rho_f > 0 (the band kernel evaluates ((2 rho_f) ds) W_sum as the
    reference does).  rho_f <= 0 has no physical meaning and raises ValueError."""
    if not float(rho_f) > 0.0:
        raise ValueError(f"rho_f={rho_f!r}: the fluid density must be positive")
    torch = _t()
    fz = torch.zeros(ny * nx * 9, dtype=torch.float64, device=_dev(Lx, "Lx").device)
    k = _band_call("DFC", Lx, Ly, None, dx, dy, 1.0, Larea, ny, nx, delta_type, False, fstar=fz, rho_f=rho_f)
    return k["lam"][: Lx.numel()].clone()


def dfc_correction_gpu(Lx, Ly, desired_vel, fstar, lambda_k, dx, dy, Larea, ny, nx, delta_type, lattice=None):
    """DFC distribution correction — replaces gpu_kernels.py:1144-1223
    (<- ibm/dfc.py:55-253): returns (Ef_corr (N, 9), dfc_force (Lb, 2))."""
    torch = _t()
    fstar = _dev(fstar, "fstar")
    k = _band_call("DFC", Lx, Ly, desired_vel, dx, dy, 1.0, Larea, ny, nx, delta_type, False,
                   fstar=fstar.reshape(-1), lambda_k=lambda_k)
    nb = k["nb"]
    corr = torch.zeros(ny * nx, 9, dtype=torch.float64, device=fstar.device)
    corr[k["nodes_l"]] = k["df"][: 9 * nb].reshape(nb, 9)
    Lb = int(Lx.numel())
    return corr, k["force"][: 2 * Lb].reshape(Lb, 2).clone()
