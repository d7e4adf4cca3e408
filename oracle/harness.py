"""Python driver of the CPU oracle (test infrastructure only).

Restates the reference's host-side pieces around the C kernels of
``iblbm_oracle.c``:

- ``init_state``   iblbm/init.py:116-265 (grid, tau, markers, feq -> fstar) and
                   iblbm/physics/sedimentation.py:94-219 (particles);
- ``OracleSim``    the time loop of iblbm/runtime/loop.py:44-151 for the fixed /
                   oscillating cylinder runtime (runtime/scenarios/fixed_cylinder.py)
                   and the multi-particle sedimentation runtime
                   (runtime/scenarios/sedimentation_multi.py), with the IBM
                   strategies of iblbm/ibm/strategies/{df,mdf,dfc}.py;
- ``mdf_omega``    iblbm/ibm/a_norm.py:204-266.

The configuration object is duck-typed: any object with the reference
``SimConfig`` attribute names works (the reference's own or the product's).
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
module; it is the checker, never the thing measured or shipped.
"""
from __future__ import annotations

import ctypes
import math
import os
from types import SimpleNamespace

import numpy as np

from .build import build_oracle

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_lib = None

BC_IDS = {"dirichlet_neumann": 0, "open_boundary": 1, "settling_channel": 2, "velocity_inlet": 3}
DELTA_IDS = {"peskin4pt": 0, "hat": 1}
MDF_COUPLED_OMEGA_MAX = 0.8  # iblbm/ibm/multi_particle.py:33


def lib():
    """Load (building first if needed) the oracle shared library."""
    global _lib
    if _lib is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "liboracle.so")
        if not os.path.exists(path):
            path = build_oracle()
        _lib = ctypes.CDLL(path)
        _lib.orc_a_norm_inf.restype = ctypes.c_double
        _lib.orc_bc.restype = ctypes.c_int
    return _lib


def _p(a):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    if a.dtype == np.float64:
        return a.ctypes.data_as(_D)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_I)
    raise TypeError(a.dtype)


# --------------------------------------------------------------------------
# Kernel wrappers (AoS arrays, the reference's layout)
# --------------------------------------------------------------------------
def feq(ro, U, incompressible=False):
    out = np.empty((ro.shape[0], 9))
    lib().orc_feq(ctypes.c_int(ro.shape[0]), _p(ro), _p(U), ctypes.c_int(int(incompressible)), _p(out))
    return out


def macroscopic(fstar, incompressible=False):
    N = fstar.shape[0]
    ro = np.empty(N)
    U = np.empty((N, 2))
    lib().orc_macro(ctypes.c_int(N), _p(fstar), ctypes.c_int(int(incompressible)), _p(ro), _p(U))
    return ro, U


def collide_bgk(fstar, feq_, U, fib, tau, dt):
    f = np.empty_like(fstar)
    lib().orc_collide_bgk(ctypes.c_int(fstar.shape[0]), _p(fstar), _p(feq_), _p(U), _p(fib),
                          ctypes.c_double(tau), ctypes.c_double(dt), _p(f))
    return f


def collide_trt(fstar, feq_, U, fib, tau, tau_minus, dt):
    f = np.empty_like(fstar)
    lib().orc_collide_trt(ctypes.c_int(fstar.shape[0]), _p(fstar), _p(feq_), _p(U), _p(fib),
                          ctypes.c_double(1.0 / tau), ctypes.c_double(1.0 / tau_minus),
                          ctypes.c_double(dt), _p(f))
    return f


def collide_cmmrt(fstar, U, fib, S_diag, dt):
    f = np.empty_like(fstar)
    S = np.ascontiguousarray(S_diag, dtype=np.float64)
    lib().orc_collide_cmmrt(ctypes.c_int(fstar.shape[0]), _p(fstar), _p(U), _p(fib), _p(S),
                            ctypes.c_double(dt), _p(f))
    return f


def stream(fstar_old, f, nx, ny):
    out = np.empty_like(fstar_old)
    lib().orc_stream(ctypes.c_int(nx), ctypes.c_int(ny), _p(fstar_old), _p(f), _p(out))
    return out


def apply_bc(bc_type, nx, ny, fstar, ro, U, inflow_u, dens, incompressible=False):
    rc = lib().orc_bc(ctypes.c_int(BC_IDS[bc_type]), ctypes.c_int(nx), ctypes.c_int(ny), _p(fstar),
                      _p(ro), _p(U), ctypes.c_double(inflow_u), ctypes.c_double(dens),
                      ctypes.c_int(int(incompressible)))
    if rc != 0:
        raise KeyError(bc_type)


def tg_velocity(X, Y, t, u0, L, nu):
    """Decaying Taylor-Green vortex — iblbm/diagnostics/core.py:216-241 (same expressions)."""
    decay = np.exp(-2.0 * nu * (np.pi / L) ** 2 * t)
    ux = -u0 * np.cos(np.pi * X / L) * np.sin(np.pi * Y / L) * decay
    uy = u0 * np.sin(np.pi * X / L) * np.cos(np.pi * Y / L) * decay
    return ux, uy


def tg_params(cfg):
    """Half-width and viscosity of the vortex (iblbm/boundary/tg_analytical.py:49-51)."""
    L_lat = 0.5 * (cfg.NN - 1)
    nu = cfg.lattice_u * (cfg.cylinder_D_ratio * (cfg.NN - 1)) / cfg.Re
    return L_lat, nu


def tg_face_velocities(cfg, nx, ny, t):
    """The analytic velocities of iblbm/boundary/tg_analytical.py:53-163 at time t:
    (left j=0..ny-1, right j=0..ny-1, bottom i=1..nx-2, top i=1..nx-2, corners),
    each an (n, 2) array."""
    L_lat, nu = tg_params(cfg)
    X = np.arange(nx, dtype=float) - (nx - 1) / 2.0
    Y = np.arange(ny, dtype=float) - (ny - 1) / 2.0
    j = np.arange(ny)
    i = np.arange(1, nx - 1)
    out = []
    for xs, ys in ((np.full_like(j, X[0], dtype=float), Y[j]), (np.full_like(j, X[nx - 1], dtype=float), Y[j]),
                   (X[i], np.full_like(i, Y[0], dtype=float)), (X[i], np.full_like(i, Y[ny - 1], dtype=float)),
                   (X[np.array([0, nx - 1, 0, nx - 1])], Y[np.array([0, 0, ny - 1, ny - 1])])):
        ux, uy = tg_velocity(xs, ys, t, cfg.tg_u0, L_lat, nu)
        out.append(np.ascontiguousarray(np.stack([ux, uy], axis=1)))
    return out


def apply_bc_tg(cfg, nx, ny, fstar, ro, U, t):
    uL, uR, uB, uT, uC = tg_face_velocities(cfg, nx, ny, t)
    lib().orc_bc_tg(ctypes.c_int(nx), ctypes.c_int(ny), _p(fstar), _p(ro), _p(U), _p(uL), _p(uR), _p(uB),
                    _p(uT), _p(uC))


def velocity_correction(U, fib, ro, dt, incompressible=False):
    lib().orc_velocity_correction(ctypes.c_int(U.shape[0]), _p(U), _p(fib), _p(ro),
                                  ctypes.c_double(dt), ctypes.c_int(int(incompressible)))


def ibm_df(Lx, Ly, dvel, Eux, Euy, Ro, dx, dy, dt, Larea, ny, nx, delta_type, incompressible=False):
    Lb = len(Lx)
    fib = np.empty((nx * ny, 2))
    out = [np.empty(Lb) for _ in range(5)]
    lib().orc_ibm_df(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(Lb), _p(Lx), _p(Ly), _p(dvel),
                     _p(Eux), _p(Euy), _p(Ro), ctypes.c_double(dx), ctypes.c_double(dy),
                     ctypes.c_double(dt), ctypes.c_double(Larea), ctypes.c_int(DELTA_IDS[delta_type]),
                     ctypes.c_int(int(incompressible)), _p(fib), *[_p(o) for o in out])
    return (fib, *out)


def ibm_mdf(Lx, Ly, dvel, U, ro, dx, dy, dt, Larea, ny, nx, n_iter, min_iter, delta_type, omega, tol):
    fib = np.empty((nx * ny, 2))
    stats = np.zeros(3, dtype=np.int32)
    res = np.zeros(1)
    lib().orc_ibm_mdf(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(len(Lx)), _p(Lx), _p(Ly),
                      _p(dvel), _p(U), _p(ro), ctypes.c_double(dx), ctypes.c_double(dy),
                      ctypes.c_double(dt), ctypes.c_double(Larea), ctypes.c_int(int(n_iter)),
                      ctypes.c_int(int(min_iter)), ctypes.c_int(DELTA_IDS[delta_type]),
                      ctypes.c_double(omega), ctypes.c_double(tol), _p(fib), _p(stats), _p(res))
    return fib, {"iter_count": int(stats[0]), "last_residual": float(res[0]),
                 "diverged": bool(stats[1]), "converged": bool(stats[2])}


def mdf_coupled(parts, U, ro, dx, dy, dt, ny, nx, n_iter, min_iter, delta_type, omega_opt, tol,
                incompressible):
    """parts: list of (Lx, Ly, desired_velocity, Larea)."""
    P = len(parts)
    moff = np.zeros(P + 1, dtype=np.int32)
    for p, (lx, _, _, _) in enumerate(parts):
        moff[p + 1] = moff[p] + len(lx)
    Lx = np.ascontiguousarray(np.concatenate([p[0] for p in parts]))
    Ly = np.ascontiguousarray(np.concatenate([p[1] for p in parts]))
    dv = np.ascontiguousarray(np.concatenate([p[2] for p in parts]))
    La = np.array([float(p[3]) for p in parts])
    N = nx * ny
    fib = np.empty((N, 2))
    fpart = np.empty((P, N, 2))
    stats = np.zeros(4, dtype=np.int32)
    dstats = np.zeros(2)
    lib().orc_mdf_coupled(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(P), _p(moff), _p(Lx), _p(Ly),
                          _p(dv), _p(La), _p(U), _p(ro), ctypes.c_double(dx), ctypes.c_double(dy),
                          ctypes.c_double(dt), ctypes.c_int(int(n_iter)), ctypes.c_int(int(min_iter)),
                          ctypes.c_int(DELTA_IDS[delta_type]), ctypes.c_double(omega_opt),
                          ctypes.c_double(MDF_COUPLED_OMEGA_MAX), ctypes.c_double(tol),
                          ctypes.c_int(int(incompressible)), _p(fib), _p(fpart), _p(stats), _p(dstats))
    return fib, fpart, {"iter_count": int(stats[0]), "last_residual": float(dstats[0]),
                        "diverged": bool(stats[1]), "converged": bool(stats[2]),
                        "guard_trips": int(stats[3]), "omega_used": float(dstats[1])}


def dfc_lambda(Lx, Ly, Larea, dx, dy, ny, nx, delta_type, rho_f=1.0):
    lam = np.empty(len(Lx))
    lib().orc_dfc_lambda(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(len(Lx)), _p(Lx), _p(Ly),
                         ctypes.c_double(rho_f), ctypes.c_double(Larea), ctypes.c_double(dx),
                         ctypes.c_double(dy), ctypes.c_int(DELTA_IDS[delta_type]), _p(lam))
    return lam


def dfc_correction(Lx, Ly, dvel, fstar, lambda_k, dx, dy, Larea, ny, nx, delta_type, scale=1.0):
    """In-place on a copy of fstar; returns (fstar_corrected, dfc_force)."""
    fs = fstar.copy()
    force = np.empty((len(Lx), 2))
    lib().orc_dfc_correction(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(len(Lx)), _p(Lx), _p(Ly),
                             _p(dvel), _p(fs), _p(lambda_k), ctypes.c_double(dx), ctypes.c_double(dy),
                             ctypes.c_double(Larea), ctypes.c_int(DELTA_IDS[delta_type]),
                             ctypes.c_double(scale), _p(force))
    return fs, force


def mdf_omega(Lx, Ly, delta_type, Larea, dx):
    """omega = 1/||A||_inf — iblbm/ibm/a_norm.py:204-266 (coordinates /dx)."""
    Lx_lu = np.ascontiguousarray(np.asarray(Lx, dtype=np.float64) / float(dx))
    Ly_lu = np.ascontiguousarray(np.asarray(Ly, dtype=np.float64) / float(dx))
    norm = lib().orc_a_norm_inf(ctypes.c_int(len(Lx_lu)), _p(Lx_lu), _p(Ly_lu),
                                ctypes.c_int(DELTA_IDS[delta_type]), ctypes.c_double(float(Larea)))
    return 1.0 / norm


# --------------------------------------------------------------------------
# Initialisation — iblbm/init.py:116-265
# --------------------------------------------------------------------------
def circle_markers(cx, cy, r, lattice_r, dx, spacing, retraction_dx):
    """iblbm/init.py:211-243 and iblbm/physics/markers.py:61-85 (identical arithmetic)."""
    dd = 2.0 * np.pi * lattice_r / spacing
    step = 1.0 / dd
    Ldx = np.arange(0, 1.0 + step * 0.5, step)
    Ldx = Ldx[Ldx <= 1.0 + 1e-12]
    if len(Ldx) > 1 and np.abs(Ldx[-1] - 1.0) < step * 0.5:
        Ldx = Ldx[:-1]
    theta = 2.0 * np.pi * Ldx
    r_ret = r - retraction_dx * dx
    Lx = r_ret * np.cos(theta) + cx
    Ly = r_ret * np.sin(theta) + cy
    Lb = len(Lx)
    Larea = 2.0 * np.pi * (lattice_r - retraction_dx) / Lb
    return np.ascontiguousarray(Lx), np.ascontiguousarray(Ly), Lb, Larea


def init_state(cfg):
    if cfg.nx_formula == "standard":
        nx = int(cfg.NN * cfg.xmax - (cfg.xmax - 1))
    else:
        nx = int(cfg.NN * cfg.xmax)
    dx = 1.0 / (cfg.NN - 1)
    ny = round(cfg.ymax / dx) + 1
    dy = cfg.ymax / (ny - 1)
    if abs(dx - dy) / dx > 1e-6:
        raise ValueError("non-square lattice")
    N = nx * ny
    phy_char = cfg.phy_l * cfg.cylinder_D_ratio
    Cx = (cfg.phy_l / (cfg.NN - 1)) / 1.0
    r = phy_char / 2.0 / cfg.phy_l
    lattice_r = (phy_char / Cx) / 2.0
    tau = 3.0 * (cfg.lattice_u * 2.0 * lattice_r / cfg.Re) + 0.5
    U = np.zeros((N, 2))
    if cfg.scenario_type == "taylor_green":
        # iblbm/init.py:178-191: the vortex at t = 0 on centred lattice coordinates
        L_lat, nu = tg_params(cfg)
        XX, YY = np.meshgrid(np.arange(nx, dtype=float) - (nx - 1) / 2.0,
                             np.arange(ny, dtype=float) - (ny - 1) / 2.0)
        U[:, 0], U[:, 1] = tg_velocity(XX.ravel(), YY.ravel(), 0.0, cfg.tg_u0, L_lat, nu)
    elif cfg.motion_type not in ("oscillating", "sedimentation"):
        U[:, 0] = cfg.inflow_u
    ro = np.ones(N)
    fe = feq(ro, U, cfg.incompressible_lbgk)
    cx, cy = cfg.cylinder_center
    if cx - r < 0 or cx + r > cfg.xmax or cy - r < 0 or cy + r > cfg.ymax:
        raise ValueError("cylinder outside the domain")
    Lx, Ly, Lb, Larea = circle_markers(cx, cy, r, lattice_r, dx, cfg.marker_spacing_factor,
                                       cfg.retraction_dx)
    s = SimpleNamespace(nx=nx, ny=ny, N=N, dx=dx, dy=dy, dt=1.0, tau=tau, r=r, lattice_r=lattice_r,
                        in_u=cfg.inflow_u, dens=1.0, fstar=fe.copy(), feq=fe, ro=ro, U=U,
                        fib=np.zeros((N, 2)), Lx=Lx, Ly=Ly, Lb=Lb, Larea=Larea,
                        desired_velocity=np.zeros((Lb, 2)), lambda_cache=None, dfc_force_lagr=None,
                        particles=None, mdf_omega=None, mdf_stats=None)
    if cfg.collision_model == "TRT":
        s.tau_minus = 0.5 + cfg.trt_magic_param / (tau - 0.5)
    if cfg.collision_model == "CM_MRT":
        s_eps = cfg.mrt_s_eps if cfg.mrt_s_eps is not None else 1.4
        s_q = cfg.mrt_s_q if cfg.mrt_s_q is not None else 1.2
        s_nu = 1.0 / tau
        s.S_diag = np.array([0.0, 0.0, 0.0, s_nu, s_nu, s_nu, s_q, s_q, s_eps])
    if cfg.motion_type == "sedimentation":
        if cfg.gravity <= 0.0 or cfg.rho_ratio <= 1.0:
            raise ValueError("sedimentation needs gravity > 0 and rho_ratio > 1")
        s.gravity_lattice = cfg.gravity
        if cfg.particles_config is not None:
            parts = []
            for pc in cfg.particles_config:
                pcx, pcy = pc["center"]
                rho_p = pc["rho_ratio"]
                mass = rho_p * np.pi * lattice_r ** 2
                plx, ply, plb, pla = circle_markers(pcx, pcy, r, lattice_r, dx,
                                                    cfg.marker_spacing_factor, cfg.retraction_dx)
                parts.append(SimpleNamespace(
                    pos=np.array([pcx, pcy], dtype=float), vel=np.zeros(2), vel_prev=np.zeros(2),
                    force=np.zeros(2), mass=mass, rho_ratio=rho_p, lattice_r=lattice_r, r_domain=r,
                    I_particle=0.5 * mass * lattice_r ** 2, Lx_c=plx.copy(), Ly_c=ply.copy(),
                    Lx=plx, Ly=ply, Lb=plb, Larea=pla, desired_velocity=np.zeros((plb, 2)),
                    cx_init=pcx, cy_init=pcy, omega=0.0, torque=0.0, angle=0.0, l_int_prev=0.0))
            s.particles = parts
    return s


# --------------------------------------------------------------------------
# Rigid-body helpers — iblbm/physics/{gravity,rigid_body,markers}.py and
# iblbm/physics/inertia/{none,explicit_history,feng_b2}.py
# --------------------------------------------------------------------------
def _net_gravity(rho_ratio, r_lat, g, direction):
    mag = (rho_ratio - 1.0) * (np.pi * r_lat ** 2) * g
    return np.array([mag, 0.0]) if direction == "right" else np.array([0.0, -mag])


def _history_dv(model, vel, vel_prev, mass, r_lat):
    if model == "explicit_history":
        return (np.pi * r_lat ** 2 / mass) * (vel - vel_prev)
    return None


def _l_int_z(U, ro, nx, ny, dx, cx, cy, r_domain):
    """Angular momentum of the fluid inside a disc, sum of rx ro uy - ry ro ux over
    the nodes within r of the centre, lattice units — iblbm/diagnostics/internal_flow.py:220-262."""
    Eux, Euy, ro2 = U[:, 0].reshape(ny, nx), U[:, 1].reshape(ny, nx), ro.reshape(ny, nx)
    ci, cj, r_lat = cx / dx, cy / dx, r_domain / dx
    ii, jj, rr = int(round(ci)), int(round(cj)), int(r_lat) + 2
    i0, i1 = max(0, ii - rr), min(nx, ii + rr + 1)
    j0, j1 = max(0, jj - rr), min(ny, jj + rr + 1)
    RX, RY = np.meshgrid(np.arange(i0, i1, dtype=float) - ci, np.arange(j0, j1, dtype=float) - cj)
    m = RX ** 2 + RY ** 2 <= r_lat ** 2
    sro, sux, suy = ro2[j0:j1, i0:i1], Eux[j0:j1, i0:i1], Euy[j0:j1, i0:i1]
    return float(np.sum(RX[m] * sro[m] * suy[m] - RY[m] * sro[m] * sux[m]))


def _update_markers(Lx_c, Ly_c, cx0, cy0, pos, angle=0.0):
    cos_a = np.cos(angle)
    sin_a = np.sin(angle)
    rx = Lx_c - cx0
    ry = Ly_c - cy0
    return cos_a * rx - sin_a * ry + pos[0], sin_a * rx + cos_a * ry + pos[1]


# --------------------------------------------------------------------------
# Time loop — iblbm/runtime/loop.py:44-151
# --------------------------------------------------------------------------
class OracleSim:
    def __init__(self, cfg):
        self.cfg = cfg
        self.s = init_state(cfg)
        if cfg.motion_type == "sedimentation" and cfg.settling_inertia_model == "full_volume":
            raise NotImplementedError("full_volume inertia is outside the hot path")
        self.force_level = cfg.ibm_method in ("DF", "MDF")
        self.ttt = 1
        self.Cd_history = []
        self.Cl_history = []
        self.history = []
        self.Lx_c = self.s.Lx.copy()
        self.Ly_c = self.s.Ly.copy()
        if cfg.ibm_method == "MDF":
            s = self.s
            s.mdf_omega = mdf_omega(s.Lx, s.Ly, cfg.delta_type, float(s.Larea), float(s.dx))
            if cfg.motion_type == "sedimentation" and cfg.enable_rotation:
                s.mdf_omega = min(float(s.mdf_omega), 1.0)
        self.f = None
        if cfg.stream_first or self.force_level:
            self.f = self.collide()

    # iblbm/runtime/step.py:26-46 + iblbm/lbm/collision/*.py step_cpu
    def collide(self):
        s, cfg = self.s, self.cfg
        if cfg.collision_model == "BGK":
            return collide_bgk(s.fstar, s.feq, s.U, s.fib, s.tau, s.dt)
        if cfg.collision_model == "TRT":
            return collide_trt(s.fstar, s.feq, s.U, s.fib, s.tau, s.tau_minus, s.dt)
        if cfg.collision_model == "CM_MRT":
            return collide_cmmrt(s.fstar, s.U, s.fib, s.S_diag, s.dt)
        raise KeyError(cfg.collision_model)

    # iblbm/runtime/step.py:49-60
    def stream_boundary_macro(self):
        s, cfg = self.s, self.cfg
        s.fstar = stream(s.fstar, self.f, s.nx, s.ny)
        if cfg.scenario_type == "taylor_green":  # iblbm/boundary/base.py:52-53
            apply_bc_tg(cfg, s.nx, s.ny, s.fstar, s.ro, s.U, self.ttt * s.dt)
        else:
            apply_bc(cfg.bc_type, s.nx, s.ny, s.fstar, s.ro, s.U, s.in_u, s.dens, cfg.incompressible_lbgk)
        s.ro, s.U = macroscopic(s.fstar, cfg.incompressible_lbgk)

    def apply_ibm(self):
        s, cfg = self.s, self.cfg
        if cfg.scenario_type == "taylor_green" and not cfg.tg_with_ibm:  # iblbm/ibm/dispatch.py:38-39
            return
        if s.particles is not None:
            return self._apply_ibm_multi()
        if cfg.ibm_method == "DF":
            s.fib, s.Lux, s.Luy, s.Lfx, s.Lfy, s.R = ibm_df(
                s.Lx, s.Ly, np.ascontiguousarray(s.desired_velocity), np.ascontiguousarray(s.U[:, 0]),
                np.ascontiguousarray(s.U[:, 1]), s.ro, s.dx, s.dy, s.dt, s.Larea, s.ny, s.nx,
                cfg.delta_type, cfg.incompressible_lbgk)
            velocity_correction(s.U, s.fib, s.ro, s.dt, cfg.incompressible_lbgk)
        elif cfg.ibm_method == "MDF":
            s.fib, s.mdf_stats = ibm_mdf(
                s.Lx, s.Ly, np.ascontiguousarray(s.desired_velocity), s.U, s.ro, s.dx, s.dy, s.dt,
                s.Larea, s.ny, s.nx, cfg.mdf_iterations, cfg.mdf_min_iterations, cfg.delta_type,
                s.mdf_omega, cfg.mdf_tolerance)
            velocity_correction(s.U, s.fib, s.ro, s.dt, cfg.incompressible_lbgk)
        elif cfg.ibm_method == "DFC":
            lam = s.lambda_cache if cfg.motion_type is None else None
            if lam is None:
                lam = dfc_lambda(s.Lx, s.Ly, s.Larea, s.dx, s.dy, s.ny, s.nx, cfg.delta_type)
            s.fstar, s.dfc_force_lagr = dfc_correction(
                s.Lx, s.Ly, np.ascontiguousarray(s.desired_velocity), s.fstar, lam, s.dx, s.dy,
                s.Larea, s.ny, s.nx, cfg.delta_type)
            if cfg.motion_type is None:
                s.lambda_cache = lam
            s.ro, s.U = macroscopic(s.fstar, cfg.incompressible_lbgk)
        else:
            raise KeyError(cfg.ibm_method)

    # iblbm/ibm/multi_particle.py:347-421 (DF): each particle's closure
    # (ibm/forcing.py:125-275, CPU branch) on the same velocity field, its
    # Eulerian force added to the total in particle order; the particle's force
    # and torque are the negated Lagrangian sums -sum(Lf ds) and
    # -sum((rx Lfy - ry Lfx) ds), rx = (Lx - cx) / dx; then the velocity
    # correction with the total (ibm/dispatch.py:43-53)
    def _apply_df_multi(self):
        s, cfg = self.s, self.cfg
        Eux, Euy = np.ascontiguousarray(s.U[:, 0]), np.ascontiguousarray(s.U[:, 1])
        fib_total = np.zeros((s.nx * s.ny, 2))
        for particle in s.particles:
            La = float(particle.Larea)
            fib_p, _, _, Lfx, Lfy, _ = ibm_df(
                np.ascontiguousarray(particle.Lx), np.ascontiguousarray(particle.Ly),
                np.ascontiguousarray(particle.desired_velocity), Eux, Euy, s.ro, s.dx, s.dy, s.dt, La, s.ny,
                s.nx, cfg.delta_type, cfg.incompressible_lbgk)
            fib_total += fib_p
            particle._fib_force = np.array([-float(np.sum(Lfx * La)), -float(np.sum(Lfy * La))])
            if cfg.enable_rotation:
                rx = (particle.Lx - float(particle.pos[0])) / s.dx
                ry = (particle.Ly - float(particle.pos[1])) / s.dy
                particle._torque_new = -float(np.sum((rx * Lfy - ry * Lfx) * La))
        s.fib = fib_total
        velocity_correction(s.U, s.fib, s.ro, s.dt, cfg.incompressible_lbgk)

    # iblbm/ibm/strategies/dfc.py:56-128 (DFC, apply_multi): every particle's markers as
    # one point set (equal arc lengths required), lambda of that set each step, one
    # correction, the moments again; a particle's force and torque are the sums of
    # its markers' Lagrangian forces and of rx Fy - ry Fx, rx = (Lx - cx) / dx
    def _apply_dfc_multi(self):
        s, cfg = self.s, self.cfg
        La = float(s.particles[0].Larea)
        if any(abs(float(p.Larea) - La) > 1e-12 for p in s.particles):
            raise ValueError("multi-particle DFC needs equal marker arc lengths")
        Lx = np.ascontiguousarray(np.concatenate([p.Lx for p in s.particles]))
        Ly = np.ascontiguousarray(np.concatenate([p.Ly for p in s.particles]))
        dv = np.ascontiguousarray(np.concatenate([p.desired_velocity for p in s.particles]))
        lam = dfc_lambda(Lx, Ly, La, s.dx, s.dy, s.ny, s.nx, cfg.delta_type)
        s.fstar, s.dfc_force_lagr = dfc_correction(Lx, Ly, dv, s.fstar, lam, s.dx, s.dy, La, s.ny, s.nx,
                                                   cfg.delta_type)
        s.ro, s.U = macroscopic(s.fstar, cfg.incompressible_lbgk)
        start = 0
        for particle in s.particles:
            end = start + len(particle.Lx)
            fl = s.dfc_force_lagr[start:end]
            particle._fib_force = np.array([float(fl[:, 0].sum()), float(fl[:, 1].sum())])
            if cfg.enable_rotation:
                rx = (np.asarray(particle.Lx) - float(particle.pos[0])) / s.dx
                ry = (np.asarray(particle.Ly) - float(particle.pos[1])) / s.dy
                particle._torque_new = float(np.sum(rx * fl[:, 1] - ry * fl[:, 0]))
            start = end

    # iblbm/ibm/multi_particle.py:424-455 (MDF) and 347-421 (DF, uncoupled)
    def _apply_ibm_multi(self):
        s, cfg = self.s, self.cfg
        if cfg.ibm_method == "DF":
            return self._apply_df_multi()
        if cfg.ibm_method == "DFC":
            return self._apply_dfc_multi()
        if cfg.ibm_method != "MDF" or len(s.particles) < 2:
            raise NotImplementedError("multi-particle oracle covers DF and coupled MDF")
        parts = [(np.ascontiguousarray(p.Lx), np.ascontiguousarray(p.Ly),
                  np.ascontiguousarray(p.desired_velocity), p.Larea) for p in s.particles]
        fib, fpart, stats = mdf_coupled(parts, s.U, s.ro, s.dx, s.dy, s.dt, s.ny, s.nx,
                                        cfg.mdf_iterations, cfg.mdf_min_iterations, cfg.delta_type,
                                        s.mdf_omega, cfg.mdf_tolerance, cfg.incompressible_lbgk)
        s.fib = fib
        s.mdf_stats = stats
        for p, particle in enumerate(s.particles):
            fp = fpart[p]
            particle._fib_force = np.array([-float(fp[:, 0].sum()), -float(fp[:, 1].sum())])
            if cfg.enable_rotation:
                # iblbm/ibm/multi_particle.py:203-208: T = -sum((i - cx) fy - (j - cy) fx)
                # over the lattice, node indices as floats, centre in lattice units
                II, JJ = np.meshgrid(np.arange(s.nx, dtype=float), np.arange(s.ny, dtype=float), indexing="xy")
                cx_lat = float(particle.pos[0]) / s.dx
                cy_lat = float(particle.pos[1]) / s.dy
                fx = np.ascontiguousarray(fp[:, 0]).reshape(s.ny, s.nx)
                fy = np.ascontiguousarray(fp[:, 1]).reshape(s.ny, s.nx)
                particle._torque_new = -float(np.sum((II - cx_lat) * fy - (JJ - cy_lat) * fx))
        velocity_correction(s.U, s.fib, s.ro, s.dt, cfg.incompressible_lbgk)

    # runtime/scenarios/sedimentation_multi.py:36-80 (Verlet half step; with rotation
    # the half kick of iblbm/physics/rigid_body.py:65-74, markers turned by the
    # angle, and for semi-implicit coupling the desired velocity U + omega x r of
    # iblbm/physics/markers.py:41-60 with the angular velocity of the last step)
    def _half_step(self):
        s, cfg = self.s, self.cfg
        rot = cfg.enable_rotation
        for p in s.particles:
            F = p.force + _net_gravity(p.rho_ratio, p.lattice_r, s.gravity_lattice, cfg.gravity_direction)
            hist = _history_dv(cfg.settling_inertia_model, p.vel, p.vel_prev, p.mass, p.lattice_r)
            vel_half = p.vel + 0.5 * s.dt * F / p.mass
            if hist is not None:
                vel_half = vel_half + 0.5 * hist
            p.pos = p.pos + s.dt * vel_half * s.dx
            if rot:
                omega_half = p.omega + 0.5 * s.dt * p.torque / p.I_particle
                p.angle += s.dt * omega_half
                p._omega_half = omega_half
            p.Lx, p.Ly = _update_markers(p.Lx_c, p.Ly_c, p.cx_init, p.cy_init, p.pos, angle=p.angle if rot else 0.0)
            dv = np.empty((p.Lb, 2))
            dv[:, 0] = float(vel_half[0])
            dv[:, 1] = float(vel_half[1])
            if rot and cfg.rotation_coupling == "semi_implicit" and p.omega != 0.0:
                dv[:, 0] += -p.omega * (p.Ly - float(p.pos[1])) / s.dx
                dv[:, 1] += p.omega * (p.Lx - float(p.pos[0])) / s.dx
            p.desired_velocity = dv
            p._vel_half = vel_half

    # runtime/scenarios/sedimentation_multi.py:83-111
    def _full_step(self):
        s, cfg = self.s, self.cfg
        for p in s.particles:
            F = p._fib_force + _net_gravity(p.rho_ratio, p.lattice_r, s.gravity_lattice,
                                            cfg.gravity_direction)
            vel_new = p._vel_half + 0.5 * s.dt * F / p.mass
            hist = _history_dv(cfg.settling_inertia_model, p.vel, p.vel_prev, p.mass, p.lattice_r)
            if hist is not None:
                vel_new = vel_new + 0.5 * hist
            if cfg.settling_inertia_model == "feng_b2":
                vel_new = vel_new + (1.0 / p.rho_ratio) * (p.vel - p.vel_prev)
            if cfg.enable_rotation:  # iblbm/physics/rigid_body.py:77-82
                p.omega = p._omega_half + 0.5 * s.dt * p._torque_new / p.I_particle
                p.torque = p._torque_new
            p.vel_prev = p.vel.copy()
            p.vel = vel_new
            p.force = p._fib_force

    # runtime/scenarios/sedimentation_multi.py:126-190: explicit Euler after the IB step
    # (iblbm/physics/inertia/{none,explicit_history}.py euler_explicit,
    # iblbm/physics/rigid_body.py:84-98 position update, feng_b2 post-correction); with
    # rotation the angular step of rigid_body.py:101-121 with the change of the fluid's
    # angular momentum inside the disc (diagnostics/internal_flow.py:220-262); then the
    # markers and desired velocity (U + omega x r) of the next step
    def _euler_step(self):
        s, cfg = self.s, self.cfg
        rot = cfg.enable_rotation
        for p in s.particles:
            if rot:
                l_now = _l_int_z(s.U, s.ro, s.nx, s.ny, s.dx, float(p.pos[0]), float(p.pos[1]), p.r_domain)
                dl = l_now - p.l_int_prev
                p.l_int_prev = l_now
                omega_new = p.omega + (dl + s.dt * p._torque_new) / p.I_particle
                if cfg.sedimentation_euler_update_scheme == "trapezoidal":
                    p.angle += 0.5 * s.dt * (p.omega + omega_new)
                else:
                    p.angle += s.dt * omega_new
                p.torque = p._torque_new
                p.omega = omega_new
            F = p._fib_force + _net_gravity(p.rho_ratio, p.lattice_r, s.gravity_lattice, cfg.gravity_direction)
            vel_new = p.vel + s.dt * F / p.mass
            hist = _history_dv(cfg.settling_inertia_model, p.vel, p.vel_prev, p.mass, p.lattice_r)
            if hist is not None:
                vel_new = vel_new + hist
            if cfg.sedimentation_euler_update_scheme == "trapezoidal":
                pos_new = p.pos + 0.5 * s.dt * (p.vel + vel_new) * s.dx
            else:
                pos_new = p.pos + s.dt * vel_new * s.dx
            if cfg.settling_inertia_model == "feng_b2":
                vel_new = vel_new + (1.0 / p.rho_ratio) * (p.vel - p.vel_prev)
            p.vel_prev = p.vel.copy()
            p.vel = vel_new
            p.pos = pos_new
            p.force = p._fib_force
            p.Lx, p.Ly = _update_markers(p.Lx_c, p.Ly_c, p.cx_init, p.cy_init, pos_new, angle=p.angle if rot else 0.0)
            dv = np.empty((p.Lb, 2))
            dv[:, 0] = float(vel_new[0])
            dv[:, 1] = float(vel_new[1])
            if rot and p.omega != 0.0:
                dv[:, 0] += -p.omega * (p.Ly - float(pos_new[1])) / s.dx
                dv[:, 1] += p.omega * (p.Lx - float(pos_new[0])) / s.dx
            p.desired_velocity = dv

    def cd_cl(self):
        """iblbm/diagnostics/core.py:53-113 via the strategies' compute_cd_cl."""
        s, cfg = self.s, self.cfg
        u_ref = cfg.lattice_u if cfg.motion_type == "oscillating" else s.in_u
        if cfg.ibm_method == "DFC":
            total = np.sum(s.dfc_force_lagr, axis=0)
            denom = float(s.ro.mean()) * u_ref ** 2 * s.lattice_r
            return float(np.abs(total[0])) / denom, float(total[1]) / denom
        denom = np.mean(s.ro) * u_ref ** 2 * s.lattice_r
        return float(np.abs(np.sum(s.fib[:, 0])) / denom), float(np.sum(s.fib[:, 1]) / denom)

    def step(self):
        """One iteration of iblbm/runtime/loop.py:63-138 (without the stop checks)."""
        s, cfg, ttt = self.s, self.cfg, self.ttt
        if cfg.scenario_type == "taylor_green" and cfg.tg_with_ibm:
            # iblbm/runtime/scenarios/taylor_green.py:21-31 (pre_step): analytic desired velocity
            L_lat, nu = tg_params(cfg)
            ux, uy = tg_velocity(s.Lx / s.dx - (s.nx - 1) / 2.0, s.Ly / s.dy - (s.ny - 1) / 2.0, ttt * s.dt,
                                 cfg.tg_u0, L_lat, nu)
            s.desired_velocity[:, 0] = ux
            s.desired_velocity[:, 1] = uy
        if s.particles is not None and cfg.time_integrator != "euler_explicit":
            self._half_step()
        if not cfg.stream_first and not self.force_level:
            self.f = self.collide()
        self.stream_boundary_macro()
        self.apply_ibm()
        if s.particles is not None:
            if cfg.time_integrator == "euler_explicit":
                self._euler_step()
            else:
                self._full_step()
        s.feq = feq(s.ro, s.U, cfg.incompressible_lbgk)
        if cfg.stream_first or self.force_level:
            self.f = self.collide()
        if cfg.motion_type == "oscillating":
            # iblbm/physics/motion.py:15-52 (desired velocity = displacement)
            f0 = cfg.lattice_u / (cfg.KC * 2.0 * s.lattice_r)
            A = cfg.KC * 2.0 * s.r / (2.0 * np.pi)
            xt = A * np.sin(f0 * 2.0 * np.pi * ttt)
            s.Lx = np.ascontiguousarray(self.Lx_c - xt)
            s.Ly = self.Ly_c.copy()
            s.desired_velocity[:, 0] = xt
            s.desired_velocity[:, 1] = 0.0
        if ttt % cfg.check_interval == 0:
            if s.particles is not None:
                self.history.append([(p.pos.copy(), p.vel.copy()) for p in s.particles])
                self.Cd_history.append(0.0)
                self.Cl_history.append(0.0)
            elif cfg.scenario_type == "taylor_green" and not cfg.tg_with_ibm:
                self.Cd_history.append(0.0)  # iblbm/runtime/scenarios/taylor_green.py:60-62
                self.Cl_history.append(0.0)
            else:
                with np.errstate(divide="ignore", invalid="ignore"):  # no inflow: u_ref = 0
                    Cd, Cl = self.cd_cl()
                self.Cd_history.append(Cd)
                self.Cl_history.append(Cl)
        self.ttt += 1

    def run(self, max_steps=None):
        steps = self.cfg.max_steps if max_steps is None else max_steps
        while self.ttt <= steps:
            self.step()
        return {"Cd_history": np.array(self.Cd_history), "Cl_history": np.array(self.Cl_history),
                "state": self.s, "final_step": self.ttt - 1}


def run(cfg, max_steps=None):
    return OracleSim(cfg).run(max_steps)


def collide_post(sim):
    """Post-collision populations of the last completed step (force-level schedule)."""
    return sim.f


__all__ = ["OracleSim", "run", "init_state", "mdf_omega", "math"]
