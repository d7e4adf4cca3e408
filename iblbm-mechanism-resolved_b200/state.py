"""Initial state of a run — the host-side setup of iblbm/init.py:116-265.

Grid sizes, relaxation times and the Lagrangian markers are computed on the
host with the reference's formulas (numpy FP64, so marker coordinates are
bit-identical to the reference's); the populations are built on the GPU by the
engine.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .physics import circle_markers


@dataclass
class Particle:
    """One rigid disc of a sedimentation run (iblbm/physics/sedimentation.py:47-90)."""
    pos: np.ndarray
    vel: np.ndarray
    vel_prev: np.ndarray
    force: np.ndarray
    mass: float
    rho_ratio: float
    lattice_r: float
    r_domain: float
    I_particle: float
    Lx_c: np.ndarray
    Ly_c: np.ndarray
    Lx: np.ndarray
    Ly: np.ndarray
    Lb: int
    Larea: float
    desired_velocity: np.ndarray
    cx_init: float
    cy_init: float
    fib_force: np.ndarray = field(default_factory=lambda: np.zeros(2))
    vel_half: np.ndarray = field(default_factory=lambda: np.zeros(2))
    # rotation (enable_rotation): angular velocity, last torque, turned angle
    omega: float = 0.0
    torque: float = 0.0
    angle: float = 0.0
    omega_half: float = 0.0
    l_int_prev: float = 0.0  # fluid angular momentum inside the disc at the last Euler step


@dataclass
class HostState:
    nx: int
    ny: int
    nodenums: int
    dx: float
    dy: float
    dt: float
    tau: float
    r: float
    lattice_r: float
    in_u: float
    dens: float
    Lx: np.ndarray
    Ly: np.ndarray
    Lb: int
    Larea: float
    desired_velocity: np.ndarray
    tau_minus: float | None = None
    S_diag: np.ndarray | None = None
    gravity_lattice: float = 0.0
    particles: list | None = None
    # filled by the engine when results are read back
    ro: np.ndarray | None = None
    U: np.ndarray | None = None
    fib: np.ndarray | None = None
    fstar: np.ndarray | None = None
    feq: np.ndarray | None = None
    dfc_force_lagr: np.ndarray | None = None
    mdf_iter_stats: dict | None = None


def grid_shape(cfg):
    """nx, ny, dx, dy — iblbm/init.py:133-152."""
    if cfg.nx_formula == "standard":
        nx = int(cfg.NN * cfg.xmax - (cfg.xmax - 1))
    else:
        nx = int(cfg.NN * cfg.xmax)
    dx = 1.0 / (cfg.NN - 1)
    ny = round(cfg.ymax / dx) + 1
    dy = cfg.ymax / (ny - 1)
    if abs(dx - dy) / dx > 1e-6:
        raise ValueError(f"non-square lattice: dx={dx:.8f}, dy={dy:.8f}; ymax={cfg.ymax} is incompatible with dx")
    return nx, ny, dx, dy


def initialize(cfg) -> HostState:
    nx, ny, dx, dy = grid_shape(cfg)
    phy_char = cfg.phy_l * cfg.cylinder_D_ratio
    cell = (cfg.phy_l / (cfg.NN - 1)) / 1.0
    r = phy_char / 2.0 / cfg.phy_l
    lattice_r = (phy_char / cell) / 2.0
    tau = 3.0 * (cfg.lattice_u * 2.0 * lattice_r / cfg.Re) + 0.5
    cx, cy = cfg.cylinder_center
    if cx - r < 0 or cx + r > cfg.xmax or cy - r < 0 or cy + r > cfg.ymax:
        raise ValueError(f"cylinder (cx={cx}, cy={cy}, r={r}) lies outside [0,{cfg.xmax}]x[0,{cfg.ymax}]")
    if cfg.retraction_dx < 0.0 or cfg.retraction_dx >= lattice_r:
        raise ValueError(f"retraction_dx={cfg.retraction_dx} outside [0, lattice_r={lattice_r})")
    Lx, Ly, Lb, Larea = circle_markers(cx, cy, r, lattice_r, dx, cfg.marker_spacing_factor, cfg.retraction_dx)
    st = HostState(nx=nx, ny=ny, nodenums=nx * ny, dx=dx, dy=dy, dt=1.0, tau=tau, r=r, lattice_r=lattice_r,
                   in_u=cfg.inflow_u, dens=1.0, Lx=Lx, Ly=Ly, Lb=Lb, Larea=Larea,
                   desired_velocity=np.zeros((Lb, 2)))
    if cfg.collision_model == "TRT":
        st.tau_minus = 0.5 + cfg.trt_magic_param / (tau - 0.5)  # lbm/collision/trt.py:73-75
    elif cfg.collision_model == "CM_MRT":
        s_eps = cfg.mrt_s_eps if cfg.mrt_s_eps is not None else 1.4
        s_q = cfg.mrt_s_q if cfg.mrt_s_q is not None else 1.2
        s_nu = 1.0 / tau
        st.S_diag = np.array([0.0, 0.0, 0.0, s_nu, s_nu, s_nu, s_q, s_q, s_eps])  # cm_mrt.py:171-188
    elif cfg.collision_model != "BGK":
        raise KeyError(f"unknown collision_model='{cfg.collision_model}' (BGK, TRT, CM_MRT)")
    if cfg.motion_type == "sedimentation":
        if cfg.gravity <= 0.0:
            raise ValueError(f"sedimentation needs gravity > 0 (got {cfg.gravity})")
        if cfg.rho_ratio <= 1.0:
            raise ValueError(f"sedimentation needs rho_ratio > 1.0 (got {cfg.rho_ratio})")
        st.gravity_lattice = cfg.gravity
        if cfg.particles_config is not None:
            parts = []
            for pc in cfg.particles_config:
                pcx, pcy = pc["center"]
                rho_p = pc["rho_ratio"]
                mass = rho_p * np.pi * lattice_r ** 2
                plx, ply, plb, pla = circle_markers(pcx, pcy, r, lattice_r, dx, cfg.marker_spacing_factor,
                                                    cfg.retraction_dx)
                parts.append(Particle(pos=np.array([pcx, pcy], dtype=float), vel=np.zeros(2),
                                      vel_prev=np.zeros(2), force=np.zeros(2), mass=mass, rho_ratio=rho_p,
                                      lattice_r=lattice_r, r_domain=r, I_particle=0.5 * mass * lattice_r ** 2,
                                      Lx_c=plx.copy(), Ly_c=ply.copy(), Lx=plx, Ly=ply, Lb=plb, Larea=pla,
                                      desired_velocity=np.zeros((plb, 2)), cx_init=pcx, cy_init=pcy))
            st.particles = parts
    return st


def initial_velocity(cfg, nodenums):
    """U at t = 0 — iblbm/init.py:168-201: the Taylor-Green vortex at t = 0 on
    centred lattice coordinates, (inflow_u, 0) for fixed bodies, rest otherwise."""
    U = np.zeros((nodenums, 2))
    if cfg.scenario_type == "taylor_green":
        from .physics import tg_base, tg_params
        nx, ny, _, _ = grid_shape(cfg)
        L, _ = tg_params(cfg)
        XX, YY = np.meshgrid(np.arange(nx, dtype=float) - (nx - 1) / 2.0, np.arange(ny, dtype=float) - (ny - 1) / 2.0)
        ux, uy = tg_base(XX.ravel(), YY.ravel(), cfg.tg_u0, L)
        U[:, 0], U[:, 1] = ux * 1.0, uy * 1.0  # decay factor exp(-0.0) = 1 at t = 0
    elif cfg.motion_type not in ("oscillating", "sedimentation"):
        U[:, 0] = cfg.inflow_u
    return U
