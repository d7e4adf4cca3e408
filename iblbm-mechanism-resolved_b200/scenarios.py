"""Scenario configuration builders of the reference (its top-level
``scenarios`` package), returning this package's ``SimConfig``.

``make_tg_config`` follows scenarios/taylor_green.py:16-85: the decaying
Taylor-Green vortex on [-L, L]^2 with L = D lattice nodes (NN = 2 D + 1,
the vortex's half-width equal to the "cylinder" diameter D = 0.5 (NN - 1)),
u0 = 0.04, Re = u0 D / nu = 10, measured after one convective time D / u0
(rounded to whole steps).  With ``use_ibm`` the marker ring of diameter D
carries the analytic velocity each step.
"""
from __future__ import annotations

from .config import SimConfig

TG_U0 = 0.04
TG_RE = 10.0


def make_tg_config(D_over_dx: int, use_ibm: bool = False, *, ibm_method: str = "DF",
                   delta_type: str = "peskin4pt", collision_model: str = "BGK") -> SimConfig:
    """Taylor-Green case with D_over_dx lattice nodes per half-width."""
    NN = 2 * int(D_over_dx) + 1
    lattice_D = 0.5 * (NN - 1)
    T = lattice_D / TG_U0  # one convective time, in steps
    steps = int(round(T))
    return SimConfig(Re=TG_RE, NN=NN, xmax=1.0, ymax=1.0, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.5,
                     lattice_u=TG_U0, inflow_u=TG_U0, bc_type="velocity_inlet", ibm_method=ibm_method,
                     delta_type=delta_type, collision_model=collision_model, max_steps=steps,
                     convergence_threshold=1e-10, convergence_start=steps, check_interval=max(1, int(T) // 10),
                     use_convergence=False, marker_spacing_factor=1.0, nx_formula="standard",
                     scenario_type="taylor_green", tg_L=1.0, tg_u0=TG_U0, tg_T_end=T, tg_with_ibm=use_ibm)
