"""Scenario configuration builders of the reference (its top-level
``scenarios`` package), returning this package's ``SimConfig``.

``make_tg_config`` follows scenarios/taylor_green.py:16-85: the decaying
Taylor-Green vortex on [-L, L]^2 with L = D lattice nodes (NN = 2 D + 1,
the vortex's half-width equal to the "cylinder" diameter D = 0.5 (NN - 1)),
u0 = 0.04, Re = u0 D / nu = 10, measured after one convective time D / u0
(rounded to whole steps).  With ``use_ibm`` the marker ring of diameter D
carries the analytic velocity each step.

``make_dirichlet_neumann_fixed_cylinder_config`` follows scenarios/steady.py:
14-81 (fixed cylinder, D = (NN - 1) / 40, Re 20 / 40 / 100 / 200 with the
reference's default lattices and step counts), and
``make_oscillating_cylinder_config`` scenarios/oscillating.py:12-45 (in-line
oscillating cylinder in quiescent fluid, Re 100, KC 5 by default).
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


# Re -> (xmax, default NN, default max_steps) of the fixed-cylinder family
_FIXED = {20.0: (1.0, 1601, 100_000), 40.0: (1.0, 1601, 100_000), 100.0: (1.25, 1601, 100_000),
          200.0: (1.25, 2401, 60_000)}


def make_dirichlet_neumann_fixed_cylinder_config(*, reynolds: float = 40.0, ibm_method: str = "DF",
                                                 delta_type: str = "hat", collision_model: str = "BGK",
                                                 max_steps: int | None = None, mdf_iterations: int | None = None,
                                                 mdf_min_iterations: int | None = None,
                                                 nn: int | None = None) -> SimConfig:
    """Fixed cylinder in the Dirichlet-Neumann channel.  MDF takes 5-20
    iterations unless given; the other methods one.  Unsupported Reynolds
    numbers raise ValueError."""
    re = float(reynolds)
    if re not in _FIXED:
        raise ValueError(f"Unsupported fixed-cylinder Reynolds number: {re}. Allowed: 20, 40, 100, 200.")
    xmax, nn0, steps0 = _FIXED[re]
    mdf = ibm_method == "MDF"
    return SimConfig(Re=re, NN=nn0 if nn is None else int(nn), xmax=xmax, ymax=1.0, cylinder_center=(0.5, 0.5),
                     cylinder_D_ratio=1.0 / 40.0, lattice_u=0.1, inflow_u=0.1, bc_type="dirichlet_neumann",
                     delta_type=delta_type, ibm_method=ibm_method, collision_model=collision_model,
                     mdf_iterations=(20 if mdf_iterations is None else int(mdf_iterations)) if mdf else 1,
                     mdf_min_iterations=(5 if mdf_min_iterations is None else int(mdf_min_iterations)) if mdf else 1,
                     max_steps=steps0 if max_steps is None else int(max_steps), check_interval=200,
                     use_convergence=False, cd_convergence_tol=1e-4, cd_convergence_window=5,
                     cd_convergence_start_step=20_000, marker_spacing_factor=2.0 / 3.0, nx_formula="standard")


def make_oscillating_cylinder_config(*, reynolds: float = 100.0, kc: float = 5.0, ibm_method: str = "DF",
                                     delta_type: str = "peskin4pt", collision_model: str = "BGK", nn: int = 1601,
                                     max_steps: int = 40_000) -> SimConfig:
    """In-line oscillating cylinder (D = (NN - 1) / 20) in an open box."""
    mdf = ibm_method == "MDF"
    return SimConfig(Re=float(reynolds), NN=int(nn), xmax=1.5, ymax=1.0, cylinder_center=(0.75, 0.5),
                     cylinder_D_ratio=1.0 / 20.0, lattice_u=0.1, inflow_u=0.0, bc_type="open_boundary",
                     delta_type=delta_type, ibm_method=ibm_method, collision_model=collision_model,
                     mdf_iterations=20 if mdf else 1, mdf_min_iterations=5 if mdf else 1, max_steps=int(max_steps),
                     check_interval=50, use_convergence=False, motion_type="oscillating", KC=float(kc),
                     marker_spacing_factor=2.0 / 3.0, nx_formula="simple")
