"""Simulation configuration with the reference's field names and defaults.

The dataclass mirrors ``SimConfig`` of iblbm/config.py:21-124 field for field so a
configuration built for the reference (its scenario builders, experiment
runners or a saved dict) drives this package unchanged.  Validation follows
iblbm/config.py:126-170 and the tau warning iblbm/config.py:172-196.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class SimConfig:
    # geometry and flow (lattice units unless stated; coordinates are domain fractions)
    Re: float
    NN: int
    xmax: float = 1.0
    ymax: float = 1.0
    cylinder_center: tuple[float, float] = (0.4, 0.5)
    cylinder_D_ratio: float = 1 / 40
    lattice_u: float = 0.1
    inflow_u: float = 0.1
    bc_type: str = "velocity_inlet"
    # immersed boundary
    delta_type: str = "peskin4pt"
    ibm_method: str = "DF"
    df_coupled: bool = False
    stream_first: bool = False
    mdf_iterations: int = 20
    mdf_min_iterations: int = 5
    mdf_tolerance: float = 1e-4
    # run control
    max_steps: int = 800_000
    convergence_threshold: float = 1e-5
    convergence_start: int = 100_000
    check_interval: int = 100
    use_convergence: bool = True
    cd_convergence_tol: float | None = None
    cd_convergence_window: int = 5
    cd_convergence_start_step: int = 20_000
    motion_type: str | None = None
    KC: float = 5.0
    # sedimentation
    rho_ratio: float = 1.0
    gravity: float = 0.0
    enable_rotation: bool = False
    retraction_dx: float = 0.0
    rotation_coupling: str = "indirect"
    prescribed_velocity: tuple[float, float] | None = None
    gravity_direction: str = "down"
    particles_config: list[dict] | None = None
    diagnostics_interval: int = 0
    settling_inertia_model: str = "unset"
    sedimentation_stop_at_contact: bool = False
    sedimentation_stop_offset_d: float = 0.0
    sedimentation_reference_basis: str = "standard"
    sedimentation_euler_update_scheme: str = "new_velocity"
    marker_spacing_factor: float = 0.5
    nx_formula: str = "standard"
    use_gpu: bool = False
    time_integrator: str = "verlet"
    incompressible_lbgk: bool = False
    # collision operator
    collision_model: str = "BGK"
    trt_magic_param: float = 0.25
    mrt_s_e: float | None = None
    mrt_s_eps: float | None = None
    mrt_s_q: float | None = None
    # Taylor-Green vortex
    scenario_type: str | None = None
    tg_L: float = 1.0
    tg_u0: float = 0.1
    tg_T_end: float | None = None
    tg_with_ibm: bool = False
    # physical units (conversion only)
    phy_u: float = 1e-3
    phy_l: float = 1e-3
    phy_density: float = 1000

    def __post_init__(self) -> None:
        if self.scenario_type not in (None, "taylor_green"):
            raise ValueError(f"scenario_type='{self.scenario_type}' is not supported "
                             "(allowed: 'taylor_green' or None)")
        if self.mdf_iterations < 1:
            raise ValueError("mdf_iterations must be >= 1")
        if self.mdf_min_iterations < 1:
            raise ValueError("mdf_min_iterations must be >= 1")
        if self.mdf_tolerance <= 0.0:
            raise ValueError("mdf_tolerance must be positive")
        if self.motion_type == "sedimentation":
            models = {"unset", "none", "explicit_history", "feng_b2", "full_volume"}
            if self.settling_inertia_model not in models:
                raise ValueError(f"settling_inertia_model='{self.settling_inertia_model}' is not "
                                 f"supported (allowed: {sorted(models)})")
            if self.settling_inertia_model == "unset":
                raise ValueError("Sedimentation benchmark requires explicit settling_inertia_model")
            if self.sedimentation_stop_at_contact and self.sedimentation_stop_offset_d > 0.0:
                raise ValueError("contact and offset stop rules are mutually exclusive")
            if self.sedimentation_reference_basis not in ("standard", "particle_basis"):
                raise ValueError("sedimentation_reference_basis must be 'standard' or 'particle_basis'")
            if self.sedimentation_euler_update_scheme not in ("new_velocity", "trapezoidal"):
                raise ValueError("sedimentation_euler_update_scheme must be 'new_velocity' or 'trapezoidal'")

    def warn_if_unstable(self) -> str | None:
        """Warn when tau = 3 nu + 1/2 approaches 1/2 (0.55 for BGK/TRT, 0.52 for CM-MRT)."""
        lattice_D = self.cylinder_D_ratio * (self.NN - 1)
        tau = 3.0 * (self.lattice_u * lattice_D / self.Re) + 0.5
        if self.collision_model == "CM_MRT":
            if tau < 0.52:
                return (f"tau={tau:.4f} < 0.52: CM_MRT may be unstable; raise NN or lower Re "
                        f"(NN={self.NN}, Re={self.Re}).")
        elif tau < 0.55:
            nn_min = int(0.6 * self.Re / (3.0 * self.lattice_u * self.cylinder_D_ratio) + 1)
            return (f"tau={tau:.4f} < 0.55: {self.collision_model}-LBM may be unstable; raise NN "
                    f"or lower Re (NN={self.NN}, Re={self.Re}). NN >= {nn_min} recommended.")
        return None
