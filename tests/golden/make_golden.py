"""Generate the golden fixtures in this folder by running the reference solver.

The reference (mulgae-life/iblbm-mechanism-resolved) is a Python package; its CPU
path (numba + numpy, selected with IBLBM_GPU=0) is imported from the read-only
checkout given by ``--reference`` and run on small inputs.  The fixtures pin the
CPU oracle in ``oracle/`` (tests/test_oracle_golden.py) and, through it, the CUDA
product path.

Three kinds of fixture are written:

* ``lambda_rho.npz`` — the reference's DFC lambda(k) for fluid densities 1.3
  and 0.7 on the marker inputs of units.npz;
* ``units.npz``   — seeded random inputs and the reference's outputs for every
  kernel on the hot path (feq, macroscopic, BGK/TRT/CM-MRT collision, streaming,
  the four boundary closures, velocity correction, DF, MDF, DFC lambda and
  correction, the MDF relaxation factor) plus the initial state that
  ``iblbm.init.initialize`` builds for each benchmark configuration.
* ``run_<case>.npz`` — short end-to-end runs of ``iblbm.run`` on small lattices:
  SHA-256 digests of the final rho/U/fib/fstar/feq arrays (bit-exact checks),
  a decimated sample of the same arrays (tolerance checks), and the Cd/Cl or
  particle histories.

Usage:  python tests/golden/make_golden.py --reference /path/to/reference
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SAMPLE_STRIDE = 97


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=np.float64)).tobytes()).hexdigest()


def _sample(a):
    a = np.asarray(a, dtype=np.float64)
    return a.reshape(a.shape[0], -1)[::SAMPLE_STRIDE].copy()


# Small end-to-end cases: each mirrors one benchmark configuration at reduced size.
RUN_CASES = {
    # fixed cylinder, config-1 geometry exactly (401 x 161, D = 20, 63 markers)
    "c1_df_bgk_hat": dict(Re=20, NN=161, xmax=2.5, ymax=1, cylinder_center=(0.625, 0.5),
                          cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.05,
                          bc_type="dirichlet_neumann", delta_type="hat", ibm_method="DF",
                          collision_model="BGK", marker_spacing_factor=1.0, max_steps=300,
                          use_convergence=False, check_interval=50),
    # config-2 method (MDF + P4, TRT magic 3/16, tol 1e-6) on a 401 x 161 lattice
    "c2_mdf_trt_p4": dict(Re=100, NN=161, xmax=2.5, ymax=1, cylinder_center=(0.5, 0.5),
                          cylinder_D_ratio=0.0625, lattice_u=0.04, inflow_u=0.04,
                          bc_type="dirichlet_neumann", delta_type="peskin4pt", ibm_method="MDF",
                          collision_model="TRT", trt_magic_param=0.1875, mdf_iterations=20,
                          mdf_min_iterations=5, mdf_tolerance=1e-6, marker_spacing_factor=1.0,
                          max_steps=200, use_convergence=False, check_interval=50),
    "c2_mdf_cmmrt_p4": dict(Re=100, NN=161, xmax=2.5, ymax=1, cylinder_center=(0.5, 0.5),
                            cylinder_D_ratio=0.0625, lattice_u=0.04, inflow_u=0.04,
                            bc_type="dirichlet_neumann", delta_type="peskin4pt", ibm_method="MDF",
                            collision_model="CM_MRT", mdf_iterations=20, mdf_min_iterations=5,
                            mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=200,
                            use_convergence=False, check_interval=50),
    # config-3 method (oscillating cylinder, open boundary, DFC + P4, BGK) on 161 x 161
    "c3_dfc_bgk_p4_osc": dict(Re=20, NN=161, xmax=1, ymax=1, cylinder_center=(0.5, 0.5),
                              cylinder_D_ratio=0.125, lattice_u=0.02, inflow_u=0.0,
                              bc_type="open_boundary", delta_type="peskin4pt", ibm_method="DFC",
                              collision_model="BGK", motion_type="oscillating", KC=5.0,
                              nx_formula="simple", marker_spacing_factor=1.0, max_steps=300,
                              use_convergence=False, check_interval=50),
    # config-5 method (two discs, settling channel, coupled MDF + P4, CM-MRT, Verlet);
    # density ratio 3 keeps the explicit particle coupling stable at D = 10
    "c5_sed2_mdf_cmmrt_p4": dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.5, 3.0),
                                 cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.0,
                                 bc_type="settling_channel", delta_type="peskin4pt",
                                 ibm_method="MDF", collision_model="CM_MRT",
                                 motion_type="sedimentation", rho_ratio=3.0, gravity=2e-5,
                                 particles_config=[{"center": (0.5, 3.4375), "rho_ratio": 3.0},
                                                   {"center": (0.50625, 3.1875), "rho_ratio": 3.0}],
                                 settling_inertia_model="explicit_history",
                                 mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                                 marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                                 check_interval=50),
    # two settling discs that also rotate (torque from the spread force, Verlet on the
    # angular velocity, markers turned by the angle); indirect and semi-implicit coupling
    "c5r_sed2_mdf_rot_indirect": dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.5, 3.0),
                                      cylinder_D_ratio=0.25, lattice_u=0.05, inflow_u=0.0,
                                      bc_type="settling_channel", delta_type="peskin4pt",
                                      ibm_method="MDF", collision_model="BGK",
                                      motion_type="sedimentation", rho_ratio=3.0, gravity=2e-5,
                                      particles_config=[{"center": (0.53, 3.4), "rho_ratio": 3.0},
                                                        {"center": (0.48, 2.9), "rho_ratio": 3.0}],
                                      settling_inertia_model="explicit_history", enable_rotation=True,
                                      mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                                      marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                                      check_interval=50),
    "c5r_sed2_mdf_rot_semi": dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.5, 3.0),
                                  cylinder_D_ratio=0.25, lattice_u=0.05, inflow_u=0.0,
                                  bc_type="settling_channel", delta_type="hat",
                                  ibm_method="MDF", collision_model="TRT",
                                  motion_type="sedimentation", rho_ratio=3.0, gravity=2e-5,
                                  particles_config=[{"center": (0.47, 3.4), "rho_ratio": 3.0},
                                                    {"center": (0.52, 2.9), "rho_ratio": 3.5}],
                                  settling_inertia_model="feng_b2", enable_rotation=True,
                                  rotation_coupling="semi_implicit",
                                  mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                                  marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                                  check_interval=50),
    # the multi-particle runtime adds omega x r only for semi-implicit coupling, so
    # iterative coupling steps like indirect there
    "c5r_sed2_mdf_rot_iterative": dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.5, 3.0),
                                       cylinder_D_ratio=0.25, lattice_u=0.05, inflow_u=0.0,
                                       bc_type="settling_channel", delta_type="peskin4pt",
                                       ibm_method="MDF", collision_model="CM_MRT",
                                       motion_type="sedimentation", rho_ratio=3.0, gravity=2e-5,
                                       particles_config=[{"center": (0.53, 3.4), "rho_ratio": 3.0},
                                                         {"center": (0.48, 2.9), "rho_ratio": 3.0}],
                                       settling_inertia_model="none", enable_rotation=True,
                                       rotation_coupling="iterative",
                                       mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                                       marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                                       check_interval=50),
    # explicit Euler integration of the settling discs (velocity then position after the
    # IB step; markers and desired velocity for the next step)
    "c5e_sed2_mdf_euler_none": dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.5, 3.0),
                                    cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.0,
                                    bc_type="settling_channel", delta_type="hat",
                                    ibm_method="MDF", collision_model="CM_MRT",
                                    motion_type="sedimentation", rho_ratio=3.0, gravity=2e-5,
                                    particles_config=[{"center": (0.5, 3.4375), "rho_ratio": 3.0},
                                                      {"center": (0.50625, 3.1875), "rho_ratio": 3.0}],
                                    settling_inertia_model="none", time_integrator="euler_explicit",
                                    mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                                    marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                                    check_interval=50),
    "c5e_sed2_mdf_euler_feng_trap": dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.5, 3.0),
                                         cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.0,
                                         bc_type="settling_channel", delta_type="hat",
                                         ibm_method="MDF", collision_model="BGK",
                                         motion_type="sedimentation", rho_ratio=3.0, gravity=2e-5,
                                         particles_config=[{"center": (0.48, 3.4375), "rho_ratio": 3.0},
                                                           {"center": (0.52, 3.1875), "rho_ratio": 2.5}],
                                         settling_inertia_model="feng_b2", time_integrator="euler_explicit",
                                         sedimentation_euler_update_scheme="trapezoidal",
                                         mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                                         marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                                         check_interval=50),
    "c5e_sed2_mdf_euler_rot": dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.5, 3.0),
                                   cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.0,
                                   bc_type="settling_channel", delta_type="hat",
                                   ibm_method="MDF", collision_model="CM_MRT",
                                   motion_type="sedimentation", rho_ratio=3.0, gravity=2e-5,
                                   particles_config=[{"center": (0.5, 3.4375), "rho_ratio": 3.0},
                                                     {"center": (0.50625, 3.1875), "rho_ratio": 3.0}],
                                   settling_inertia_model="none", time_integrator="euler_explicit",
                                   enable_rotation=True,
                                   mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                                   marker_spacing_factor=1.0, max_steps=300, use_convergence=False,
                                   check_interval=50),
    # default boundary family (velocity inlet / pressure outlet / no-slip walls), DF + P4
    "vin_df_bgk_p4": dict(Re=10, NN=81, xmax=2, ymax=1, cylinder_center=(0.5, 0.5),
                          cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.05,
                          bc_type="velocity_inlet", delta_type="peskin4pt", ibm_method="DF",
                          collision_model="BGK", marker_spacing_factor=1.0, max_steps=200,
                          use_convergence=False, check_interval=50),
    # fixed-body DFC (cached lambda), TRT + hat
    "dfc_trt_hat_fixed": dict(Re=40, NN=81, xmax=2, ymax=1, cylinder_center=(0.5, 0.5),
                              cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.05,
                              bc_type="dirichlet_neumann", delta_type="hat", ibm_method="DFC",
                              collision_model="TRT", marker_spacing_factor=1.0, max_steps=200,
                              use_convergence=False, check_interval=50),
    # Taylor-Green decaying vortex (scenario_type="taylor_green"): the analytic
    # time-dependent closure on all four faces; pure lattice Boltzmann (no IBM step)
    "tg_lbm_bgk": dict(Re=20, NN=41, xmax=1, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.25,
                       lattice_u=0.05, inflow_u=0.0, scenario_type="taylor_green", tg_u0=0.05,
                       tg_with_ibm=False, delta_type="hat", ibm_method="DF", collision_model="BGK",
                       marker_spacing_factor=1.0, max_steps=300, use_convergence=False, check_interval=50),
    "tg_lbm_cmmrt": dict(Re=20, NN=41, xmax=1, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.25,
                         lattice_u=0.05, inflow_u=0.0, scenario_type="taylor_green", tg_u0=0.05,
                         tg_with_ibm=False, delta_type="hat", ibm_method="MDF", collision_model="CM_MRT",
                         marker_spacing_factor=1.0, max_steps=300, use_convergence=False, check_interval=50),
    # ... and with the IBM step: markers driven to the analytic velocity every step
    "tg_ibm_mdf_trt_p4": dict(Re=20, NN=41, xmax=1, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.25,
                              lattice_u=0.05, inflow_u=0.0, scenario_type="taylor_green", tg_u0=0.05,
                              tg_with_ibm=True, delta_type="peskin4pt", ibm_method="MDF",
                              collision_model="TRT", trt_magic_param=0.1875, mdf_iterations=20,
                              mdf_min_iterations=5, mdf_tolerance=1e-6, marker_spacing_factor=1.0,
                              max_steps=300, use_convergence=False, check_interval=50),
    # incompressible LBGK branch (feq, macro, DF force law, velocity correction)
    "inc_df_bgk_hat": dict(Re=40, NN=81, xmax=2, ymax=1, cylinder_center=(0.5, 0.5),
                           cylinder_D_ratio=0.125, lattice_u=0.05, inflow_u=0.05,
                           bc_type="dirichlet_neumann", delta_type="hat", ibm_method="DF",
                           collision_model="BGK", incompressible_lbgk=True,
                           marker_spacing_factor=1.0, max_steps=200, use_convergence=False,
                           check_interval=50),
}

# Benchmark configurations whose initial state (grid, tau, markers) is pinned.
INIT_CASES = {
    "C1": dict(Re=20, NN=161, xmax=2.5, ymax=1, cylinder_center=(0.625, 0.5), cylinder_D_ratio=0.125,
               lattice_u=0.05, inflow_u=0.05, bc_type="dirichlet_neumann", delta_type="hat",
               ibm_method="DF", collision_model="BGK", marker_spacing_factor=1.0),
    "C2": dict(Re=100, NN=641, xmax=2.5, ymax=1, cylinder_center=(0.5, 0.5),
               cylinder_D_ratio=0.0625, lattice_u=0.04, inflow_u=0.04,
               bc_type="dirichlet_neumann", delta_type="peskin4pt", ibm_method="MDF",
               collision_model="TRT", trt_magic_param=0.1875, marker_spacing_factor=1.0),
    "C3": dict(Re=100, NN=1281, xmax=1, ymax=1, cylinder_center=(0.5, 0.5),
               cylinder_D_ratio=0.03125, lattice_u=0.02, inflow_u=0.0, bc_type="open_boundary",
               delta_type="peskin4pt", ibm_method="DFC", collision_model="BGK",
               motion_type="oscillating", KC=5.0, nx_formula="simple", marker_spacing_factor=1.0),
    "C5": dict(Re=20, NN=321, xmax=1, ymax=4, cylinder_center=(0.5, 3.4375), cylinder_D_ratio=0.125,
               lattice_u=0.05, inflow_u=0.0, bc_type="settling_channel", delta_type="peskin4pt",
               ibm_method="MDF", collision_model="CM_MRT", motion_type="sedimentation",
               rho_ratio=1.5, gravity=1e-5,
               particles_config=[{"center": (0.5, 1100 / 320), "rho_ratio": 1.5},
                                 {"center": (0.5 + 2 / 320, 1020 / 320), "rho_ratio": 1.5}],
               settling_inertia_model="explicit_history", marker_spacing_factor=1.0),
}

# the stream-first schedule (iblbm/runtime/loop.py:60-61,77,86-87: collide once
# before the loop, then at the end of every step) on the DFC cases, the one
# method whose default schedule collides at the start of the step
RUN_CASES["dfc_trt_hat_fixed_sf"] = dict(RUN_CASES["dfc_trt_hat_fixed"], stream_first=True)
RUN_CASES["c3_dfc_bgk_p4_osc_sf"] = dict(RUN_CASES["c3_dfc_bgk_p4_osc"], stream_first=True, max_steps=120)

# two settling discs under DF (iblbm/ibm/multi_particle.py:347-421): Lagrangian force and
# torque sums per particle; translation only, and with semi-implicit rotation
RUN_CASES["c5_sed2_df_bgk_hat"] = dict(RUN_CASES["c5_sed2_mdf_cmmrt_p4"], ibm_method="DF", delta_type="hat",
                                       collision_model="BGK", max_steps=200)
RUN_CASES["c5r_sed2_df_rot_semi"] = dict(RUN_CASES["c5r_sed2_mdf_rot_semi"], ibm_method="DF", max_steps=200)

# two settling discs under DFC (iblbm/ibm/strategies/dfc.py:56-128): one correction over
# both marker sets, per-particle Lagrangian force sums; translation only, and with
# semi-implicit rotation
RUN_CASES["c5_sed2_dfc_trt_p4"] = dict(RUN_CASES["c5_sed2_mdf_cmmrt_p4"], ibm_method="DFC", collision_model="TRT",
                                       max_steps=200)
RUN_CASES["c5r_sed2_dfc_rot_semi"] = dict(RUN_CASES["c5r_sed2_mdf_rot_semi"], ibm_method="DFC", max_steps=200)

# Single settling discs (iblbm/runtime/scenarios/sedimentation_single.py): the
# reference's single-particle runtime, whose state keeps the disc in
# particle_pos / particle_vel / ... instead of a particle list.  Written as
# sed1_<name>.npz: the engine is compared with them directly.
_SED1_BASE = dict(Re=20, NN=81, xmax=1, ymax=4, cylinder_center=(0.47, 3.0), cylinder_D_ratio=0.25,
                  lattice_u=0.05, inflow_u=0.0, bc_type="settling_channel", motion_type="sedimentation",
                  rho_ratio=1.5, gravity=2e-5, marker_spacing_factor=1.0, max_steps=240, use_convergence=False,
                  check_interval=40, mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6)
SINGLE_CASES = {
    # the layout of the bundled single-particle runs: DF + Peskin-4, BGK, explicit Euler, rotation
    "df_euler_rot": dict(_SED1_BASE, delta_type="peskin4pt", ibm_method="DF", collision_model="BGK",
                         settling_inertia_model="explicit_history", time_integrator="euler_explicit",
                         enable_rotation=True, rotation_coupling="indirect"),
    "mdf_verlet": dict(_SED1_BASE, delta_type="hat", ibm_method="MDF", collision_model="TRT",
                       trt_magic_param=0.1875, settling_inertia_model="none"),
    "dfc_verlet_semi_rot": dict(_SED1_BASE, delta_type="peskin4pt", ibm_method="DFC", collision_model="CM_MRT",
                                settling_inertia_model="feng_b2", enable_rotation=True,
                                rotation_coupling="semi_implicit"),
    "df_prescribed": dict(_SED1_BASE, delta_type="hat", ibm_method="DF", collision_model="BGK",
                          settling_inertia_model="none", prescribed_velocity=(0.0, -0.01)),
    # with the fluid-inside-the-disc diagnostics every other check
    "df_verlet_diag": dict(_SED1_BASE, delta_type="peskin4pt", ibm_method="DF", collision_model="TRT",
                           trt_magic_param=0.1875, settling_inertia_model="explicit_history",
                           diagnostics_interval=80),
}


def make_single(name, kw, out_dir):
    from iblbm import SimConfig, run
    res = run(SimConfig(**kw), verbose=False)
    st = res["state"]
    d = {"config_json": np.frombuffer(json.dumps(kw).encode(), dtype=np.uint8)}
    for k, a in {"ro": st.ro, "U": st.U, "fib": st.fib, "fstar": st.fstar, "feq": st.feq}.items():
        d[f"sha_{k}"] = np.frombuffer(bytes.fromhex(_sha(a)), dtype=np.uint8)
    d["particle"] = np.array([*st.particle_pos, *st.particle_vel, *st.particle_force])
    d["rotation"] = np.array([float(st.particle_omega), float(st.particle_angle), float(st.particle_torque)])
    d["history_json"] = np.frombuffer(json.dumps(res["sedimentation_history"]).encode(), dtype=np.uint8)
    d["final_step"] = np.array([res["final_step"]])
    d["termination"] = np.frombuffer(res["termination_reason"].encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(out_dir, f"sed1_{name}.npz"), **d)


def _import_reference(path):
    os.environ["IBLBM_GPU"] = "0"
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/iblbm_numba_cache")
    sys.dont_write_bytecode = True
    sys.path.insert(0, path)
    import iblbm  # noqa: F401
    return iblbm


def make_units(out):
    from iblbm.lbm import make_d2q9
    from iblbm.lbm.equilibrium import _compute_feq_nb
    from iblbm.lbm.macroscopic import _macroscopic_nb
    from iblbm.lbm.streaming import _streaming_step_nb
    from iblbm.lbm.collision.bgk import _collision_bgk_nb
    from iblbm.lbm.collision.trt import _collision_trt_nb
    from iblbm.lbm.collision.cm_mrt import _collision_cm_mrt_nb
    from iblbm.boundary import (apply_bc_dirichlet_neumann, apply_bc_open_boundary,
                                apply_bc_settling_channel, apply_bc_velocity_inlet,
                                build_boundary_indices)
    from iblbm.ibm.df import ibm_direct_forcing
    from iblbm.ibm.mdf import ibm_multi_direct_forcing
    from iblbm.ibm.dfc import apply_dfc_correction, compute_lambda
    from iblbm.ibm.a_norm import estimate_optimal_omega_from_type
    from iblbm.config import SimConfig
    from iblbm.init import initialize

    lat = make_d2q9()
    rng = np.random.default_rng(20261203)
    d = {}
    # dense per-node kernels on N random nodes
    N = 1024
    ro = 1.0 + rng.uniform(-0.02, 0.02, N)
    U = rng.uniform(-0.08, 0.08, (N, 2))
    fib = rng.uniform(-1e-3, 1e-3, (N, 2))
    fib[::3] = 0.0
    fstar = lat.w[None, :] * (1.0 + rng.uniform(-0.05, 0.05, (N, 9)))
    d["u_ro"], d["u_U"], d["u_fib"], d["u_fstar"] = ro, U, fib, fstar
    d["u_feq"] = _compute_feq_nb(ro, U, lat.e, lat.w, False)
    d["u_feq_inc"] = _compute_feq_nb(ro, U, lat.e, lat.w, True)
    feq = d["u_feq"]
    r_ro, r_U = _macroscopic_nb(fstar, lat.e, False)
    d["u_macro_ro"], d["u_macro_U"] = r_ro, r_U
    _, d["u_macro_U_inc"] = _macroscopic_nb(fstar, lat.e, True)
    tau = 0.548
    d["u_tau"] = np.array([tau])
    d["u_bgk"] = _collision_bgk_nb(fstar, feq, U, fib, tau, 1.0, lat.e, lat.w)
    tau_m = 0.5 + 0.1875 / (tau - 0.5)
    d["u_tau_minus"] = np.array([tau_m])
    d["u_trt"] = _collision_trt_nb(fstar, feq, U, fib, 1.0 / tau, 1.0 / tau_m, 1.0, lat.e, lat.w, lat.opp)
    S = np.array([0.0, 0.0, 0.0, 1 / tau, 1 / tau, 1 / tau, 1.2, 1.2, 1.4])
    d["u_S"] = S
    d["u_cmmrt"] = _collision_cm_mrt_nb(fstar, feq, U, fib, S, 1.0, lat.e, lat.w)
    # streaming + boundary closures on a 37 x 23 lattice
    nx, ny = 37, 23
    M = nx * ny
    d["g_nx"], d["g_ny"] = np.array([nx]), np.array([ny])
    fold = lat.w[None, :] * (1.0 + rng.uniform(-0.05, 0.05, (M, 9)))
    fpost = lat.w[None, :] * (1.0 + rng.uniform(-0.05, 0.05, (M, 9)))
    d["g_fold"], d["g_fpost"] = fold, fpost
    d["g_stream"] = _streaming_step_nb(fold, fpost, nx, ny)
    roM = 1.0 + rng.uniform(-0.01, 0.01, M)
    UM = rng.uniform(-0.05, 0.05, (M, 2))
    d["g_ro"], d["g_U"] = roM, UM
    for bc, fn in [("dirichlet_neumann", None), ("open_boundary", None),
                   ("settling_channel", None), ("velocity_inlet", None)]:
        cfg = SimConfig(Re=20, NN=23, bc_type=bc)
        idx = build_boundary_indices(cfg, nx, ny)
        fs = d["g_stream"].copy()
        r2 = roM.copy()
        u2 = UM.copy()
        if bc == "dirichlet_neumann":
            apply_bc_dirichlet_neumann(fs, r2, u2, 0.05, 1.0, idx, lat)
        elif bc == "open_boundary":
            apply_bc_open_boundary(fs, r2, u2, 1.0, idx, lat)
        elif bc == "settling_channel":
            apply_bc_settling_channel(fs, r2, u2, 1.0, idx, lat, incompressible=False)
        else:
            apply_bc_velocity_inlet(fs, r2, u2, 0.05, 1.0, idx, lat)
        d[f"bc_{bc}_f"], d[f"bc_{bc}_ro"], d[f"bc_{bc}_U"] = fs, r2, u2
    # IBM on a 48 x 40 field with a circle of markers (domain units, dx = 1/39)
    nx, ny = 48, 40
    dx = 1.0 / 39
    d["i_nx"], d["i_ny"], d["i_dx"] = np.array([nx]), np.array([ny]), np.array([dx])
    Ro = 1.0 + rng.uniform(-0.01, 0.01, (ny, nx))
    Eux = 0.04 + rng.uniform(-0.01, 0.01, (ny, nx))
    Euy = rng.uniform(-0.01, 0.01, (ny, nx))
    th = np.linspace(0, 2 * np.pi, 40, endpoint=False)
    Lx = 0.65 + 0.16 * np.cos(th)
    Ly = 0.5 + 0.16 * np.sin(th)
    Lx[0] = 0.999 * (nx - 1) * dx  # one marker at the right edge: clipped stencil
    dv = rng.uniform(-0.01, 0.01, (40, 2))
    Larea = 2 * np.pi * 0.16 / dx / 40
    d["i_Ro"], d["i_Eux"], d["i_Euy"], d["i_Lx"], d["i_Ly"], d["i_dv"] = Ro, Eux, Euy, Lx, Ly, dv
    d["i_Larea"] = np.array([Larea])
    for dt_name in ("hat", "peskin4pt"):
        for inc in (False, True):
            fibo, Lux, Luy, Lfx, Lfy, R = ibm_direct_forcing(Lx, Ly, dv, Eux, Euy, Ro, dx, dx, 1.0, Larea,
                                                             ny, nx, delta_type=dt_name, incompressible=inc)
            k = f"df_{dt_name}_{int(inc)}"
            d[k + "_fib"], d[k + "_Lux"], d[k + "_Luy"], d[k + "_Lfx"], d[k + "_R"] = fibo, Lux, Luy, Lfx, R
        Uf = np.stack([Eux.ravel(), Euy.ravel()], axis=1)
        om = estimate_optimal_omega_from_type(Lx, Ly, dt_name, Larea, dx)
        d[f"omega_{dt_name}"] = np.array([om])
        fibm, st = ibm_multi_direct_forcing(Lx, Ly, dv, Uf, Ro.ravel(), dx, dx, 1.0, Larea, ny, nx,
                                            n_iter=20, min_iter=5, delta_type=dt_name, omega=om, tol=1e-6)
        d[f"mdf_{dt_name}_fib"] = fibm
        d[f"mdf_{dt_name}_stats"] = np.array([st["iter_count"], st["last_residual"], st["diverged"],
                                              st["converged"]], dtype=np.float64)
        lam = compute_lambda(Lx, Ly, 1.0, Larea, dx, dx, ny, nx, dt_name)
        d[f"lam_{dt_name}"] = lam
        fs = lat.w[None, :] * (1.0 + rng.uniform(-0.05, 0.05, (nx * ny, 9)))
        d[f"dfc_{dt_name}_fstar"] = fs
        fc, force, _ = apply_dfc_correction(Lx, Ly, dv, fs, dx, dx, Larea, ny, nx, dt_name, lat,
                                            lambda_cache=lam)
        d[f"dfc_{dt_name}_fc"], d[f"dfc_{dt_name}_force"] = fc, force
    # initial states of the benchmark configurations
    for name, kw in INIT_CASES.items():
        st = initialize(SimConfig(**kw))
        d[f"init_{name}_scal"] = np.array([st.nx, st.ny, st.dx, st.dy, st.tau, st.Larea, st.lattice_r,
                                           st.r, st.Lb], dtype=np.float64)
        d[f"init_{name}_Lx"], d[f"init_{name}_Ly"] = np.asarray(st.Lx), np.asarray(st.Ly)
        if st.particles:
            for p, part in enumerate(st.particles):
                d[f"init_{name}_p{p}_Lx"], d[f"init_{name}_p{p}_Ly"] = part.Lx, part.Ly
                d[f"init_{name}_p{p}_scal"] = np.array([part.mass, part.I_particle, part.Larea, part.Lb])
        d[f"init_{name}_feq_sha"] = np.frombuffer(bytes.fromhex(_sha(st.feq)), dtype=np.uint8)
    np.savez_compressed(out, **d)


def make_lambda_rho(units_path, out):
    """lambda(k) of the reference's compute_lambda for fluid densities other
    than 1, on the marker inputs stored in units.npz."""
    from iblbm.ibm.dfc import compute_lambda
    u = np.load(units_path)
    nx, ny, dx, La = int(u["i_nx"][0]), int(u["i_ny"][0]), float(u["i_dx"][0]), float(u["i_Larea"][0])
    d = {}
    for dt_name in ("hat", "peskin4pt"):
        for rho_f in (1.3, 0.7):
            d[f"lam_{dt_name}_{rho_f}"] = compute_lambda(u["i_Lx"], u["i_Ly"], rho_f, La, dx, dx, ny, nx, dt_name)
    np.savez_compressed(out, **d)


def make_run(name, kw, out_dir):
    from iblbm import SimConfig, run
    cfg = SimConfig(**kw)
    res = run(cfg, verbose=False)
    st = res["state"]
    d = {"config_json": np.frombuffer(json.dumps(kw).encode(), dtype=np.uint8)}
    arrays = {"ro": st.ro, "U": st.U, "fib": st.fib, "fstar": st.fstar, "feq": st.feq}
    for k, a in arrays.items():
        d[f"sha_{k}"] = np.frombuffer(bytes.fromhex(_sha(a)), dtype=np.uint8)
        d[f"sample_{k}"] = _sample(a)
    d["Cd_history"] = np.asarray(res["Cd_history"], dtype=np.float64)
    d["Cl_history"] = np.asarray(res["Cl_history"], dtype=np.float64)
    d["final_step"] = np.array([res["final_step"]])
    if st.particles:
        d["particles"] = np.array([[*p.pos, *p.vel, *p.force] for p in st.particles])
        if cfg.enable_rotation:
            d["rotation"] = np.array([[p.omega, p.angle, p.torque] for p in st.particles])
    if getattr(st, "_mdf_iter_stats", None):
        s = st._mdf_iter_stats
        d["mdf_stats"] = np.array([s["iter_count"], s["last_residual"]])
    if getattr(st, "dfc_force_lagr", None) is not None:
        d["dfc_force"] = np.asarray(st.dfc_force_lagr)
    d["markers"] = np.stack([np.asarray(st.Lx), np.asarray(st.Ly)])
    np.savez_compressed(os.path.join(out_dir, f"run_{name}.npz"), **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IBLBM_REFERENCE"),
                    required="IBLBM_REFERENCE" not in os.environ,
                    help="reference checkout (or set IBLBM_REFERENCE)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    _import_reference(args.reference)
    if args.only in (None, "units"):
        make_units(os.path.join(HERE, "units.npz"))
        print("units.npz written")
    if args.only in (None, "units", "lambda_rho"):
        make_lambda_rho(os.path.join(HERE, "units.npz"), os.path.join(HERE, "lambda_rho.npz"))
        print("lambda_rho.npz written")
    for name, kw in RUN_CASES.items():
        if args.only not in (None, name):
            continue
        make_run(name, kw, HERE)
        print(f"run_{name}.npz written")
    for name, kw in SINGLE_CASES.items():
        if args.only not in (None, "sed1_" + name):
            continue
        make_single(name, kw, HERE)
        print(f"sed1_{name}.npz written")


if __name__ == "__main__":
    main()
