"""``run(cfg)`` — the time loop of iblbm/runtime/loop.py:44-151 on the fused engine.

The returned dictionary has the reference's keys (Cd_history, Cl_history,
state, converged, final_step, termination_reason, and sedimentation_history
for sedimentation runs).  Between diagnostics the engine replays CUDA graphs of
whole timesteps; at every ``check_interval`` step the moments are written out
and Cd/Cl, the velocity-convergence error and the stop rules are evaluated as
in the reference.  Cd / Cl and the convergence error are reduced on the
device (``iblbm_force_coeffs``, ``iblbm_velocity_change``); when no stop rule,
callback or particle record needs them at each check, the coefficients of up
to SPAN_CHECKS checks collect in the engine's device ring and reach the host
in one copy, so the host never waits on the GPU between those checks.
"""
from __future__ import annotations

import json
import math
import time

import numpy as np

from .engine import Engine


def _sedimentation_record(p, ttt, d_lattice, g, cfg, dx, pid):
    """Per-particle record — iblbm/diagnostics/internal_flow.py record_sedimentation_state
    (vertical gravity) and runtime/scenarios/sedimentation_multi.py:241-265 (horizontal)."""
    if cfg.gravity_direction == "right":
        u_g = float(math.sqrt(abs(p.rho_ratio - 1.0) * g * d_lattice))
        ok = u_g > 1e-15
        return {"id": pid, "rho_ratio": p.rho_ratio,
                "t_star": float(ttt * u_g / d_lattice) if ok else 0.0,
                "dist_star": float((p.pos[0] - p.cx_init) / (d_lattice * dx)) if ok else 0.0,
                "vx_star": float(p.vel[0] / u_g) if ok else 0.0, "vy_star": float(p.vel[1] / u_g) if ok else 0.0,
                "x": float(p.pos[0]), "y": float(p.pos[1]), "vx": float(p.vel[0]), "vy": float(p.vel[1])}
    u_g = float(math.sqrt(abs(p.rho_ratio - 1.0) * g * d_lattice))
    return {"id": pid, "rho_ratio": p.rho_ratio, "step": ttt, "x": float(p.pos[0]), "y": float(p.pos[1]),
            "vx": float(p.vel[0]), "vy": float(p.vel[1]),
            "y_star": float((p.pos[1] - p.cy_init) / (d_lattice * dx)),
            "vy_star": float(p.vel[1] / u_g) if u_g > 1e-15 else 0.0}


def _single_record(p, ttt, d_lattice, g, cfg, dx):
    """The single-particle runtime's record (iblbm/diagnostics/internal_flow.py:156-214,
    record_sedimentation_state, and runtime/scenarios/sedimentation_single.py:294-297):
    distance fallen and velocities made dimensionless with u_g = sqrt(|rho_r - 1| g D),
    and the hydrodynamic force."""
    u_g = np.sqrt(abs(cfg.rho_ratio - 1.0) * g * d_lattice)
    pos, vel = p.pos, p.vel
    if u_g < 1e-15:
        rec = {"step": int(ttt), "t_star": 0.0, "y_star": 0.0, "vy_star": 0.0, "vx_star": 0.0,
               "x": float(pos[0]), "y": float(pos[1]), "vx": float(vel[0]), "vy": float(vel[1])}
    else:
        rec = {"step": int(ttt), "t_star": float(ttt * u_g / d_lattice),
               "y_star": float((p.cy_init - pos[1]) / (d_lattice * dx)), "vy_star": float(-vel[1] / u_g),
               "vx_star": float(vel[0] / u_g), "x": float(pos[0]), "y": float(pos[1]), "vx": float(vel[0]),
               "vy": float(vel[1])}
    rec["f_hydro_x"] = float(p.force[0])
    rec["f_hydro_y"] = float(p.force[1])
    return rec


def _single_flow_diagnostics(rec, eng, cfg, d_lattice):
    """The fluid inside the disc (sedimentation_single.py:298-322): residual
    velocity, momentum and angular momentum from this step's fields."""
    from .diagnostics import (compute_inside_residual, compute_internal_angular_momentum,
                              compute_internal_momentum)
    st = eng.read_state()
    p = st.particles[0]
    dx = st.dx
    cx, cy = float(p.pos[0]), float(p.pos[1])
    r_domain = st.lattice_r * dx
    Eux, Euy = st.U[:, 0].reshape(st.ny, st.nx), st.U[:, 1].reshape(st.ny, st.nx)
    ro = st.ro.reshape(st.ny, st.nx)
    u_g = math.sqrt(abs(cfg.rho_ratio - 1.0) * st.gravity_lattice * d_lattice)
    res = compute_inside_residual(Eux, Euy, dx, dx, cx, cy, d_lattice * dx, kappa=2.0, u_ref=max(float(u_g), 1e-12))
    rec["inside_residual_mean"] = res["mean"]
    rec["inside_residual_max"] = res["max"]
    rec["inside_residual_mean_norm"] = res["mean_normalized"]
    px, py = compute_internal_momentum(Eux, Euy, ro, dx, dx, cx, cy, r_domain)
    rec["p_int_x"] = px
    rec["p_int_y"] = py
    rec["l_int_z"] = compute_internal_angular_momentum(Eux, Euy, ro, dx, dx, cx, cy, r_domain)


def _stop_reason(p, cfg, dx):
    """iblbm/runtime/scenarios/sedimentation_common.py:19-66."""
    pos, r = p.pos, p.r_domain
    if cfg.sedimentation_stop_at_contact:
        if cfg.gravity_direction == "right":
            if float(pos[0]) >= cfg.xmax - r:
                return "contact"
        elif float(pos[1]) <= r:
            return "contact"
    if cfg.sedimentation_stop_offset_d > 0.0:
        d = cfg.cylinder_D_ratio
        if cfg.gravity_direction == "right":
            if float(pos[0]) >= cfg.xmax - cfg.sedimentation_stop_offset_d * d:
                return "offset"
        elif float(pos[1]) <= cfg.sedimentation_stop_offset_d * d:
            return "offset"
    return None


def _near_wall(p, cfg, dx, safety=2.0):
    margin = safety * dx
    x, y, r = float(p.pos[0]), float(p.pos[1]), p.r_domain
    terminal = cfg.sedimentation_stop_at_contact or cfg.sedimentation_stop_offset_d > 0.0
    if cfg.gravity_direction == "right":
        return (y - r < margin or y + r > cfg.ymax - margin or x - r < margin
                or (not terminal and x + r > cfg.xmax - margin))
    return ((not terminal and y - r < margin) or y + r > cfg.ymax - margin or x - r < margin
            or x + r > cfg.xmax - margin)


SPAN_CHECKS = 256  # checks queued on the device between host reads when no stop rule needs them


def run(cfg, verbose: bool = True, callback=None, save_dir=None, engine: Engine | None = None) -> dict:
    eng = engine if engine is not None else Engine(cfg)
    torch = eng.torch
    Cd_history, Cl_history, history = [], [], []
    converged, error, termination = False, 1.0, "max_steps"
    have_prev = False
    t0 = time.time()
    ttt = 1
    ci = int(cfg.check_interval)
    sed = eng.st.particles is not None
    single = eng.single
    d_lattice = 2.0 * eng.st.lattice_r
    # Without a stop rule, a callback or particle records nothing at a check
    # needs its values on the host before the run goes on: the Cd / Cl of many
    # checks are reduced into the engine's device ring and read in one copy.
    span = not sed and callback is None and not cfg.use_convergence and cfg.cd_convergence_tol is None
    pending = []  # (step, ring entry or None for no immersed body)

    def flush():
        if not pending:
            return
        idx = [k for _, k in pending if k is not None]
        rows = eng.read_force_coeffs(idx[0], len(idx)) if idx else None
        r = 0
        for step, k in pending:
            if k is None:
                Cd, Cl = 0.0, 0.0
            else:
                Cd, Cl = float(rows[r, 0]), float(rows[r, 1])
                r += 1
            Cd_history.append(Cd)
            Cl_history.append(Cl)
            if verbose:
                print(f"step {step:>7d} | Cd={Cd:.6f} Cl={Cl:.6f} | err={error:.2e} | {time.time() - t0:.1f}s")
        pending.clear()

    while True:
        if converged and (cfg.use_convergence or cfg.cd_convergence_tol is not None):
            if termination == "max_steps":
                termination = "converged"
            break
        if ttt > cfg.max_steps:
            break
        target = min(((ttt - 1) // ci + 1) * ci, cfg.max_steps)
        eng.advance(target - ttt + 1, outputs_last=True)
        ttt = target
        if span:
            if ttt % ci == 0:
                pending.append((ttt, None if eng.no_ibm else eng.queue_force_coeffs()))
            if len(pending) >= SPAN_CHECKS or ttt >= cfg.max_steps:
                flush()
            ttt += 1
            continue
        if ttt % ci == 0:
            if single:
                rec = _single_record(eng.st.particles[0], ttt, d_lattice, eng.st.gravity_lattice, cfg, eng.st.dx)
                if cfg.diagnostics_interval and cfg.diagnostics_interval > 0 and ttt % cfg.diagnostics_interval == 0:
                    _single_flow_diagnostics(rec, eng, cfg, d_lattice)
                history.append(rec)
                Cd = Cl = 0.0
            elif sed:
                rec = {"step": ttt, "particles": [
                    _sedimentation_record(p, ttt, d_lattice, eng.st.gravity_lattice, cfg, eng.st.dx, k)
                    for k, p in enumerate(eng.st.particles)]}
                history.append(rec)
                Cd = Cl = 0.0
            else:
                Cd, Cl = eng.cd_cl()
            Cd_history.append(Cd)
            Cl_history.append(Cl)
            if verbose:
                print(f"step {ttt:>7d} | Cd={Cd:.6f} Cl={Cl:.6f} | err={error:.2e} | {time.time() - t0:.1f}s")
            if callback is not None:
                callback(step=ttt, Cd=Cd, Cl=Cl, error=error, state=eng.read_state(),
                         elapsed=time.time() - t0, converged=converged)
            if sed:
                p0 = eng.st.particles[0]
                if single:  # sedimentation_single.py:332-345
                    v = rec["vy_star"]
                else:
                    v = float(p0.vel[0]) if cfg.gravity_direction == "right" else float(p0.vel[1])
                reason = "nan" if not math.isfinite(v) else _stop_reason(p0, cfg, eng.st.dx)
                if reason is None and any(_near_wall(p, cfg, eng.st.dx) for p in eng.st.particles):
                    reason = "domain_bounds"
                if reason is not None:
                    termination = reason
                    break
                if save_dir and ttt % 5000 == 0:
                    with open(save_dir + "/sedimentation_history.json", "w") as fh:
                        json.dump(history, fh)
            if cfg.use_convergence:
                # iblbm/diagnostics/core.py:116-135, reduced on the device
                if ttt == cfg.convergence_start:
                    eng.velocity_change()  # stores this step's field as the reference
                    have_prev = True
                elif ttt > cfg.convergence_start and have_prev:
                    error = float(eng.velocity_change()[2].item())
                    if error < cfg.convergence_threshold:
                        converged = True
            if (cfg.cd_convergence_tol is not None and ttt > cfg.cd_convergence_start_step
                    and len(Cd_history) >= cfg.cd_convergence_window):
                recent = Cd_history[-cfg.cd_convergence_window:]
                if max(recent) - min(recent) < cfg.cd_convergence_tol:
                    converged = True
                    termination = "cd_converged"
        ttt += 1
    flush()
    torch.cuda.synchronize(eng.dev)
    state = eng.read_state() if eng.last_out_step > 0 else eng.st
    result = {"Cd_history": np.array(Cd_history), "Cl_history": np.array(Cl_history), "state": state,
              "converged": converged, "final_step": ttt - 1, "termination_reason": termination}
    if sed:
        result["sedimentation_history"] = history
    if single:
        # the single-particle runtime keeps the disc on the state (iblbm/physics/sedimentation.py:109-128)
        p = eng.st.particles[0]
        state.particle_pos, state.particle_vel = p.pos.copy(), p.vel.copy()
        state.particle_vel_prev, state.particle_force = p.vel_prev.copy(), p.force.copy()
        state.particle_omega, state.particle_angle, state.particle_torque = p.omega, p.angle, p.torque
    elif eng.last_out_step > 0 and not eng.no_ibm:
        from .diagnostics import engine_slip
        result["slip"] = engine_slip(eng)  # marker slip of the last output step / U_ref
    result["engine"] = eng
    return result
