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
            if sed:
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
    elif eng.last_out_step > 0 and not eng.no_ibm:
        from .diagnostics import engine_slip
        result["slip"] = engine_slip(eng)  # marker slip of the last output step / U_ref
    result["engine"] = eng
    return result
