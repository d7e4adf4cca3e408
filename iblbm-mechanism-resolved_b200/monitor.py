"""Sedimentation output files in the reference's formats: ``status.json``,
``sedimentation_history.json`` and the velocity-field ``.npz`` files
(monitor/sedimentation.py:41-48, 50-208, 211-488), so that the reference's
analysis scripts read runs of this package unchanged.

``create_sedimentation_callback`` returns a callable with the reference's
callback signature ``(step, Cd, Cl, error, state, elapsed, converged)`` for
``run(cfg, callback=...)``, with ``finalize(converged, final_state, final_step,
termination_reason)`` and ``history`` attached as in the reference.  The
reference's plots and video frames are not produced (figures are out of this
package's scope); the JSON and ``.npz`` outputs are.

The state may be this package's (``state.particles``, ``mdf_iter_stats``) or
carry the reference's single-particle attributes (``particle_pos``,
``particle_vel``, ``particle_force``, ``_mdf_iter_stats``).
"""
from __future__ import annotations

import json
import os
from datetime import datetime

import numpy as np


def _format_elapsed(seconds: float) -> str:
    """'Xh YYm ZZs' / 'Ym ZZs' / 'Zs' (monitor/sedimentation.py:29-38)."""
    h = int(seconds // 3600)
    m = int((seconds % 3600) // 60)
    s = int(seconds % 60)
    if h > 0:
        return f"{h}h {m:02d}m {s:02d}s"
    if m > 0:
        return f"{m}m {s:02d}s"
    return f"{s}s"


def _write_json(path, data, indent=2):
    """Write through a temporary file and rename (monitor/sedimentation.py:41-47)."""
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(data, fh, indent=indent)
    os.replace(tmp, path)


class MdfIterStats:
    """Running MDF iteration statistics over the callback's records
    (monitor/sedimentation.py:50-108): count, sum / max / min of the
    iteration counts, a histogram over 0..20, diverged / converged counts and
    the residual sum / max (infinite residuals excluded)."""

    BINS = 21

    def __init__(self):
        self.n = 0
        self.it_sum = 0
        self.it_max = 0
        self.it_min = -1
        self.diverged = 0
        self.converged = 0
        self.hist = [0] * self.BINS
        self.res_sum = 0.0
        self.res_max = 0.0

    def add(self, stats):
        if stats is None:
            return
        ic = int(stats.get("iter_count", 0))
        res = float(stats.get("last_residual", 0.0))
        self.n += 1
        self.it_sum += ic
        self.it_max = max(self.it_max, ic)
        self.it_min = ic if self.it_min < 0 else min(self.it_min, ic)
        if 0 <= ic < self.BINS:
            self.hist[ic] += 1
        self.diverged += 1 if stats.get("diverged") else 0
        self.converged += 1 if stats.get("converged") else 0
        if res != float("inf"):
            self.res_sum += res
            self.res_max = max(self.res_max, res)

    def summary(self):
        if self.n == 0:
            return None
        return {"n_steps": self.n, "iter_avg": round(self.it_sum / self.n, 3), "iter_max": int(self.it_max),
                "iter_min": int(self.it_min) if self.it_min >= 0 else 0, "diverge_count": int(self.diverged),
                "converge_count": int(self.converged), "residual_avg": round(self.res_sum / self.n, 6),
                "residual_max": round(self.res_max, 6), "histogram": list(self.hist)}


def _host(a):
    return a.get() if hasattr(a, "get") else (a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a))


def _re_metrics(speed, lattice_D, nu_lat, rho_ratio, basis):
    """Particle Reynolds numbers of a speed (monitor/sedimentation.py:116-127)."""
    re_std = 0.0 if nu_lat <= 0.0 else float(speed * lattice_D / nu_lat)
    re_pb = float(re_std * rho_ratio)
    re_ref = re_pb if basis == "particle_basis" else re_std
    return round(re_std, 2), round(re_pb, 2), round(re_ref, 2)


def peak_re_metrics(history, lattice_D, nu_lat, rho_ratios, basis):
    """Per particle, the Reynolds numbers at the largest speed in the history and
    the step of that speed (monitor/sedimentation.py:130-182; the first record
    of the largest speed wins)."""
    out = {"Re_standard_peaks": [], "Re_particle_basis_peaks": [], "Re_reference_peaks": [], "peak_steps": []}
    if not history:
        return out
    if "particles" in history[0]:
        series = [[(r["particles"][k]["vx"], r["particles"][k]["vy"], r["step"]) for r in history]
                  for k in range(len(rho_ratios))]
    else:
        series = [[(r["vx"], r["vy"], r["step"]) for r in history]]
    for k, recs in enumerate(series):
        peak, peak_step = 0.0, 0
        for vx, vy, step in recs:
            sp = float(np.sqrt(vx ** 2 + vy ** 2))
            if sp > peak:
                peak, peak_step = sp, int(step)
        a, b, c = _re_metrics(peak, lattice_D, nu_lat, rho_ratios[k], basis)
        out["Re_standard_peaks"].append(a)
        out["Re_particle_basis_peaks"].append(b)
        out["Re_reference_peaks"].append(c)
        out["peak_steps"].append(peak_step)
    return out


def _first_particle(state):
    """(pos, vel, force) of the first particle, from either state convention."""
    parts = getattr(state, "particles", None)
    if parts:
        p = parts[0]
        force = getattr(p, "fib_force", None)
        return _host(p.pos), _host(p.vel), force
    return _host(state.particle_pos), _host(state.particle_vel), getattr(state, "particle_force", None)


def _mdf_stats(state):
    s = getattr(state, "_mdf_iter_stats", None)
    return s if s is not None else getattr(state, "mdf_iter_stats", None)


def _velocity_npz(path, state, pos, step=None, f32=False):
    """Eux, Euy on the (ny, nx) grid, dx, dy, [step], particle_pos
    (monitor/sedimentation.py:185-208 and 447-460)."""
    ny, nx = state.ny, state.nx
    U = _host(state.U)
    ex, ey = U[:, 0].reshape(ny, nx), U[:, 1].reshape(ny, nx)
    if f32:
        ex, ey = ex.astype(np.float32), ey.astype(np.float32)
    extra = {} if step is None else {"step": int(step)}
    np.savez_compressed(path, Eux=ex, Euy=ey, dx=state.dx, dy=state.dy, **extra,
                        particle_pos=np.asarray(pos, dtype=np.float64) if step is not None else pos)


def create_sedimentation_callback(output_dir, cfg, plot_every=10, save_frames=False, snapshot_every=50):
    """The reference's sedimentation monitor without its figures
    (monitor/sedimentation.py:211-488): a record per callback (per particle
    with t*, x, y, velocities and their gravitational-velocity scalings; MDF
    iteration count / residual / divergence), ``status.json`` rewritten at
    every call, the history written at the first call and every
    ``plot_every``-th, a float32 velocity snapshot every ``snapshot_every``-th
    call, and at ``finalize`` the history, the final velocity field, the
    completion flags and the peak Reynolds numbers."""
    os.makedirs(output_dir, exist_ok=True)
    lattice_D = cfg.cylinder_D_ratio * (cfg.NN - 1)
    dx_dom = 1.0 / (cfg.NN - 1)
    D_dom = lattice_D * dx_dom
    g = cfg.gravity
    rho_ratio = cfg.rho_ratio
    x0, y0 = cfg.cylinder_center
    u_g = np.sqrt(abs(rho_ratio - 1.0) * g * lattice_D)
    history, calls, last_elapsed, last_state = [], [0], [0.0], [None]
    mdf = MdfIterStats()
    multi = getattr(cfg, "particles_config", None) is not None and len(cfg.particles_config) > 1
    right = getattr(cfg, "gravity_direction", "down") == "right"
    hist_path = os.path.join(output_dir, "sedimentation_history.json")
    status_path = os.path.join(output_dir, "status.json")

    def scaled(step, pos, vel, ug):
        """t*, y*, vy*, vx* (vertical or horizontal gravity)."""
        if ug <= 1e-15:
            return 0.0, 0.0, 0.0, 0.0
        t_star = float(step * ug / lattice_D)
        if right:
            return t_star, float((pos[0] - x0) / D_dom), float(vel[1] / ug), float(vel[0] / ug)
        return t_star, float((y0 - pos[1]) / D_dom), float(-vel[1] / ug), float(vel[0] / ug)

    def callback(step, Cd, Cl, error, state, elapsed, converged):
        calls[0] += 1
        interval = elapsed - last_elapsed[0]
        last_elapsed[0] = elapsed
        last_state[0] = state
        stats = _mdf_stats(state)
        if multi and getattr(state, "particles", None) is not None:
            pdata = []
            for k, p in enumerate(state.particles):
                pos, vel = _host(p.pos), _host(p.vel)
                ug = np.sqrt(abs(p.rho_ratio - 1.0) * g * lattice_D)
                t_star, _, vy_s, vx_s = scaled(step, pos, vel, ug)
                pdata.append({"id": k, "rho_ratio": p.rho_ratio, "t_star": t_star, "x": float(pos[0]),
                              "y": float(pos[1]), "vx": float(vel[0]), "vy": float(vel[1]), "vx_star": vx_s,
                              "vy_star": vy_s})
            rec = {"step": int(step), "particles": pdata}
            pos, vel, _ = _first_particle(state)
            vy_star, vx_star = pdata[0]["vy_star"], pdata[0]["vx_star"]
            y_star = float((pos[0] - x0) / D_dom) if right else float((y0 - pos[1]) / D_dom)
        else:
            pos, vel, force = _first_particle(state)
            t_star, y_star, vy_star, vx_star = scaled(step, pos, vel, u_g)
            rec = {"t_star": t_star, "y_star": y_star, "vy_star": vy_star, "vx_star": vx_star,
                   "x": float(pos[0]), "y": float(pos[1]), "vx": float(vel[0]), "vy": float(vel[1]),
                   "step": int(step),
                   "f_hydro_x": float(force[0]) if force is not None else 0.0,
                   "f_hydro_y": float(force[1]) if force is not None else 0.0}
            for k in ("angle", "omega", "torque"):
                if hasattr(state, "particle_" + k):
                    rec[k] = float(getattr(state, "particle_" + k))
            if getattr(state, "inside_residual_mean", 0.0) != 0.0:
                rec["inside_residual_mean"] = state.inside_residual_mean
                rec["inside_residual_max"] = state.inside_residual_max
            if getattr(state, "p_int", None) is not None:
                rec["p_int_x"] = float(state.p_int[0])
                rec["p_int_y"] = float(state.p_int[1])
                rec["l_int_z"] = state.l_int
        if stats is not None:
            rec["mdf_iter"] = int(stats.get("iter_count", 0))
            rec["mdf_residual"] = float(stats.get("last_residual", 0.0))
            rec["mdf_diverged"] = bool(stats.get("diverged", False))
            mdf.add(stats)
        history.append(rec)
        status = {
            "experiment_type": "sedimentation", "completed": False, "step": int(step),
            "elapsed_sec": round(elapsed, 1), "elapsed_str": _format_elapsed(elapsed),
            "interval_time": round(interval, 2), "converged": False,
            "vy_star": round(vy_star, 6), "y_star": round(y_star, 4), "vx_star": round(vx_star, 6),
            "particle_x": round(float(pos[0]), 6), "particle_y": round(float(pos[1]), 6),
            "config": {
                "rho_ratio": rho_ratio, "ibm_method": cfg.ibm_method,
                "delta_type": getattr(cfg, "delta_type", "peskin4pt"),
                "collision_model": getattr(cfg, "collision_model", "BGK"),
                "settling_inertia_model": getattr(cfg, "settling_inertia_model", "unset"),
                "NN": cfg.NN, "max_steps": cfg.max_steps, "check_interval": cfg.check_interval, "gravity": g,
                "gravity_direction": getattr(cfg, "gravity_direction", "down"),
                "time_integrator": getattr(cfg, "time_integrator", "verlet"),
                "enable_rotation": getattr(cfg, "enable_rotation", False),
                "rotation_coupling": getattr(cfg, "rotation_coupling", "indirect"),
                "marker_spacing_factor": getattr(cfg, "marker_spacing_factor", 1.0),
                "retraction_dx": getattr(cfg, "retraction_dx", 0.0),
                "mdf_iterations": getattr(cfg, "mdf_iterations", 1),
                "incompressible_lbgk": getattr(cfg, "incompressible_lbgk", False),
                "sedimentation_stop_at_contact": getattr(cfg, "sedimentation_stop_at_contact", False),
                "sedimentation_stop_offset_d": getattr(cfg, "sedimentation_stop_offset_d", 0.0),
                "sedimentation_reference_basis": getattr(cfg, "sedimentation_reference_basis", "standard"),
                "sedimentation_euler_update_scheme": getattr(cfg, "sedimentation_euler_update_scheme",
                                                             "new_velocity"),
            },
            "updated_at": datetime.now().isoformat(timespec="seconds"),
        }
        summ = mdf.summary()
        if summ is not None:
            status["mdf_iter_stats"] = summ
        _write_json(status_path, status)
        if snapshot_every > 0 and calls[0] % snapshot_every == 0:
            snap = os.path.join(output_dir, "snapshots")
            os.makedirs(snap, exist_ok=True)
            _velocity_npz(os.path.join(snap, f"velocity_{int(step):07d}.npz"), state, pos, step=step, f32=True)
        if calls[0] == 1 or calls[0] % plot_every == 0:
            _write_json(hist_path, history)

    def finalize(converged=False, final_state=None, final_step=None, termination_reason=None):
        with open(hist_path, "w") as fh:
            json.dump(history, fh, indent=2)
        state = final_state if final_state is not None else last_state[0]
        if state is not None:
            pos, _, _ = _first_particle(state)
            _velocity_npz(os.path.join(output_dir, "velocity_field.npz"), state, pos)
        if not os.path.exists(status_path):
            return
        with open(status_path) as fh:
            data = json.load(fh)
        data["completed"] = True
        data["converged"] = converged
        if final_step is not None:
            data["step"] = int(final_step)
            data["final_step"] = int(final_step)
        if termination_reason is not None:
            data["termination_reason"] = termination_reason
        if state is not None:
            nu_lat = (float(state.tau) - 0.5) / 3.0
            if multi and getattr(state, "particles", None) is not None:
                rho_ratios = [float(p.rho_ratio) for p in state.particles]
            else:
                rho_ratios = [float(getattr(cfg, "rho_ratio", 1.0))]
            basis = getattr(cfg, "sedimentation_reference_basis", "standard")
            peaks = peak_re_metrics(history, lattice_D, nu_lat, rho_ratios, basis)
            data.update(peaks)
            data["history_len"] = len(history)
            data["re_reference_basis"] = basis
            if peaks["Re_standard_peaks"]:
                data["Re_standard_peak"] = peaks["Re_standard_peaks"][0]
                data["Re_particle_basis_peak"] = peaks["Re_particle_basis_peaks"][0]
                data["Re_reference_peak"] = peaks["Re_reference_peaks"][0]
        _write_json(status_path, data)

    callback.finalize = finalize
    callback.history = history
    return callback
