"""Diagnostics of the reference's result analysis, on this package's arrays.

``compute_strouhal`` restates iblbm/diagnostics/core.py:138-214 (Strouhal
number from a Cl history: second half, detrended, peak of the rfft power
spectrum without the DC term, with the reference's handling of rectified |Cl|
series).  ``compute_slip_error`` restates iblbm/diagnostics/ibm_quality.py:
132-188 (boundary slip of a velocity field on a diagnostic marker ring);
``compute_leakage_flux`` restates :189-251 (the normal flux through that ring);
their interpolation runs on the GPU through the band kernel (field-input mode),
in the reference's summation order.  ``engine_slip`` evaluates the same on the
engine's own markers and last output velocity.  ``tg_analytical_velocity_field``
and ``compute_l2_error`` restate iblbm/diagnostics/core.py:216-268 (the
decaying Taylor-Green vortex and the relative L2 error against it), and
``tg_l2_error`` applies them to a Taylor-Green run's final velocity.  The
post-processing statistics of the reference's histories and fields restate
iblbm/diagnostics/core.py: ``tail_start_index`` / ``tail_values`` /
``tail_mean`` / ``tail_peak_to_peak_amp`` (:31-51, the last 30 % of a
series), ``check_convergence`` (:115-136), ``compute_recirculation_length``
(:264-310) and ``compute_cl_amplitude`` (:312-333).  The flow inside a body
restates iblbm/diagnostics/internal_flow.py: ``compute_inside_residual``
(:32-85), ``compute_internal_momentum`` (:87-119),
``compute_internal_angular_momentum`` (:121-154) and ``compute_l_int_z``
(:220-262).  ``compute_stress_tensor`` and ``integrate_surface_force`` restate
iblbm/diagnostics/surface.py:30-163 (force on a cylinder from the stress of
the non-equilibrium populations).
"""
from __future__ import annotations

import numpy as np


def compute_strouhal(Cl_history, steps, D_lattice, u_ref, check_interval):
    """St = f_shed D / U from the second half of a Cl series sampled every
    check_interval steps (signed Cl, or |Cl| whose peak sits at 2 f_shed)."""
    cl = np.asarray(Cl_history, dtype=float)
    half = cl[len(cl) // 2:]
    rectified = bool(np.all(cl >= -1e-10))
    power = np.abs(np.fft.rfft(half - np.mean(half))) ** 2
    power[0] = 0
    f_peak = int(np.argmax(power)) / (len(half) * check_interval)
    if not rectified:
        f_shed = f_peak
    else:
        fs = 1.0 / check_interval
        direct = (f_peak / 2) * D_lattice / u_ref
        # |Cl| peaks at 2 f_shed, or at its alias fs - 2 f_shed above Nyquist;
        # a direct reading inside the shedding range (>= 0.1) is taken as is
        f_shed = f_peak / 2 if direct >= 0.1 else (fs - f_peak) / 2
    return f_shed * D_lattice / u_ref


def diagnostic_markers(cx, cy, r, NN, marker_spacing_factor=0.5):
    """Marker ring on the body surface (no retraction), the reference's spacing
    rule: 2 pi r_lattice / spacing points, the closing duplicate dropped."""
    n_param = 2.0 * np.pi * (r * (NN - 1)) / marker_spacing_factor
    step = 1.0 / n_param
    s = np.arange(0, 1.0 + step * 0.5, step)
    s = s[s <= 1.0 + 1e-12]
    if len(s) > 1 and np.abs(s[-1] - 1.0) < step * 0.5:
        s = s[:-1]
    theta = 2.0 * np.pi * s
    return r * np.cos(theta) + cx, r * np.sin(theta) + cy, theta


def _interp_gpu(Eux, Euy, Lx, Ly, dx, dy, delta_type):
    import torch
    from . import gpu_kernels as gk
    ny, nx = Eux.shape
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")
    ex, ey = d(Eux).reshape(-1), d(Euy).reshape(-1)
    ro = torch.ones_like(ex)
    Lb = len(Lx)
    _, Lux, Luy = gk.ibm_direct_forcing_gpu(d(Lx), d(Ly), torch.zeros(Lb, 2, dtype=torch.float64, device="cuda"),
                                            ex, ey, ro, dx, dy, 1.0, 1.0, ny, nx, delta_type, True, False)
    return Lux.cpu().numpy(), Luy.cpu().numpy()


def compute_slip_error(Eux, Euy, dx, dy, cx, cy, D, NN, delta_type, u_target_x=None, u_target_y=None, u_ref=0.1):
    """Slip |u(X_m) - u_target| / U_ref on a diagnostic ring: mean, max, RMS and
    per marker.  Eux, Euy: (ny, nx) host or device arrays."""
    Eux = np.asarray(Eux.cpu() if hasattr(Eux, "cpu") else Eux, dtype=np.float64)
    Euy = np.asarray(Euy.cpu() if hasattr(Euy, "cpu") else Euy, dtype=np.float64)
    Lx, Ly, theta = diagnostic_markers(cx, cy, D / 2.0, NN)
    Lux, Luy = _interp_gpu(Eux, Euy, Lx, Ly, dx, dy, delta_type)
    tx = np.zeros(len(Lx)) if u_target_x is None else u_target_x
    ty = np.zeros(len(Lx)) if u_target_y is None else u_target_y
    mag = np.sqrt((Lux - tx) ** 2 + (Luy - ty) ** 2)
    return {"mean": float(np.mean(mag) / u_ref), "max": float(np.max(mag) / u_ref),
            "rms": float(np.sqrt(np.mean(mag ** 2)) / u_ref), "per_marker": mag / u_ref, "theta": theta}


def compute_leakage_flux(Eux, Euy, dx, dy, cx, cy, D, NN, delta_type, u_target_x=None, u_target_y=None,
                         u_ref=0.1):
    """Flux through the body surface, the integral of (u(X_m) - u_target) . n ds
    over the diagnostic ring (outward normal (cos t, sin t), ds = 2 pi r / N),
    raw and over U_ref pi D, with the per-marker normal velocity over U_ref
    (iblbm/diagnostics/ibm_quality.py:189-251).  Near zero when the boundary
    holds.  The interpolation runs on the GPU as for compute_slip_error."""
    Eux = np.asarray(Eux.cpu() if hasattr(Eux, "cpu") else Eux, dtype=np.float64)
    Euy = np.asarray(Euy.cpu() if hasattr(Euy, "cpu") else Euy, dtype=np.float64)
    r = D / 2.0
    Lx, Ly, theta = diagnostic_markers(cx, cy, r, NN)
    Lb = len(Lx)
    Lux, Luy = _interp_gpu(Eux, Euy, Lx, Ly, dx, dy, delta_type)
    tx = np.zeros(Lb) if u_target_x is None else u_target_x
    ty = np.zeros(Lb) if u_target_y is None else u_target_y
    un = (Lux - tx) * np.cos(theta) + (Luy - ty) * np.sin(theta)
    raw = float(np.sum(un * (2.0 * np.pi * r / Lb)))
    return {"total": raw / (u_ref * np.pi * D), "total_raw": raw, "per_marker": un / u_ref, "theta": theta}


def engine_slip(engine, u_ref=None):
    """Slip of the engine's last output velocity on its own markers (the
    simulation's ring, desired velocities as targets): mean, max and RMS over
    U_ref (the inflow speed, the oscillation speed scale, or the Taylor-Green
    vortex amplitude)."""
    st, cfg = engine.st, engine.cfg
    if u_ref is None:
        if cfg.scenario_type == "taylor_green":
            u_ref = cfg.tg_u0  # no inflow: the vortex amplitude
        else:
            u_ref = cfg.lattice_u if cfg.motion_type == "oscillating" else st.in_u
    U = engine.U_out.double().reshape(st.ny, st.nx, 2)
    Lx = engine.d_Lx[: engine.Lb].cpu().numpy()
    Ly = engine.d_Ly[: engine.Lb].cpu().numpy()
    if engine.xt is not None:
        # markers in force during the last output step
        xt = float(engine.xt[engine.last_out_step].item())
        Lx = engine.d_Lxc.cpu().numpy() - xt
        Ly = engine.d_Lyc.cpu().numpy()
        dv = np.stack([np.full(engine.Lb, xt), np.zeros(engine.Lb)], axis=1)
    else:
        dv = engine.d_dv[: 2 * engine.Lb].reshape(engine.Lb, 2).cpu().numpy()
        if engine.tg:  # Taylor-Green markers: the analytic velocity of the last output step
            dv = dv * float(engine.d_tg_table[engine.last_out_step].item())
    Lux, Luy = _interp_gpu(U[..., 0].cpu().numpy(), U[..., 1].cpu().numpy(), Lx, Ly, st.dx, st.dy, cfg.delta_type)
    mag = np.sqrt((Lux - dv[:, 0]) ** 2 + (Luy - dv[:, 1]) ** 2)
    return {"mean": float(np.mean(mag) / u_ref), "max": float(np.max(mag) / u_ref),
            "rms": float(np.sqrt(np.mean(mag ** 2)) / u_ref)}


def tg_analytical_velocity_field(X, Y, t, u0, L, nu):
    """Velocity of the decaying vortex at centred coordinates (X, Y) and time t:
    ux = -u0 cos(pi X/L) sin(pi Y/L) e^(-2 nu (pi/L)^2 t), uy = u0 sin(pi X/L)
    cos(pi Y/L) e^(-2 nu (pi/L)^2 t), the decay factor multiplied last."""
    decay = np.exp(-2.0 * nu * (np.pi / L) ** 2 * t)
    ux = -u0 * np.cos(np.pi * X / L) * np.sin(np.pi * Y / L) * decay
    uy = u0 * np.sin(np.pi * X / L) * np.cos(np.pi * Y / L) * decay
    return ux, uy


def compute_l2_error(U_num, U_ana):
    """||U_num - U_ana||_2 / ||U_ana||_2 over all entries (inf when U_ana is 0)."""
    diff = np.asarray(U_num) - np.asarray(U_ana)
    den = np.sqrt(np.sum(np.asarray(U_ana) ** 2))
    if den == 0.0:
        return float("inf")
    return float(np.sqrt(np.sum(diff ** 2)) / den)


def tg_l2_error(U, cfg, nx, ny, step=None):
    """Relative L2 error of a Taylor-Green run's velocity U (nx*ny x 2, row-major
    in y) against the vortex at t = step (default cfg.max_steps), on the lattice
    centred at ((nx-1)/2, (ny-1)/2) with half-width (NN-1)/2."""
    from .physics import tg_params
    L, nu = tg_params(cfg)
    X, Y = np.meshgrid(np.arange(nx) - (nx - 1) / 2.0, np.arange(ny) - (ny - 1) / 2.0)
    t = float(cfg.max_steps if step is None else step)
    ux, uy = tg_analytical_velocity_field(X.ravel(), Y.ravel(), t, cfg.tg_u0, L, nu)
    return compute_l2_error(U, np.stack([ux, uy], axis=1))


STEADY_TAIL_FRAC = 0.3


def tail_start_index(length, frac=STEADY_TAIL_FRAC):
    """First index of the tail: floor(length (1 - frac)), kept inside the series."""
    if length <= 0:
        raise ValueError("empty history array")
    return min(max(int(length * (1.0 - frac)), 0), length - 1)


def tail_values(values, frac=STEADY_TAIL_FRAC):
    arr = np.asarray(values, dtype=np.float64)
    if arr.size == 0:
        raise ValueError("empty history array")
    return arr[tail_start_index(arr.size, frac):]


def tail_mean(values, frac=STEADY_TAIL_FRAC):
    return float(np.mean(tail_values(values, frac)))


def tail_peak_to_peak_amp(values, frac=STEADY_TAIL_FRAC):
    """Half the peak-to-peak range of the tail."""
    t = tail_values(values, frac)
    return float((t.max() - t.min()) / 2.0)


def check_convergence(Eux_new, Euy_new, Eux_old, Euy_old):
    """sqrt(sum |u_new - u_old|^2 / sum |u_old|^2), 1.0 when the old field is zero."""
    num = np.sum((Eux_new - Eux_old) ** 2 + (Euy_new - Euy_old) ** 2)
    den = np.sum(Eux_old ** 2 + Euy_old ** 2)
    return 1.0 if den == 0.0 else np.sqrt(num / den)


def compute_recirculation_length(Eux, dx, dy, cx, cy, D):
    """Length of the wake's reverse-flow region over D: along the centre row,
    the first sign change of ux from negative to non-negative behind the body
    (searched from one node past the rear), located by linear interpolation,
    measured from the rear x = cx + D/2.  NaN when there is none."""
    Eux = np.asarray(Eux)
    nx = Eux.shape[1]
    row = Eux[int(round(cy / dy)), :]
    x_rear = cx + D / 2.0
    for i in range(int(np.ceil(x_rear / dx)) + 1, nx - 1):
        u0, u1 = row[i], row[i + 1]
        if u0 < 0 and u1 >= 0:
            x0, x1 = i * dx, (i + 1) * dx
            return (x0 + (0.0 - u0) / (u1 - u0) * (x1 - x0) - x_rear) / D
    return float("nan")


def compute_cl_amplitude(Cl_history):
    """Amplitude of the second half of a Cl series: its maximum for a rectified
    |Cl| series (every value >= -1e-10), else half its peak-to-peak range."""
    cl = np.asarray(Cl_history, dtype=float)
    half = cl[len(cl) // 2:]
    if np.all(cl >= -1e-10):
        return float(np.max(half))
    return float((np.max(half) - np.min(half)) / 2.0)


def _node_grid(shape, dx, dy):
    ny, nx = shape
    return np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dy)


def compute_inside_residual(Eux, Euy, dx, dy, cx, cy, D, kappa=2.0, u_ref=0.1):
    """Speed of the flow left inside a body, over the nodes deeper than kappa dx
    below its surface: mean, max, count, and mean / max over u_ref (zeros when
    no node is that deep)."""
    XX, YY = _node_grid(Eux.shape, dx, dy)
    inside = np.sqrt((XX - cx) ** 2 + (YY - cy) ** 2) - D / 2.0 < -kappa * dx
    n = int(np.sum(inside))
    if n == 0:
        return {"mean": 0.0, "max": 0.0, "n_points": 0, "mean_normalized": 0.0, "max_normalized": 0.0}
    speed = np.sqrt(Eux[inside] ** 2 + Euy[inside] ** 2)
    return {"mean": float(np.mean(speed)), "max": float(np.max(speed)), "n_points": n,
            "mean_normalized": float(np.mean(speed) / u_ref), "max_normalized": float(np.max(speed) / u_ref)}


def compute_internal_momentum(Eux, Euy, ro, dx, dy, cx, cy, r):
    """Momentum of the fluid inside a disc of radius r: sum of ro u over the
    nodes within r, times the cell area."""
    XX, YY = _node_grid(Eux.shape, dx, dy)
    m = (XX - cx) ** 2 + (YY - cy) ** 2 <= r ** 2
    dA = dx * dy
    return float(np.sum(ro[m] * Eux[m]) * dA), float(np.sum(ro[m] * Euy[m]) * dA)


def compute_internal_angular_momentum(Eux, Euy, ro, dx, dy, cx, cy, r):
    """Angular momentum of the fluid inside a disc about its centre:
    sum of rx ro uy - ry ro ux over the nodes within r, times the cell area."""
    XX, YY = _node_grid(Eux.shape, dx, dy)
    m = (XX - cx) ** 2 + (YY - cy) ** 2 <= r ** 2
    rx, ry = XX[m] - cx, YY[m] - cy
    return float(np.sum((rx * ro[m] * Euy[m] - ry * ro[m] * Eux[m])) * (dx * dy))


def compute_l_int_z(U, ro, nx, ny, dx, cx, cy, r_domain):
    """The same angular momentum in lattice units, from (N, 2) / (N,) arrays,
    summed over the box of the disc only."""
    U, ro = np.asarray(U), np.asarray(ro)
    ci, cj, r_lat = cx / dx, cy / dx, r_domain / dx
    ii, jj, rr = int(round(ci)), int(round(cj)), int(r_lat) + 2
    i0, i1 = max(0, ii - rr), min(nx, ii + rr + 1)
    j0, j1 = max(0, jj - rr), min(ny, jj + rr + 1)
    RX, RY = np.meshgrid(np.arange(i0, i1, dtype=float) - ci, np.arange(j0, j1, dtype=float) - cj)
    m = RX ** 2 + RY ** 2 <= r_lat ** 2
    sro = ro.reshape(ny, nx)[j0:j1, i0:i1]
    sux = U[:, 0].reshape(ny, nx)[j0:j1, i0:i1]
    suy = U[:, 1].reshape(ny, nx)[j0:j1, i0:i1]
    return float(np.sum(RX[m] * sro[m] * suy[m] - RY[m] * sro[m] * sux[m]))


# D2Q9 velocities in the reference's order (rest, E, N, W, S, NE, NW, SW, SE)
D2Q9_E = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]], dtype=np.float64)


def compute_stress_tensor(fstar, feq, ro, tau, lattice, ny, nx):
    """Cauchy stress (ny, nx, 2, 2) of a D2Q9 state: -(1 - 1/(2 tau)) sum_i
    (f*_i - feq_i) e_ia e_ib, minus rho / 3 on the diagonal.  lattice: an object
    with the velocities as .e (9 x 2), or None for D2Q9."""
    e = D2Q9_E if lattice is None else np.asarray(lattice.e)
    f_neq = fstar - feq
    visc = -(1.0 - 1.0 / (2.0 * tau))
    out = np.zeros((ny, nx, 2, 2))
    for a in range(2):
        for b in range(2):
            out[:, :, a, b] = visc * np.sum(f_neq * (e[:, a] * e[:, b])[None, :], axis=1).reshape(ny, nx)
    ro2 = ro.reshape(ny, nx)
    out[:, :, 0, 0] -= (1.0 / 3.0) * ro2
    out[:, :, 1, 1] -= (1.0 / 3.0) * ro2
    return out


def integrate_surface_force(stress, cx, cy, r, dx, dy, nx, ny, n_points=360):
    """Force on a cylinder: the traction sigma . n, bilinearly interpolated at
    n_points equally spaced points of the circle (cell of each point clamped
    inside the lattice), times the arc length in lattice units, summed point
    by point in order."""
    th = np.linspace(0, 2 * np.pi, n_points, endpoint=False)
    ds = (r / dx) * (2.0 * np.pi / n_points)
    xi = (cx + r * np.cos(th)) / dx
    yi = (cy + r * np.sin(th)) / dy
    i0 = np.clip(np.floor(xi).astype(int), 0, nx - 2)
    j0 = np.clip(np.floor(yi).astype(int), 0, ny - 2)
    fx, fy = xi - i0, yi - j0
    w00, w10, w01, w11 = (1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy
    n = (np.cos(th), np.sin(th))
    F = np.zeros(2)
    for a in range(2):
        t = 0.0
        for b in range(2):
            s_ab = (w00 * stress[j0, i0, a, b] + w10 * stress[j0, i0 + 1, a, b]
                    + w01 * stress[j0 + 1, i0, a, b] + w11 * stress[j0 + 1, i0 + 1, a, b])
            t = t + s_ab * n[b]
        F[a] = np.cumsum(np.concatenate([[0.0], t * ds]))[-1]
    return F
