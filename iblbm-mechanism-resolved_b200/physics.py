"""Host-side setup physics: marker geometry, the MDF relaxation factor, the
oscillation table and rigid-body (Newton-Euler) helpers.

These run once per run (or once per step on a few scalars) on the host in FP64
numpy, as in the reference; the per-node and per-marker work is on the GPU.
"""
from __future__ import annotations

import numpy as np

DELTA_RADIUS = {"peskin4pt": 2, "hat": 1}


def circle_markers(cx, cy, r_domain, lattice_r, dx, spacing_factor, retraction_dx):
    """Equally spaced markers on a circle — iblbm/init.py:211-243 and
    iblbm/physics/markers.py:61-85 (both use this arithmetic).

    Returns (Lx, Ly, Lb, Larea); coordinates in domain units, Larea (the arc
    length per marker) in lattice units."""
    n_param = 2.0 * np.pi * lattice_r / spacing_factor
    step = 1.0 / n_param
    s = np.arange(0, 1.0 + step * 0.5, step)
    s = s[s <= 1.0 + 1e-12]
    if len(s) > 1 and np.abs(s[-1] - 1.0) < step * 0.5:
        s = s[:-1]  # the last point would duplicate the first
    theta = 2.0 * np.pi * s
    radius = r_domain - retraction_dx * dx
    Lx = radius * np.cos(theta) + cx
    Ly = radius * np.sin(theta) + cy
    Lb = len(Lx)
    Larea = 2.0 * np.pi * (lattice_r - retraction_dx) / Lb
    return np.ascontiguousarray(Lx), np.ascontiguousarray(Ly), Lb, Larea


def _phi_np(delta_type, r):
    ar = np.abs(r)
    if delta_type == "hat":
        return np.maximum(1.0 - ar, 0.0)
    out = np.zeros_like(ar)
    near = ar <= 1.0
    far = (~near) & (ar <= 2.0)
    a1, a2 = ar[near], ar[far]
    out[near] = 0.125 * (3.0 - 2.0 * a1 + np.sqrt(np.maximum(1.0 + 4.0 * a1 - 4.0 * a1 ** 2, 0.0)))
    out[far] = 0.125 * (5.0 - 2.0 * a2 - np.sqrt(np.maximum(-7.0 + 12.0 * a2 - 4.0 * a2 ** 2, 0.0)))
    return out


def mdf_relaxation_factor(Lx, Ly, delta_type, Larea, dx):
    """omega = 1 / ||A||_inf of the marker coupling matrix (Zhang et al. 2020,
    Eqs. 39 and 46) — iblbm/ibm/a_norm.py:75-266.

    A_lm = (ds / dx^2) * S_x(l, m) * S_y(l, m) with separable 1-D overlaps
    S_x = sum_i phi(i - x_l) phi(i - x_m) over the integer nodes the two stencils
    share.  Evaluated for all l at once, accumulating over m in order so every
    row sum is formed exactly as the reference's double loop forms it."""
    a = DELTA_RADIUS[delta_type]
    x = np.asarray(Lx, dtype=np.float64) / float(dx)
    y = np.asarray(Ly, dtype=np.float64) / float(dx)
    factor = float(Larea) / (1.0 * 1.0)
    cutoff = 2.0 * a * 1.0
    acc = np.zeros(len(x))
    for m in range(len(x)):
        sums = []
        for pl, pm in ((x, x[m]), (y, y[m])):
            lo = np.maximum(pl, pm) - a * 1.0
            hi = np.minimum(pl, pm) + a * 1.0
            i_lo = np.ceil(lo / 1.0)
            n = np.floor(hi / 1.0) + 1 - i_lo  # node count of the shared support
            s = np.zeros(len(x))
            for t in range(2 * a + 1):
                node = (i_lo + t) * 1.0
                v = _phi_np(delta_type, (node - pl) / 1.0) * _phi_np(delta_type, (node - pm) / 1.0)
                s = s + np.where(t < n, v, 0.0)
            sums.append(s)
        far = (np.abs(x - x[m]) >= cutoff) | (np.abs(y - y[m]) >= cutoff)
        term = factor * sums[0] * sums[1]
        acc = acc + np.where(far | (sums[0] == 0.0) | (sums[1] == 0.0), 0.0, term)
    return 1.0 / float(np.max(acc))


def oscillation_table(max_steps, lattice_u, KC, r_domain, lattice_r):
    """Marker displacement used at each step of the oscillating cylinder.

    iblbm/physics/motion.py:15-52 moves the markers after the collision of step
    t to Lx_c - x(t), x(t) = A sin(2 pi f0 t), and sets the desired velocity to
    (x(t), 0) (the reference's displacement convention); step t + 1 uses them.
    Entry t of the table is the displacement in force during step t (entry 1
    is 0: the initial markers).  Evaluated with the same scalar numpy calls as
    the reference so every entry is bit-identical."""
    f0 = lattice_u / (KC * 2.0 * lattice_r)
    A = KC * 2.0 * r_domain / (2.0 * np.pi)
    table = np.zeros(max_steps + 2)
    for t in range(1, max_steps + 1):
        table[t + 1] = A * np.sin(f0 * 2.0 * np.pi * t)
    return table


def net_gravity(rho_ratio, r_lattice, g_lattice, direction="down"):
    """(rho_s/rho_f - 1) * pi r^2 * g — iblbm/physics/gravity.py:16-34."""
    mag = (rho_ratio - 1.0) * (np.pi * r_lattice ** 2) * g_lattice
    return np.array([mag, 0.0]) if direction == "right" else np.array([0.0, -mag])


def history_increment(model, vel, vel_prev, mass, r_lattice):
    """explicit_history: (m_f/m_s)(U^n - U^{n-1}) — physics/inertia/explicit_history.py:53-66."""
    if model == "explicit_history":
        return (np.pi * r_lattice ** 2 / mass) * (vel - vel_prev)
    return None


def pairwise_tree(n):
    """The summation tree numpy's np.sum applies to n float64 values (its
    pairwise summation: blocks of at most 128 values, each summed in 8 strided
    accumulators combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)) and then its
    tail; a longer range splits at half its length rounded down to a multiple
    of 8 and adds the two halves' sums).  Returns (leaves, inner, levels):
    leaves an (L, 2) int32 array of (offset, length) left to right; inner an
    (I, 2) int32 array of child ids (ids below L are leaves, inner node k has
    id L + k) ordered by depth from the deepest, so children come before
    parents; levels the I + 1 boundaries of the equal-depth groups.  The root
    is the last inner node (or leaf 0 when n <= 128)."""
    leaves, inner = [], []

    def rec(off, m, depth):
        if m <= 128:
            leaves.append((off, m))
            return ("L", len(leaves) - 1)
        m2 = m // 2
        m2 -= m2 % 8
        a = rec(off, m2, depth + 1)
        b = rec(off + m2, m - m2, depth + 1)
        inner.append((a, b, depth))
        return ("I", len(inner) - 1)

    rec(0, int(n), 0)
    L = len(leaves)
    order = sorted(range(len(inner)), key=lambda k: -inner[k][2])  # stable: deepest first
    pos = {k: i for i, k in enumerate(order)}
    ids = lambda c: c[1] if c[0] == "L" else L + pos[c[1]]
    nodes = np.array([[ids(inner[k][0]), ids(inner[k][1])] for k in order], dtype=np.int32).reshape(-1, 2)
    depths = [inner[k][2] for k in order]
    levels = [0] + [i for i in range(1, len(depths)) if depths[i] != depths[i - 1]] + [len(depths)]
    return np.array(leaves, dtype=np.int32).reshape(-1, 2), nodes, np.array(levels, dtype=np.int32)


def pairwise_tree_index(n, leaves, nodes):
    """Look-up tables for evaluating pairwise_tree(n) on the device: lut[i] is
    the leaf holding element 64 i (every leaf but one holds at least 64
    elements, so the leaf of element e is lut[e // 64] or the next one), and
    span[k] the first and last leaf under inner node k."""
    starts = leaves[:, 0]
    lut = (np.searchsorted(starts, np.arange(0, int(n), 64), side="right") - 1).astype(np.int32)
    L = len(leaves)
    span = np.zeros((len(nodes), 2), dtype=np.int32)
    for k, (a, b) in enumerate(nodes):  # children come before parents
        span[k, 0] = a if a < L else span[a - L, 0]
        span[k, 1] = b if b < L else span[b - L, 1]
    return lut, span


def pairwise_sum_sparse(n, idx, val):
    """np.sum of a length-n float64 array that is zero except val at the
    sorted indices idx, evaluated over the pairwise_tree without the zeros
    (a zero term leaves every partial sum unchanged): the host model of the
    device's force sums."""
    leaves, nodes, _ = pairwise_tree(n)
    idx = np.asarray(idx)
    vals = np.zeros(len(leaves) + len(nodes))
    for li, (off, m) in enumerate(leaves):
        lo, hi = np.searchsorted(idx, off), np.searchsorted(idx, off + m)
        if m < 8:
            res = 0.0
            for b in range(lo, hi):
                res += float(val[b])
        else:
            r, res, cut = [0.0] * 8, None, m - m % 8
            tail = []
            for b in range(lo, hi):
                k = int(idx[b]) - off
                if k < cut:
                    r[k % 8] += float(val[b])
                else:
                    tail.append(float(val[b]))
            res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]))
            for v in tail:
                res += v
        vals[li] = res
    for k, (a, b) in enumerate(nodes):
        vals[len(leaves) + k] = vals[a] + vals[b]
    return 0.0 + float(vals[-1] if len(nodes) else vals[0])


def rigid_markers(Lx_c, Ly_c, cx0, cy0, pos, angle=0.0):
    """X = R(angle) (X_c - X_0) + x_p — iblbm/physics/markers.py:23-38."""
    c, s = np.cos(angle), np.sin(angle)
    rx = Lx_c - cx0
    ry = Ly_c - cy0
    return c * rx - s * ry + pos[0], s * rx + c * ry + pos[1]


# ---- decaying Taylor-Green vortex (scenario_type="taylor_green") -------------------
def tg_params(cfg):
    """Half-width and viscosity of the vortex in lattice units
    (iblbm/boundary/tg_analytical.py:49-51)."""
    return 0.5 * (cfg.NN - 1), cfg.lattice_u * (cfg.cylinder_D_ratio * (cfg.NN - 1)) / cfg.Re


def tg_base(X, Y, u0, L):
    """The vortex without its decay factor: (-u0 cos(pi X/L)) sin(pi Y/L) and
    (u0 sin(pi X/L)) cos(pi Y/L).  Times the decay factor this is
    iblbm/diagnostics/core.py:216-241 with the same rounding (the reference
    multiplies by the decay last)."""
    ux = -u0 * np.cos(np.pi * X / L) * np.sin(np.pi * Y / L)
    uy = u0 * np.sin(np.pi * X / L) * np.cos(np.pi * Y / L)
    return ux, uy


def tg_decay_table(cfg, n, dt):
    """exp(-2 nu (pi/L)^2 t) at t = k dt, k = 0 .. n-1, each evaluated as the
    reference evaluates it for one step (iblbm/diagnostics/core.py:238)."""
    L, nu = tg_params(cfg)
    return np.array([np.exp(-2.0 * nu * (np.pi / L) ** 2 * (k * dt)) for k in range(n)], dtype=np.float64)


def tg_face_table(cfg, nx, ny):
    """Velocities before decay of the boundary nodes, (ux, uy) pairs in the order
    of iblbm/boundary/tg_analytical.py:53-163: left face j = 0..ny-1, right face
    j = 0..ny-1, bottom i = 1..nx-2, top i = 1..nx-2, then the corners (0,0),
    (nx-1,0), (0,ny-1), (nx-1,ny-1); coordinates centred on the lattice."""
    L, _ = tg_params(cfg)
    X = np.arange(nx, dtype=float) - (nx - 1) / 2.0
    Y = np.arange(ny, dtype=float) - (ny - 1) / 2.0
    j, i = np.arange(ny), np.arange(1, nx - 1)
    faces = ((np.full_like(j, X[0], dtype=float), Y[j]), (np.full_like(j, X[nx - 1], dtype=float), Y[j]),
             (X[i], np.full_like(i, Y[0], dtype=float)), (X[i], np.full_like(i, Y[ny - 1], dtype=float)),
             (X[np.array([0, nx - 1, 0, nx - 1])], Y[np.array([0, 0, ny - 1, ny - 1])]))
    out = [np.stack(tg_base(xs, ys, cfg.tg_u0, L), axis=1) for xs, ys in faces]
    return np.ascontiguousarray(np.concatenate(out).reshape(-1))


def tg_marker_base(cfg, Lx, Ly, dx, dy, nx, ny):
    """Marker velocities before decay (iblbm/runtime/scenarios/taylor_green.py:21-31)."""
    L, _ = tg_params(cfg)
    ux, uy = tg_base(Lx / dx - (nx - 1) / 2.0, Ly / dy - (ny - 1) / 2.0, cfg.tg_u0, L)
    return np.stack([ux, uy], axis=1)
