"""Fused-step engine: device state in HBM and the per-step launch sequence.

Per timestep the engine launches, on one CUDA stream:

1. ``iblbm_ibm_step_f64`` (one CTA) — band rebuild when markers move, band
   moments, DF / MDF / coupled MDF / DFC;
2. ``iblbm_dense_step_f64`` — pull-stream + closure + band correction +
   moments + collision over the whole lattice, ping-ponging two population
   buffers.

With ``precision="f32"`` the same schedule runs on the shifted FP32 form
(``iblbm_ibm_step_f32`` / ``iblbm_dense_step_f32``): populations are held as
g = f - w in FP32; marker data, per-marker forces and every force sum stay FP64.

Steps between diagnostics are captured once into CUDA graphs and replayed, so
the host issues one graph launch per chunk instead of two kernel launches per
step.  Device layout: populations are pitched structure-of-arrays planes
(q, j, i) with the row pitch rounded up to 32 elements (256-byte rows in FP64).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (BC_IDS, COLL_IDS, DELTA_IDS, DELTA_RADIUS, IBM_IDS, BandView, Case, Dense32Args, DenseArgs,
                   Geom, Ibm32Args, IbmArgs, TILES, check, lib, ptr)
from .physics import (history_increment, mdf_relaxation_factor, net_gravity, oscillation_table,
                      rigid_markers)
from .state import Particle, initial_velocity, initialize

MDF_COUPLED_OMEGA_MAX = 0.8  # iblbm/ibm/multi_particle.py:33
OUT_MOMENTS = 2  # output flag of a step that writes rho and U but not f*
MOVING_ROTATION_OMEGA_MAX = 1.0  # iblbm/ibm/strategies/mdf.py:23


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("iblbm_b200 needs a CUDA device; this package has no CPU fallback")
    return torch


def band_capacity(Lx, Ly, dx, dy, nx, ny, delta_type):
    """Band capacity for markers (Lx, Ly) in domain units: 1.5 x the number of
    distinct stencil nodes plus 256, within [1, min(Lb * S, 2048)] (S stencil
    slots per marker; 2048 is the band kernel's limit)."""
    a = DELTA_RADIUS[delta_type]
    S = (2 * a + 1) ** 2
    Lx, Ly = np.asarray(Lx, dtype=np.float64), np.asarray(Ly, dtype=np.float64)
    ix0 = np.floor(Lx / dx + 0.5).astype(np.int64)
    iy0 = np.floor(Ly / dy + 0.5).astype(np.int64)
    off = np.arange(-a, a + 1)
    ii = np.clip(ix0[:, None, None] + off[None, :, None], 0, nx - 1)
    jj = np.clip(iy0[:, None, None] + off[None, None, :], 0, ny - 1)
    n0 = len(np.unique((jj * nx + ii).ravel()))
    return int(min(max(1, int(1.5 * n0) + 256), len(Lx) * S, 2048))


class Engine:
    """One lattice case on one GPU: FP64 form (the reference's arithmetic) or
    the shifted FP32 form (``precision="f32"``)."""

    def __init__(self, cfg, device=None, precision="f64", device_particles=None, cluster=None):
        """cluster: CTAs of the thread-block cluster that runs the MDF band step
        of one fixed body in the FP64 form (2, 4 or 8; None: 8 where the body
        fits, 0: the single-CTA step)."""
        torch = _torch()
        if precision not in ("f64", "f32"):
            raise ValueError(f"precision='{precision}' (f64 or f32)")
        self.precision = precision
        self.f32 = precision == "f32"
        self.torch = torch
        self.cfg = cfg
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.L = lib()
        st = self.st = initialize(cfg)
        if cfg.ibm_method not in ("DF", "MDF", "DFC"):
            raise KeyError(f"unregistered ibm_method='{cfg.ibm_method}' (DF, MDF, DFC)")
        if cfg.bc_type not in BC_IDS:
            raise KeyError(f"bc_type='{cfg.bc_type}' is not on the accelerated path ({sorted(BC_IDS)})")
        if cfg.delta_type not in DELTA_IDS:
            raise KeyError(f"unknown delta_type='{cfg.delta_type}'")
        if cfg.motion_type not in (None, "oscillating", "sedimentation"):
            raise ValueError(f"motion_type='{cfg.motion_type}' is not supported")
        # the single-particle runtime (iblbm/runtime/scenarios/sedimentation_single.py):
        # its disc steps as a one-particle set, with the single runtime's own force
        # extraction, desired velocity and prescribed-velocity mode
        self.single = cfg.motion_type == "sedimentation" and st.particles is None
        if self.single:
            if cfg.enable_rotation and cfg.rotation_coupling == "iterative" and cfg.ibm_method == "MDF":
                raise NotImplementedError("iterative rotation coupling inside MDF is not on the accelerated path")
            if cfg.settling_inertia_model not in ("none", "explicit_history", "feng_b2"):
                raise NotImplementedError(f"settling_inertia_model='{cfg.settling_inertia_model}' for a single "
                                          "particle is not on the accelerated path")
            # iblbm/physics/sedimentation.py:97-128
            cx, cy = cfg.cylinder_center
            mass = cfg.rho_ratio * np.pi * st.lattice_r ** 2
            st.particles = [Particle(pos=np.array([cx, cy], dtype=float), vel=np.zeros(2), vel_prev=np.zeros(2),
                                     force=np.zeros(2), mass=mass, rho_ratio=cfg.rho_ratio, lattice_r=st.lattice_r,
                                     r_domain=st.r, I_particle=0.5 * mass * st.lattice_r ** 2, Lx_c=st.Lx.copy(),
                                     Ly_c=st.Ly.copy(), Lx=st.Lx.copy(), Ly=st.Ly.copy(), Lb=st.Lb, Larea=st.Larea,
                                     desired_velocity=np.zeros((st.Lb, 2)), cx_init=cx, cy_init=cy)]
        if cfg.motion_type == "sedimentation":
            if cfg.settling_inertia_model == "full_volume":
                raise NotImplementedError("full_volume inertia is not on the accelerated path")
            if cfg.time_integrator not in ("verlet", "euler_explicit"):
                raise NotImplementedError(f"time_integrator='{cfg.time_integrator}' (verlet, euler_explicit)")
            if cfg.ibm_method == "DFC" and any(abs(float(p.Larea) - float(st.particles[0].Larea)) > 1e-12
                                               for p in st.particles):
                # iblbm/ibm/strategies/dfc.py:73-74
                raise ValueError("multi-particle DFC needs equal marker arc lengths")
        # cfg.stream_first (iblbm/runtime/loop.py:60-61,77,86-87) moves each
        # collision from the start of a step to the end of the previous one, with
        # the same inputs: the fused pass (streaming ... collision) already runs
        # in that order, so both schedules are this engine's step bit for bit
        nx, ny = st.nx, st.ny
        self.N = N = nx * ny
        pitch = (nx + 31) // 32 * 32
        self.geom = Geom(nx, ny, pitch, pitch * ny)
        self.qstride = pitch * ny
        dev, f64, i32 = self.dev, torch.float64, torch.int32
        ldt = self.ldt = torch.float32 if self.f32 else torch.float64  # lattice and band fields
        self.stream = lambda: torch.cuda.current_stream(self.dev).cuda_stream
        self.case = Case()
        c = self.case
        c.collision = COLL_IDS[cfg.collision_model]
        c.bc = BC_IDS[cfg.bc_type]
        c.incompressible = int(bool(cfg.incompressible_lbgk))
        c.tau = st.tau
        c.dt = st.dt
        c.s_minus = (1.0 / st.tau_minus) if st.tau_minus is not None else 0.0
        for q in range(9):
            c.S[q] = float(st.S_diag[q]) if st.S_diag is not None else 0.0
        c.inflow_u = st.in_u
        c.dens = st.dens
        # Taylor-Green vortex: the analytic closure on all faces (iblbm/boundary/base.py:52-53)
        # and no IBM step unless tg_with_ibm (iblbm/ibm/dispatch.py:38-39)
        self.tg = cfg.scenario_type == "taylor_green"
        self.no_ibm = self.tg and not cfg.tg_with_ibm
        if self.tg:
            from .physics import tg_face_table, tg_marker_base
            c.bc = BC_IDS["tg_analytical"]
            self.d_tg_face = torch.as_tensor(tg_face_table(cfg, nx, ny), device=dev)
            self.d_tg_step = torch.ones(1, dtype=torch.int64, device=dev)
            self.d_tg_idx = torch.ones(1, dtype=torch.int64, device=dev)
            self.d_tg_cur = torch.ones(1, dtype=f64, device=dev)
            self._tg_table(int(cfg.max_steps) + 2)
            c.tg_face, c.tg_decay = ptr(self.d_tg_face), ptr(self.d_tg_cur)
            if cfg.tg_with_ibm:
                st.desired_velocity = tg_marker_base(cfg, np.asarray(st.Lx), np.asarray(st.Ly), st.dx, st.dy, nx, ny)

        # ---- initial populations: feq(1, U0), then the first collision ----------
        U0 = torch.as_tensor(initial_velocity(cfg, N), device=dev).contiguous()
        ro0 = torch.ones(N, dtype=f64, device=dev)
        feq0 = torch.empty(N * 9, dtype=f64, device=dev)
        s = self.stream()
        check(self.L.iblbm_feq(ptr(ro0), ptr(U0), N, c.incompressible, ptr(feq0), s), "iblbm_feq")
        fib0 = torch.zeros(N * 2, dtype=f64, device=dev)
        fpost0 = torch.empty_like(feq0)
        self._collide_aos(feq0, feq0, U0, fib0, fpost0)
        self.f = [torch.empty(9 * self.qstride, dtype=ldt, device=dev) for _ in range(2)]
        if self.f32:
            check(self.L.iblbm_to_shifted_f32(ptr(fpost0), self.geom, ptr(self.f[0]), s), "iblbm_to_shifted_f32")
        else:
            check(self.L.iblbm_aos_to_soa(ptr(fpost0), self.geom, ptr(self.f[0]), s), "iblbm_aos_to_soa")
        del feq0, fpost0, fib0
        self.uring = [U0.reshape(-1).to(ldt).clone(), U0.reshape(-1).to(ldt).clone()]
        self.ro_out = torch.empty(N, dtype=ldt, device=dev)
        self.U_out = torch.empty(N * 2, dtype=ldt, device=dev)
        self.fstar_out = torch.zeros(9 * self.qstride, dtype=ldt, device=dev)
        self.parity = 0
        self.ttt = 1

        # ---- immersed boundary -------------------------------------------------------
        self.method = cfg.ibm_method
        self.moving = cfg.motion_type is not None
        parts = st.particles
        if parts is not None:
            lbs = [p.Lb for p in parts]
            self.larea_h = np.array([p.Larea for p in parts])
        else:
            lbs = [st.Lb]
            self.larea_h = np.array([st.Larea])
        self.P = len(lbs)
        self.Lb = int(sum(lbs))
        moff = np.concatenate([[0], np.cumsum(lbs)]).astype(np.int32)
        S = (2 * DELTA_RADIUS[cfg.delta_type] + 1) ** 2
        self.B = B = self._band_capacity(S)
        t = lambda n, dt=f64: torch.zeros(max(int(n), 1), dtype=dt, device=dev)
        self.d_moff = torch.as_tensor(moff, device=dev)
        self.d_moff_set = torch.as_tensor(np.array([0, self.Lb], dtype=np.int32), device=dev)
        self.d_larea = torch.as_tensor(self.larea_h, device=dev)
        self.d_Lx, self.d_Ly, self.d_dv = t(self.Lb), t(self.Lb), t(2 * self.Lb)
        self._upload_markers()
        self.d_box = t(4, i32)
        self.d_map = torch.full((N,), -1, dtype=i32, device=dev)
        self.d_nodes, self.d_count = t(B, i32), t(1, i32)
        self.d_fib, self.d_df = t(2 * B, ldt), t(9 * B, ldt)
        self.d_fib_part = t(2 * B * self.P, ldt)
        delta_id = DELTA_IDS[cfg.delta_type]
        self.d_scr = t(self.L.iblbm_ibm_scratch_doubles(self.Lb, B, self.P), ldt)
        self.d_iscr = t(self.L.iblbm_ibm_scratch_ints(self.Lb, B, delta_id), i32)
        cache_ints = self.L.iblbm_ibm32_list_cache_ints if self.f32 else self.L.iblbm_ibm_list_cache_ints
        self.d_lists = t(cache_ints(self.Lb, B, delta_id), i32)
        # the cluster plan of a fixed body's FP64 MDF step (built at each band rebuild)
        self.cluster, self.d_plan = 0, None
        if not self.f32 and cfg.ibm_method == "MDF" and self.P == 1 and not self.moving and cluster != 0:
            size = 8 if cluster is None else int(cluster)
            n = self.L.iblbm_ibm_cluster_plan_ints(self.Lb, delta_id, size)
            if n > 0:
                self.cluster, self.d_plan = size, t(n, i32)
            elif cluster is not None:
                raise ValueError(f"cluster={cluster}: a body of {self.Lb} markers does not fit")
        self.d_excl = torch.zeros(2, 4, dtype=i32, device=dev)
        self.d_Lux, self.d_Luy, self.d_Lfx, self.d_Lfy = (t(self.Lb) for _ in range(4))
        self.d_dfc_force = t(2 * self.Lb)
        self.d_stats, self.d_dstats = t(5, i32), t(2)
        self.d_lambda, self.d_lambda_valid = t(self.Lb), t(1, i32)
        self.d_counter = t(1, i32)
        # diagnostics reduced on the device: force coefficients ring, convergence error
        self.ring_len = 4096
        self.d_ring = torch.zeros(self.ring_len, 5, dtype=f64, device=dev)
        self.d_ring_pos = t(1, i32)
        self.ring_read = 0  # entries queued so far (the host's copy of the device counter)
        self.d_diag_part = t(self.L.iblbm_diag_partials(N))
        self.d_diag_ticket = t(1, i32)
        self.d_uprev = None
        self.d_vchange = t(3)
        self.xt = None
        if cfg.motion_type == "oscillating":
            table = oscillation_table(cfg.max_steps + 2, cfg.lattice_u, cfg.KC, st.r, st.lattice_r)
            self.xt = torch.as_tensor(table, device=dev)
            self.d_Lxc = torch.as_tensor(st.Lx, device=dev)
            self.d_Lyc = torch.as_tensor(st.Ly, device=dev)
            self.d_counter.fill_(1)
        self.omega = 1.0
        if self.method == "MDF":
            # iblbm/ibm/strategies/mdf.py:26-38 (markers of the initial cylinder)
            self.omega = mdf_relaxation_factor(st.Lx, st.Ly, cfg.delta_type, float(st.Larea), float(st.dx))
            if cfg.motion_type == "sedimentation" and cfg.enable_rotation:
                self.omega = min(float(self.omega), MOVING_ROTATION_OMEGA_MAX)
        self.ibm_args = [self._make_ibm_args(p) for p in (0, 1)]
        self.tile = "rows2"  # FP32 pass tile shape (iblbm_b200._lib.TILES)
        self.d_pipe_status = torch.zeros(1, dtype=i32, device=dev)
        self.graphs = {}
        self._make_dense_variants()
        # free particles: their Verlet or explicit Euler step on the device by
        # default (in the FP64 form its force and torque sums follow numpy's
        # pairwise order, so it equals the host step bit for bit);
        # device_particles=False keeps the host step.  Rotating FP64 runs keep
        # the host step unless asked: their markers turn by the device's cos and
        # sin, which may differ from the host's in the last bit
        self.dev_particles = False
        self.part_after_lattice = self.moments_always = False
        self._torque_ij = None
        if st.particles is not None:
            rot = bool(cfg.enable_rotation)
            default = not (rot and not self.f32)
            self.dev_particles = default if device_particles is None else bool(device_particles)
            if self.single and cfg.prescribed_velocity is not None and (rot or cfg.time_integrator != "verlet"):
                # a disc moved at a prescribed velocity steps on the host with
                # rotation or the Euler integrator set (the host step ignores both)
                if device_particles:
                    raise NotImplementedError("a prescribed-velocity disc with rotation or explicit Euler set "
                                              "steps on the host")
                self.dev_particles = False
            if self.dev_particles:
                self._setup_device_particles()
        self.side = torch.cuda.Stream(self.dev, priority=-1)
        self.ev_bulk = torch.cuda.Event()
        self.ev_side = torch.cuda.Event()
        # the particle step runs beside the box pass (both only read the band
        # step's output) on a stream of its own
        self.pstream = torch.cuda.Stream(self.dev, priority=-1) if self.dev_particles else None
        self.ev_band = torch.cuda.Event()
        self.ev_part = torch.cuda.Event()
        self.overlap = not self.tg  # the per-step decay factor needs one stream
        self.rebuild_next = True
        self.last_out_step = 0

    def _setup_device_particles(self):
        from ._lib import INERTIA_IDS, PARTICLE_CONSTS, PARTICLE_STATE, ParticlesArgs
        torch, st, cfg = self.torch, self.st, self.cfg
        if cfg.settling_inertia_model not in INERTIA_IDS:
            raise NotImplementedError(f"inertia model '{cfg.settling_inertia_model}' on the device")
        ps = st.particles
        state = np.zeros((len(ps), PARTICLE_STATE))
        consts = np.zeros((len(ps), PARTICLE_CONSTS))
        for k, p in enumerate(ps):
            state[k, 0:2] = p.pos
            state[k, 2:4] = p.vel
            state[k, 4:6] = p.vel_prev
            state[k, 6:8] = p.vel_half
            state[k, 8:10] = p.force
            state[k, 10:12] = p.pos
            state[k, 12:16] = [p.omega, p.omega_half, p.angle, p.torque]
            state[k, 16:18] = p.vel_half
            state[k, 18:22] = [p.omega_half, p.angle, p.omega, p.l_int_prev]
            g = net_gravity(p.rho_ratio, p.lattice_r, st.gravity_lattice, cfg.gravity_direction)
            consts[k] = [p.mass, 1.0 / p.rho_ratio, np.pi * p.lattice_r ** 2 / p.mass, g[0], g[1], p.cx_init,
                         p.cy_init, p.I_particle, p.r_domain, float(p.Larea)]
        self.d_pstate = torch.as_tensor(state.reshape(-1), device=self.dev)
        self.d_pconsts = torch.as_tensor(consts.reshape(-1), device=self.dev)
        self.d_Lxc_all = torch.as_tensor(np.concatenate([p.Lx_c for p in ps]), device=self.dev)
        self.d_Lyc_all = torch.as_tensor(np.concatenate([p.Ly_c for p in ps]), device=self.dev)
        self.d_pforces = torch.zeros(2 * len(ps), dtype=torch.float64, device=self.dev)
        a = ParticlesArgs()
        a.n_particles, a.model, a.fib_f32 = len(ps), INERTIA_IDS[cfg.settling_inertia_model], int(self.f32)
        a.moff, a.Lx_c, a.Ly_c = ptr(self.d_moff), ptr(self.d_Lxc_all), ptr(self.d_Lyc_all)
        a.Lx, a.Ly, a.dvel = ptr(self.d_Lx), ptr(self.d_Ly), ptr(self.d_dv)
        a.state, a.consts = ptr(self.d_pstate), ptr(self.d_pconsts)
        a.dt, a.dx = float(st.dt), float(st.dx)
        a.band_fib_part, a.band_count, a.band_capacity = ptr(self.d_fib_part), ptr(self.d_count), self.B
        a.forces_out = ptr(self.d_pforces)
        a.rotation = int(bool(cfg.enable_rotation))
        a.semi_implicit = int(cfg.rotation_coupling == "semi_implicit")
        a.euler_trapezoidal = int(cfg.sedimentation_euler_update_scheme == "trapezoidal")
        a.nx, a.dy, a.n_nodes, a.band_nodes = st.nx, float(st.dy), self.N, ptr(self.d_nodes)
        # Verlet: a half step before the first band kernel, then the full step of
        # each timestep and the half step of the next; explicit Euler: the whole
        # step after each band kernel, from the markers the host set up
        self.part_phase = 4 if cfg.time_integrator == "euler_explicit" else 3
        # a rotating Euler step reads this step's rho and U (the fluid's angular
        # momentum inside each disc): every step writes them, and the particle
        # launch follows the whole lattice pass
        self.part_after_lattice = self.part_phase == 4 and bool(cfg.enable_rotation)
        self.moments_always = self.part_after_lattice
        # DF and DFC particles: force and torque from the markers' forces
        # (iblbm/ibm/forcing.py:262-275, iblbm/ibm/strategies/dfc.py:114-128)
        # (the single-particle runtime sums the DF field like MDF's)
        a.lagrangian = {"DF": 0 if self.single else 1, "DFC": 2}.get(self.method, 0)
        a.half_kick_omega = int(self.single)
        if self.single and cfg.prescribed_velocity is not None:
            a.prescribed = 1
            a.prescribed_velocity[0], a.prescribed_velocity[1] = (float(x) for x in cfg.prescribed_velocity)
        a.Lfx, a.Lfy, a.dfc_force = ptr(self.d_Lfx), ptr(self.d_Lfy), ptr(self.d_dfc_force)
        cap = max(p.Lb for p in ps) if a.lagrangian else 0
        if self.part_after_lattice:
            cap = max([cap] + [(2 * (int(p.r_domain / st.dx) + 2) + 1) ** 2 for p in ps])
            a.rho, a.U, a.moments_f32, a.ny = ptr(self.ro_out), ptr(self.U_out), int(self.f32), st.ny
        if cap:
            self.d_lint = torch.zeros(cap, dtype=torch.float64, device=self.dev)
            a.lint_scratch, a.lint_capacity = ptr(self.d_lint), cap
        if not self.f32 and not a.lagrangian:
            # the FP64 form sums the forces in numpy's pairwise order over the
            # dense lattice field, so the device step equals the host step bit
            # for bit; the FP32 form keeps the cheaper fixed-order sum
            from .physics import pairwise_tree, pairwise_tree_index
            leaves, inner, levels = pairwise_tree(self.N)
            lut, span = pairwise_tree_index(self.N, leaves, inner)
            z2 = np.zeros(2, np.int32)
            self.d_pw_leaf = torch.as_tensor(leaves.reshape(-1), device=self.dev)
            self.d_pw_node = torch.as_tensor(inner.reshape(-1) if inner.size else z2, device=self.dev)
            self.d_pw_level = torch.as_tensor(levels, device=self.dev)
            self.d_pw_lut = torch.as_tensor(lut, device=self.dev)
            self.d_pw_span = torch.as_tensor(span.reshape(-1) if span.size else z2, device=self.dev)
            self.d_pw_scratch = torch.zeros((len(leaves) + len(inner)) * 3 * len(ps), dtype=torch.float64,
                                            device=self.dev)
            a.pw_leaves, a.pw_internal, a.pw_levels = len(leaves), len(inner), len(levels) - 1
            a.pw_leaf, a.pw_node, a.pw_level = ptr(self.d_pw_leaf), ptr(self.d_pw_node), ptr(self.d_pw_level)
            a.pw_lut, a.pw_span, a.pw_scratch = ptr(self.d_pw_lut), ptr(self.d_pw_span), ptr(self.d_pw_scratch)
        self.part_args = a
        self.part_started = False

    def _particles(self, stream, phase):
        a = self.part_args
        a.phase = phase
        check(self.L.iblbm_particles_step_f64(ctypes.byref(a), stream), "iblbm_particles_step_f64")

    def pull_particles(self):
        """Copy the device particle state of the last completed step (position,
        velocities, force, angular velocity, angle, torque) into the host
        Particle objects, with that step's markers and desired velocities."""
        if not self.dev_particles:
            return
        self.join()
        s = self.d_pstate.reshape(-1, _lib.PARTICLE_STATE).cpu().numpy()
        euler = self.part_phase == 4
        if euler:  # the device holds the markers the Euler step left for the next step
            Lx, Ly = self.d_Lx.cpu().numpy(), self.d_Ly.cpu().numpy()
            dv = self.d_dv[: 2 * self.Lb].reshape(-1, 2).cpu().numpy()
            moff = self.d_moff.cpu().numpy()
        rot, semi = bool(self.cfg.enable_rotation), self.cfg.rotation_coupling == "semi_implicit"
        for k, p in enumerate(self.st.particles):
            p.pos = s[k, 0:2].copy()
            p.vel = s[k, 2:4].copy()
            p.vel_prev = s[k, 4:6].copy()
            p.vel_half = s[k, 6:8].copy()
            p.force = s[k, 8:10].copy()
            p.fib_force = p.force.copy()
            p.omega, p.omega_half, p.angle, p.torque = (float(x) for x in s[k, 12:16])
            p.l_int_prev = float(s[k, 21])
            if euler:
                p.Lx, p.Ly = Lx[moff[k]:moff[k + 1]].copy(), Ly[moff[k]:moff[k + 1]].copy()
                p.desired_velocity = dv[moff[k]:moff[k + 1]].copy()
            else:  # the markers of the last step (the device holds the next step's)
                om = p.omega_half if self.single else float(s[k, 20])
                self._set_markers(p, p.vel_half, om if rot and semi else 0.0)

    def _band_capacity(self, S):
        st = self.st
        if st.particles is not None:
            Lx = np.concatenate([p.Lx for p in st.particles])
            Ly = np.concatenate([p.Ly for p in st.particles])
        else:
            Lx, Ly = st.Lx, st.Ly
        return band_capacity(Lx, Ly, st.dx, st.dy, st.nx, st.ny, self.cfg.delta_type)

    # ------------------------------------------------------------------------------
    def _collide_aos(self, fstar, feq, U, fib, out):
        c, s, N = self.case, self.stream(), self.N
        if c.collision == 0:
            rc = self.L.iblbm_collision_bgk(ptr(fstar), ptr(feq), ptr(U), ptr(fib), N, c.tau, c.dt, ptr(out), s)
        elif c.collision == 1:
            rc = self.L.iblbm_collision_trt(ptr(fstar), ptr(feq), ptr(U), ptr(fib), N, c.tau, self.st.tau_minus,
                                            c.dt, ptr(out), s)
        else:
            Sd = (ctypes.c_double * 9)(*[float(v) for v in self.st.S_diag])
            rc = self.L.iblbm_collision_cm_mrt(ptr(fstar), ptr(U), ptr(fib), N, Sd, c.dt, ptr(out), s)
        check(rc, "initial collision")

    def _tg_table(self, n):
        """Decay factors of steps 0 .. n-1 on the device (host-computed with numpy,
        as the reference computes them)."""
        from .physics import tg_decay_table
        self.d_tg_table = self.torch.as_tensor(tg_decay_table(self.cfg, n, self.st.dt), device=self.dev)
        self.graphs = {}

    def _tg_tick(self):
        """This step's decay factor into the scalar the closures and the band
        kernel read, then the step counter advances (graph-capturable).  The host
        keeps the table longer than the steps taken; the index is clamped to it on
        the device all the same, so no step can read outside the table."""
        torch = self.torch
        torch.clamp(self.d_tg_step, max=self.d_tg_table.numel() - 1, out=self.d_tg_idx)
        torch.index_select(self.d_tg_table, 0, self.d_tg_idx, out=self.d_tg_cur)
        self.d_tg_step.add_(1)

    def _upload_markers(self):
        st = self.st
        if st.particles is not None:
            Lx = np.concatenate([p.Lx for p in st.particles])
            Ly = np.concatenate([p.Ly for p in st.particles])
            dv = np.concatenate([p.desired_velocity for p in st.particles])
        else:
            Lx, Ly, dv = st.Lx, st.Ly, st.desired_velocity
        tt = self.torch
        self.d_Lx.copy_(tt.as_tensor(np.ascontiguousarray(Lx, dtype=np.float64)))
        self.d_Ly.copy_(tt.as_tensor(np.ascontiguousarray(Ly, dtype=np.float64)))
        self.d_dv.copy_(tt.as_tensor(np.ascontiguousarray(dv, dtype=np.float64).reshape(-1)))

    def _make_ibm_args(self, parity):
        cfg, a = self.cfg, (Ibm32Args if self.f32 else IbmArgs)()
        a.g, a.c = self.geom, self.case
        a.method = IBM_IDS[self.method]
        a.delta_type = DELTA_IDS[cfg.delta_type]
        a.rebuild = 1
        a.n_particles, a.lb_total = self.P, self.Lb
        if self.method == "DFC" and self.P > 1:
            # iblbm/ibm/strategies/dfc.py:56-110: every particle's markers as one point
            # set with the first particle's arc length, lambda of that set each step
            a.n_particles = 1
        a.moff, a.Lx, a.Ly, a.dvel, a.larea = (ptr(x) for x in (self.d_moff, self.d_Lx, self.d_Ly, self.d_dv,
                                                                 self.d_larea))
        if self.method == "DFC" and self.P > 1:
            a.moff = ptr(self.d_moff_set)
        a.dx, a.dy = self.st.dx, self.st.dy
        if self.tg and cfg.tg_with_ibm:
            a.dvel_scale = ptr(self.d_tg_cur)
        if self.xt is not None:
            a.Lx_c, a.Ly_c, a.xt_table, a.step_counter = ptr(self.d_Lxc), ptr(self.d_Lyc), ptr(self.xt), ptr(
                self.d_counter)
            a.xt_len = int(self.xt.numel())
        a.mdf_iterations = int(cfg.mdf_iterations)
        a.mdf_min_iterations = int(cfg.mdf_min_iterations)
        a.mdf_coupled = int(self.P >= 2)
        a.mdf_omega, a.mdf_tol, a.mdf_omega_max = float(self.omega), float(cfg.mdf_tolerance), MDF_COUPLED_OMEGA_MAX
        a.lambda_, a.lambda_valid = ptr(self.d_lambda), ptr(self.d_lambda_valid)
        a.dfc_cache_lambda = int(cfg.motion_type is None)
        a.correction_scale = 1.0
        a.fpost_prev, a.uring_prev = ptr(self.f[parity]), ptr(self.uring[parity])
        a.box, a.map, a.band_nodes, a.band_count = (ptr(x) for x in (self.d_box, self.d_map, self.d_nodes,
                                                                     self.d_count))
        a.list_cache = ptr(self.d_lists)
        a.excl_cur = ptr(self.d_excl[parity])
        a.excl_next = ptr(self.d_excl[1 - parity])
        a.band_capacity, a.box_capacity = self.B, self.N
        a.band_fib, a.band_df, a.band_fib_part = ptr(self.d_fib), ptr(self.d_df), ptr(self.d_fib_part)
        a.scratch, a.iscratch = ptr(self.d_scr), ptr(self.d_iscr)
        a.Lux, a.Luy, a.Lfx, a.Lfy = (ptr(x) for x in (self.d_Lux, self.d_Luy, self.d_Lfx, self.d_Lfy))
        a.dfc_force = ptr(self.d_dfc_force)
        a.stats, a.dstats = ptr(self.d_stats), ptr(self.d_dstats)
        if self.d_plan is not None:
            a.cluster_plan, a.cluster_size = ptr(self.d_plan), self.cluster
        return a

    def _make_dense_variants(self):
        """Dense pass variants per parity and output flag (0: none, 1: rho, U and
        f*, 2: rho and U only): whole lattice, bulk (skips the exclusion box), box
        (only the exclusion box)."""
        outs = (False, True, OUT_MOMENTS)
        self.dense_full = [[self._make_dense_args(p, out, "full") for out in outs] for p in (0, 1)]
        self.dense_bulk = [[self._make_dense_args(p, out, "bulk") for out in outs] for p in (0, 1)]
        self.dense_box = [[self._make_dense_args(p, out, "box") for out in outs] for p in (0, 1)]

    def set_mlp(self, mode, net=None):
        """Learned MDF warm start of the FP32 form (single-body MDF): mode bit 1
        records each step's marker features and accumulated forces into
        d_mlp_feat (Lb x 64) / d_mlp_targ (Lb x 2); bit 2 starts every MDF loop
        from the forces that `net` (an iblbm_b200.learned.MdfNet) predicts."""
        if not self.f32:
            raise NotImplementedError("the learned warm start belongs to the FP32 form")
        if mode and (self.method != "MDF" or self.P != 1):
            raise NotImplementedError("the learned warm start covers single-body MDF")
        if (mode & 2) and net is None:
            raise ValueError("mode 2 needs a network")
        torch = self.torch
        if mode & 1 and not hasattr(self, "d_mlp_feat"):
            self.d_mlp_feat = torch.zeros(self.Lb, 64, dtype=torch.float32, device=self.dev)
            self.d_mlp_targ = torch.zeros(self.Lb, 2, dtype=torch.float32, device=self.dev)
        self.mlp_net = net
        cfg = self.cfg
        uref = cfg.lattice_u if cfg.motion_type == "oscillating" else self.st.in_u
        for a in self.ibm_args:
            a.mlp_mode = int(mode)
            a.mlp_uref = float(uref) if uref else 1.0
            a.mlp_re = float(cfg.Re)
            a.mlp_params = ptr(net.params) if (net is not None and mode & 2) else 0
            a.mlp_features = ptr(self.d_mlp_feat) if mode & 1 else 0
            a.mlp_targets = ptr(self.d_mlp_targ) if mode & 1 else 0
        self.graphs = {}

    def set_tile(self, tile):
        """Tile shape of the FP32 whole-lattice/bulk pass (a key of
        iblbm_b200._lib.TILES).  Drops captured graphs."""
        if tile not in TILES:
            raise ValueError(f"tile {tile!r} (one of {sorted(TILES)})")
        self.tile = tile
        self._make_dense_variants()
        self.graphs = {}

    def _make_dense_args(self, parity, outputs, mode):
        a = Dense32Args() if self.f32 else DenseArgs()
        if self.f32:
            a.tile = TILES[self.tile]
            a.status = ptr(self.d_pipe_status)
        a.g, a.c = self.geom, self.case
        a.ibm = 0 if (mode == "bulk" or self.no_ibm) else IBM_IDS[self.method]
        a.fpost_prev, a.fpost_next = ptr(self.f[parity]), ptr(self.f[1 - parity])
        a.uring_prev, a.uring_next = ptr(self.uring[parity]), ptr(self.uring[1 - parity])
        a.band = BandView(ptr(self.d_box), ptr(self.d_map), ptr(self.d_fib), ptr(self.d_df))
        if outputs:
            a.ro_out, a.U_out = ptr(self.ro_out), ptr(self.U_out)
            a.fstar_out = 0 if outputs == OUT_MOMENTS else ptr(self.fstar_out)
        if mode == "bulk":
            a.skip_box = ptr(self.d_excl[parity])
        elif mode == "box":
            a.only_box = ptr(self.d_excl[parity])
            a.box_blocks = 2 * 148
        return a

    # ------------------------------------------------------------------------------
    def _ibm(self, stream, excl_check):
        ia = self.ibm_args[self.parity]
        ia.rebuild = 1 if (self.rebuild_next or self.moving) else 0
        ia.excl_cur = ptr(self.d_excl[self.parity]) if excl_check else 0
        if self.f32:
            check(self.L.iblbm_ibm_step_f32(ctypes.byref(ia), stream), "iblbm_ibm_step_f32")
        else:
            check(self.L.iblbm_ibm_step_f64(ctypes.byref(ia), stream), "iblbm_ibm_step_f64")
        self.rebuild_next = False

    def _dense(self, variant, outputs, stream):
        if not outputs and self.moments_always:
            outputs = OUT_MOMENTS
        da = variant[self.parity][2 if outputs == OUT_MOMENTS else (1 if outputs else 0)]
        if self.f32:
            check(self.L.iblbm_dense_step_f32(ctypes.byref(da), stream), "iblbm_dense_step_f32")
        else:
            check(self.L.iblbm_dense_step_f64(ctypes.byref(da), stream), "iblbm_dense_step_f64")

    def _step_serial(self, outputs=False, events=None):
        """One timestep on the current stream: band kernel, then the whole lattice.
        With events=(e0, e1, e2): recorded before, between and after the kernels."""
        torch = self.torch
        s = self.stream()
        if events:
            events[0].record()
        if self.tg:
            self._tg_tick()
        if self.dev_particles and not self.part_started:
            if self.part_phase == 3:
                self._particles(s, 2)  # half step of the first timestep
            else:
                self._upload_markers()  # the Euler step starts from the set-up markers
            self.part_started = True
        if self.no_ibm:
            self.rebuild_next = False
        else:
            self._ibm(s, excl_check=False)
        if self.dev_particles and not self.part_after_lattice:
            self._particles(s, self.part_phase)  # full step of this timestep (and half step of the next)
        if events:
            events[1].record()
        self._dense(self.dense_full, outputs, s)
        if self.dev_particles and self.part_after_lattice:
            self._particles(s, self.part_phase)
        if events:
            events[2].record()
        self.parity ^= 1

    def _step_overlapped(self, outputs=False, bulk_events=None):
        """One timestep with the band kernel and the box pass on the side stream,
        concurrent with the bulk pass on the current stream.

        Dependencies (n = this step): band(n) and box(n) wait for bulk(n-1);
        bulk(n) waits for box(n-1).  Reads of f_post(n-1) and writes of f_post(n)
        therefore never race, and the ping-pong buffers are safe to reuse.  A
        device particle step runs on its own stream after band(n), beside box(n);
        bulk(n)'s event waits for it, so band(n+1) reads the markers it wrote."""
        torch = self.torch
        main = torch.cuda.current_stream(self.dev)
        side = self.side
        side.wait_event(self.ev_bulk)
        self._ibm(side.cuda_stream, excl_check=True)
        beside = self.dev_particles and not self.part_after_lattice
        if beside:
            self.ev_band.record(side)
            self.pstream.wait_event(self.ev_band)
            self._particles(self.pstream.cuda_stream, self.part_phase)
            self.ev_part.record(self.pstream)
        self._dense(self.dense_box, outputs, side.cuda_stream)
        main.wait_event(self.ev_side)
        self.ev_side.record(side)
        if bulk_events:
            bulk_events[0].record(main)
        self._dense(self.dense_bulk, outputs, main.cuda_stream)
        if bulk_events:
            bulk_events[1].record(main)
        if beside:
            main.wait_event(self.ev_part)  # the next band step reads the markers it wrote
        if self.dev_particles and self.part_after_lattice:
            main.wait_event(self.ev_side)  # this step's box pass
            self._particles(main.cuda_stream, self.part_phase)
        self.ev_bulk.record(main)
        self.parity ^= 1

    def join(self):
        """Make the current stream wait for the side stream's work."""
        self.torch.cuda.current_stream(self.dev).wait_event(self.ev_side)

    def fence(self):
        """Order everything queued so far on the current stream before the next
        step's work on both streams."""
        main = self.torch.cuda.current_stream(self.dev)
        self.ev_bulk.record(main)
        self.ev_side.record(main)

    def _launch(self, outputs=False, events=None):
        """One timestep: serial for the first step (and when overlap is off), else overlapped."""
        if self.rebuild_next or not self.overlap or (self.st.particles is not None and not self.dev_particles):
            self._step_serial(outputs, events)
            main = self.torch.cuda.current_stream(self.dev)
            self.ev_bulk.record(main)
            self.ev_side.record(main)
        else:
            self._step_overlapped(outputs)
            if outputs or events is not None:
                self.join()

    def _graph(self, length):
        key = (self.parity, length)
        g = self.graphs.get(key)
        if g is None:
            torch = self.torch
            cap = torch.cuda.Stream(self.dev)
            cap.wait_stream(torch.cuda.current_stream(self.dev))
            cap.wait_stream(self.side)
            g = torch.cuda.CUDAGraph()
            p0 = self.parity
            with torch.cuda.stream(cap):
                with torch.cuda.graph(g, stream=cap):
                    # fork: the side stream's first wait must be on captured work
                    self.ev_bulk.record(cap)
                    self.ev_side.record(cap)
                    for _ in range(length):
                        self._launch(False)
                    self.join()
            torch.cuda.current_stream(self.dev).wait_stream(cap)
            self.parity = p0  # capture does not execute; restore the bookkeeping
            self.graphs[key] = g
        return g

    def step_io(self, host_in, host_out, wait=True):
        """One timestep with its host I/O, as a host program drives a fixed body:
        marker positions and desired velocities ([Lx, Ly, dvel], 4 Lb FP64
        values) from pinned host memory host_in, the step, and the total force
        on the band (2 FP64 values) into pinned host memory host_out.  Replayed
        from one CUDA graph per parity and buffer pair (copies included).  With
        wait, returns when host_out holds this step's force; otherwise returns
        at once with an event that completes then (see Batch.step_io)."""
        torch = self.torch
        if self.moving or self.st.particles is not None:
            raise NotImplementedError("step_io drives fixed bodies (moving markers come from the device)")
        if self.rebuild_next:
            self.advance(1, outputs_last=False)
        if self.tg and self.ttt + 1 >= self.d_tg_table.numel():
            self._tg_table(2 * (self.ttt + 1) + 2)  # drops the captured graphs
        self.join()  # before a capture: events recorded inside one cannot be waited on outside
        main = torch.cuda.current_stream(self.dev)
        key = ("io", self.parity, host_in.data_ptr(), host_out.data_ptr())
        g = self.graphs.get(key)
        if g is None:
            Lb, nb = self.Lb, int(self.d_count.item())
            cap = torch.cuda.Stream(self.dev)
            cap.wait_stream(main)
            cap.wait_stream(self.side)
            g = torch.cuda.CUDAGraph()
            p0 = self.parity
            with torch.cuda.stream(cap):
                with torch.cuda.graph(g, stream=cap):
                    self.ev_bulk.record(cap)
                    self.ev_side.record(cap)  # the bulk pass needs no marker data
                    # markers in ahead of the band kernel, on the stream it runs on
                    copy_stream = self.side if self.overlap else cap
                    copy_stream.wait_event(self.ev_bulk)
                    with torch.cuda.stream(copy_stream):
                        self.d_Lx.copy_(host_in[:Lb], non_blocking=True)
                        self.d_Ly.copy_(host_in[Lb:2 * Lb], non_blocking=True)
                        self.d_dv.copy_(host_in[2 * Lb:4 * Lb], non_blocking=True)
                    self._launch(False)
                    self.join()
                    host_out.copy_(self.d_fib[: 2 * nb].view(nb, 2).double().sum(0), non_blocking=True)
            main.wait_stream(cap)
            self.parity = p0
            self.graphs[key] = g
        g.replay()
        self.parity ^= 1
        self.ttt += 1
        self.fence()
        if wait:
            main.synchronize()
            return None
        done = torch.cuda.Event()
        done.record(main)
        return done

    def advance(self, nsteps, outputs_last=True, use_graph=True):
        """Advance nsteps timesteps; the last one writes rho/U/f* when outputs_last."""
        if nsteps <= 0:
            return
        if self.tg and self.ttt + nsteps >= self.d_tg_table.numel():
            self._tg_table(2 * (self.ttt + nsteps) + 2)
        if self.st.particles is not None and not self.dev_particles:
            for k in range(nsteps):
                self._sedimentation_step(outputs=outputs_last and k == nsteps - 1)
            return
        if self.rebuild_next:
            self._launch(outputs=(outputs_last and nsteps == 1))
            self.ttt += 1
            nsteps -= 1
        body = nsteps - 1 if outputs_last else nsteps
        if body > 0:
            if use_graph and body >= 4:
                self.join()
                g = self._graph(body)
                g.replay()
                self.parity ^= (body & 1)
                main = self.torch.cuda.current_stream(self.dev)
                self.ev_bulk.record(main)
                self.ev_side.record(main)
            else:
                for _ in range(body):
                    self._launch(False)
                self.join()
            self.ttt += body
        if outputs_last and nsteps > 0:
            self._launch(True)
            self.ttt += 1
            self.last_out_step = self.ttt - 1
        if self.dev_particles and outputs_last:
            self.pull_particles()

    # ---- multi-particle sedimentation (host Newton-Euler, as the reference) ----------
    def _sedimentation_step(self, outputs):
        if self.cfg.time_integrator == "euler_explicit":
            return self._sedimentation_step_euler(outputs)
        cfg, st = self.cfg, self.st
        rot = cfg.enable_rotation
        if self.single and cfg.prescribed_velocity is not None:
            return self._sedimentation_step_prescribed(outputs)
        for p in st.particles:  # runtime/scenarios/sedimentation_multi.py:36-80
            F = p.force + net_gravity(p.rho_ratio, p.lattice_r, st.gravity_lattice, cfg.gravity_direction)
            vel_half = p.vel + 0.5 * st.dt * F / p.mass
            hist = history_increment(cfg.settling_inertia_model, p.vel, p.vel_prev, p.mass, p.lattice_r)
            if hist is not None:
                vel_half = vel_half + 0.5 * hist
            p.pos = p.pos + st.dt * vel_half * st.dx
            if rot:  # angular half kick, physics/rigid_body.py:65-74
                p.omega_half = p.omega + 0.5 * st.dt * p.torque / p.I_particle
                p.angle += st.dt * p.omega_half
            # U + omega x r (physics/markers.py:41-60) for semi-implicit coupling: the
            # multi-particle runtime takes the last step's omega, the single-particle
            # runtime this step's half-kicked one (sedimentation_single.py:148-158)
            om = (p.omega_half if self.single else p.omega) if rot else 0.0
            self._set_markers(p, vel_half, om if cfg.rotation_coupling == "semi_implicit" else 0.0)
            p.vel_half = vel_half
        self._upload_markers()
        self._launch(outputs)
        self.ttt += 1
        if outputs:
            self.last_out_step = self.ttt - 1
        forces, torques = self.particle_forces(torques=rot)
        for k, (p, fp) in enumerate(zip(st.particles, forces)):  # runtime/scenarios/sedimentation_multi.py:83-111
            if rot:  # physics/rigid_body.py:77-82
                p.omega = p.omega_half + 0.5 * st.dt * torques[k] / p.I_particle
                p.torque = torques[k]
            p.fib_force = fp
            F = fp + net_gravity(p.rho_ratio, p.lattice_r, st.gravity_lattice, cfg.gravity_direction)
            vel_new = p.vel_half + 0.5 * st.dt * F / p.mass
            hist = history_increment(cfg.settling_inertia_model, p.vel, p.vel_prev, p.mass, p.lattice_r)
            if hist is not None:
                vel_new = vel_new + 0.5 * hist
            if cfg.settling_inertia_model == "feng_b2":
                vel_new = vel_new + (1.0 / p.rho_ratio) * (p.vel - p.vel_prev)
            p.vel_prev = p.vel.copy()
            p.vel = vel_new
            p.force = fp

    def _set_markers(self, p, vel, om):
        """Particle p's markers at its position and angle (physics/markers.py:23-38)
        and their desired velocity vel + om x (X - x) / dx (:41-60; om = 0.0: vel)."""
        rot = self.cfg.enable_rotation
        p.Lx, p.Ly = rigid_markers(p.Lx_c, p.Ly_c, p.cx_init, p.cy_init, p.pos, angle=p.angle if rot else 0.0)
        dv = np.empty((p.Lb, 2))
        dv[:, 0] = float(vel[0])
        dv[:, 1] = float(vel[1])
        if om != 0.0:
            dv[:, 0] += -om * (p.Ly - float(p.pos[1])) / self.st.dx
            dv[:, 1] += om * (p.Lx - float(p.pos[0])) / self.st.dx
        p.desired_velocity = dv

    def _sedimentation_step_prescribed(self, outputs):
        """A single disc moved at cfg.prescribed_velocity
        (runtime/scenarios/sedimentation_single.py:91-97,174-180): position and
        markers advance, the desired velocity is the prescribed one, and after
        the IB step the disc keeps that velocity and records the force."""
        cfg, st = self.cfg, self.st
        p = st.particles[0]
        pv = np.array(cfg.prescribed_velocity, dtype=float)
        p.pos = p.pos + st.dt * pv * st.dx
        p.Lx, p.Ly = rigid_markers(p.Lx_c, p.Ly_c, p.cx_init, p.cy_init, p.pos)
        dv = np.empty((p.Lb, 2))
        dv[:, 0] = float(pv[0])
        dv[:, 1] = float(pv[1])
        p.desired_velocity = dv
        p.vel_half = pv
        self._upload_markers()
        self._launch(outputs)
        self.ttt += 1
        if outputs:
            self.last_out_step = self.ttt - 1
        forces, _ = self.particle_forces()
        p.vel = pv.copy()
        p.fib_force = forces[0]
        p.force = forces[0]

    def _l_int_z(self, p):
        """Angular momentum of the fluid inside particle p's disc from this step's
        velocity and density (diagnostics/internal_flow.py:220-262): the box of
        the disc copied to the host, summed like the reference."""
        st = self.st
        ci, cj, r_lat = float(p.pos[0]) / st.dx, float(p.pos[1]) / st.dx, p.r_domain / st.dx
        ii, jj, rr = int(round(ci)), int(round(cj)), int(r_lat) + 2
        i0, i1 = max(0, ii - rr), min(st.nx, ii + rr + 1)
        j0, j1 = max(0, jj - rr), min(st.ny, jj + rr + 1)
        U = self.U_out.reshape(st.ny, st.nx, 2)[j0:j1, i0:i1].double().cpu().numpy()
        ro = self.ro_out.reshape(st.ny, st.nx)[j0:j1, i0:i1].double().cpu().numpy()
        RX, RY = np.meshgrid(np.arange(i0, i1, dtype=float) - ci, np.arange(j0, j1, dtype=float) - cj)
        m = RX ** 2 + RY ** 2 <= r_lat ** 2
        sux, suy = np.ascontiguousarray(U[..., 0]), np.ascontiguousarray(U[..., 1])
        return float(np.sum(RX[m] * ro[m] * suy[m] - RY[m] * ro[m] * sux[m]))

    def _sedimentation_step_euler(self, outputs):
        """Explicit Euler (runtime/scenarios/sedimentation_multi.py:126-190): the
        IB step with the markers and desired velocity the last step left, then
        velocity and position from this step's force (physics/inertia/
        {none,explicit_history}.py euler_explicit, physics/rigid_body.py:84-98,
        feng_b2 post-correction); with rotation the angular step of
        rigid_body.py:101-121, whose angular momentum change of the fluid inside
        each disc needs this step's velocity and density (every step writes
        them); then the next step's markers and desired velocity."""
        cfg, st = self.cfg, self.st
        rot = cfg.enable_rotation
        self._upload_markers()
        # with rotation every step writes rho and U (not f*) for the angular
        # momentum of the fluid inside each disc
        self._launch(outputs or (OUT_MOMENTS if rot else False))
        self.ttt += 1
        if outputs:
            self.last_out_step = self.ttt - 1
        forces, torques = self.particle_forces(torques=rot)
        for k, (p, fp) in enumerate(zip(st.particles, forces)):
            if rot:
                l_now = self._l_int_z(p)
                dl = l_now - p.l_int_prev
                p.l_int_prev = l_now
                omega_new = p.omega + (dl + st.dt * torques[k]) / p.I_particle
                if cfg.sedimentation_euler_update_scheme == "trapezoidal":
                    p.angle += 0.5 * st.dt * (p.omega + omega_new)
                else:
                    p.angle += st.dt * omega_new
                p.torque = torques[k]
                p.omega = omega_new
            p.fib_force = fp
            F = fp + net_gravity(p.rho_ratio, p.lattice_r, st.gravity_lattice, cfg.gravity_direction)
            vel_new = p.vel + st.dt * F / p.mass
            hist = history_increment(cfg.settling_inertia_model, p.vel, p.vel_prev, p.mass, p.lattice_r)
            if hist is not None:
                vel_new = vel_new + hist
            if cfg.sedimentation_euler_update_scheme == "trapezoidal":
                pos_new = p.pos + 0.5 * st.dt * (p.vel + vel_new) * st.dx
            else:
                pos_new = p.pos + st.dt * vel_new * st.dx
            if cfg.settling_inertia_model == "feng_b2":
                vel_new = vel_new + (1.0 / p.rho_ratio) * (p.vel - p.vel_prev)
            p.vel_prev = p.vel.copy()
            p.vel = vel_new
            p.pos = pos_new
            p.force = fp
            self._set_markers(p, vel_new, p.omega if rot else 0.0)

    def particle_forces(self, torques=False):
        """-sum of each particle's spread force over the lattice, summed like the
        reference (numpy over the dense N x 2 field: iblbm/ibm/multi_particle.py:199-202);
        with torques also T = -sum((i - cx) fy - (j - cy) fx) over the lattice, node
        indices as floats and the particle centre in lattice units (:203-208).
        Under DF the reference sums the particle's marker forces instead
        (iblbm/ibm/forcing.py:262-275): F = -sum(Lf ds), T = -sum((rx Lfy - ry Lfx) ds),
        rx = (Lx - cx) / dx over the markers this step used; under DFC the sums of
        its markers' Lagrangian forces F and of rx Fy - ry Fx.
        Returns (forces, torques or None)."""
        st = self.st
        if self.method == "DFC":
            # iblbm/ibm/strategies/dfc.py:114-128: sums of the markers' Lagrangian forces
            fl = self.d_dfc_force[: 2 * self.Lb].reshape(self.Lb, 2).cpu().numpy()
            moff = self.d_moff.cpu().numpy()
            out, tq = [], ([] if torques else None)
            for p, part in enumerate(st.particles):
                f = fl[moff[p]:moff[p + 1]]
                out.append(np.array([float(f[:, 0].sum()), float(f[:, 1].sum())]))
                if torques:
                    rx = (np.asarray(part.Lx) - float(part.pos[0])) / st.dx
                    ry = (np.asarray(part.Ly) - float(part.pos[1])) / st.dy
                    tq.append(float(np.sum(rx * f[:, 1] - ry * f[:, 0])))
            return out, tq
        if self.method == "DF" and not self.single:  # (the single runtime sums the field, below)
            Lfx, Lfy = self.d_Lfx.cpu().numpy(), self.d_Lfy.cpu().numpy()
            moff = self.d_moff.cpu().numpy()
            out, tq = [], ([] if torques else None)
            for p, part in enumerate(st.particles):
                fx, fy = Lfx[moff[p]:moff[p + 1]], Lfy[moff[p]:moff[p + 1]]
                La = float(part.Larea)
                out.append(np.array([-float(np.sum(fx * La)), -float(np.sum(fy * La))]))
                if torques:
                    rx = (part.Lx - float(part.pos[0])) / st.dx
                    ry = (part.Ly - float(part.pos[1])) / st.dy
                    tq.append(-float(np.sum((rx * fy - ry * fx) * La)))
            return out, tq
        nb = int(self.d_count.item())
        nodes = self.d_nodes[:nb].cpu().numpy()
        part = self.d_fib_part[: 2 * self.B * self.P].reshape(self.P, self.B, 2)[:, :nb].cpu().numpy()
        part = part.astype(np.float64)
        out, tq = [], ([] if torques else None)
        if torques:
            if self._torque_ij is None:  # node indices as floats, kept between steps
                self._torque_ij = np.meshgrid(np.arange(st.nx, dtype=float), np.arange(st.ny, dtype=float),
                                              indexing="xy")
            II, JJ = self._torque_ij
        for p in range(self.P):
            dense = np.zeros((self.N, 2))
            dense[nodes] = part[p]
            out.append(np.array([-float(dense[:, 0].sum()), -float(dense[:, 1].sum())]))
            if torques:
                pos = st.particles[p].pos
                fx = np.ascontiguousarray(dense[:, 0]).reshape(st.ny, st.nx)
                fy = np.ascontiguousarray(dense[:, 1]).reshape(st.ny, st.nx)
                tq.append(-float(np.sum((II - float(pos[0]) / st.dx) * fy - (JJ - float(pos[1]) / st.dy) * fx)))
        return out, tq

    # ---- read-back ----------------------------------------------------------------
    def band_fib_dense(self):
        torch = self.torch
        nb = int(self.d_count.item())
        fib = torch.zeros(self.N, 2, dtype=torch.float64, device=self.dev)
        if self.method in ("DF", "MDF") and nb > 0:
            fib[self.d_nodes[:nb].long()] = self.d_fib[: 2 * nb].reshape(nb, 2).double()
        return fib

    def queue_force_coeffs(self):
        """Queue, on the current stream, the reduction of the last output step's
        Cd / Cl (iblbm/diagnostics/core.py:53-113) into the device ring buffer;
        no host synchronisation.  Returns the entry's sequence number (read it
        with read_force_coeffs)."""
        from ._lib import ForceCoeffArgs
        cfg, st = self.cfg, self.st
        a = ForceCoeffArgs()
        a.ro, a.n_nodes, a.f32 = ptr(self.ro_out), self.N, int(self.f32)
        a.method = 0 if self.no_ibm else IBM_IDS[self.method]
        a.band_fib, a.band_count = ptr(self.d_fib), ptr(self.d_count)
        a.dfc_force, a.lb_total = ptr(self.d_dfc_force), self.Lb
        a.u_ref = float(cfg.lattice_u if cfg.motion_type == "oscillating" else st.in_u)
        a.lattice_r = float(st.lattice_r)
        a.partials, a.ticket = ptr(self.d_diag_part), ptr(self.d_diag_ticket)
        a.ring, a.ring_len, a.ring_pos = ptr(self.d_ring), self.ring_len, ptr(self.d_ring_pos)
        check(self.L.iblbm_force_coeffs(ctypes.byref(a), self.stream()), "iblbm_force_coeffs")
        self.ring_read += 1
        return self.ring_read - 1

    def read_force_coeffs(self, first, count):
        """Entries first .. first + count - 1 of the ring (at most ring_len
        back) as a (count, 5) host array: Cd, Cl, mean rho, sum Fx, sum Fy.
        Waits for the work queued on the current stream."""
        if count <= 0:
            return np.zeros((0, 5))
        if count > self.ring_len or self.ring_read - first > self.ring_len:
            raise ValueError("ring entries overwritten: read the ring at least every ring_len checks")
        s0 = first % self.ring_len
        n0 = min(count, self.ring_len - s0)
        rows = self.d_ring[s0:s0 + n0].cpu().numpy()
        if n0 < count:  # wrapped past the end of the ring
            rows = np.concatenate([rows, self.d_ring[: count - n0].cpu().numpy()])
        return rows

    def cd_cl(self):
        """Cd, Cl of the last output step — iblbm/diagnostics/core.py:53-113,
        reduced on the device (iblbm_force_coeffs); 0, 0 without an immersed
        body (iblbm/runtime/scenarios/taylor_green.py:60-62)."""
        if self.no_ibm:
            return 0.0, 0.0
        k = self.queue_force_coeffs()
        r = self.read_force_coeffs(k, 1)[0]
        return float(r[0]), float(r[1])

    def velocity_change(self):
        """Queue the velocity-convergence error of the last output step against
        the previous check's field (iblbm/diagnostics/core.py:116-135) and make
        this step's field the next reference; returns the device array
        [sum (U - U_prev)^2, sum U_prev^2, error].  The first call compares
        against zeros (error 1.0), as the reference's first check only stores
        the field."""
        from ._lib import VelocityChangeArgs
        torch = self.torch
        if self.d_uprev is None:
            self.d_uprev = torch.zeros(2 * self.N, dtype=torch.float64, device=self.dev)
        a = VelocityChangeArgs()
        a.U, a.U_prev, a.n_nodes, a.f32 = ptr(self.U_out), ptr(self.d_uprev), self.N, int(self.f32)
        a.partials, a.ticket, a.out = ptr(self.d_diag_part), ptr(self.d_diag_ticket), ptr(self.d_vchange)
        check(self.L.iblbm_velocity_change(ctypes.byref(a), self.stream()), "iblbm_velocity_change")
        return self.d_vchange

    def mdf_stats(self):
        s = self.d_stats.cpu().numpy()
        d = self.d_dstats.cpu().numpy()
        return {"iter_count": int(s[0]), "diverged": bool(s[1]), "converged": bool(s[2]),
                "guard_trips": max(int(s[3]), 0), "marker_space": int(s[3]) == -1,
                "restructured_node_space": int(s[3]) == -2, "cluster": int(s[3]) == -3,
                "last_residual": float(d[0]), "omega_used": float(d[1])}

    def status(self):
        """Band-kernel status word (0 = ok); a pipeline timeout of the FP32 pass
        reads as 100 + its code."""
        self.join()
        st = int(self.d_stats[4].item())
        if st == 0 and self.f32:
            p = int(self.d_pipe_status.item())
            if p:
                return 100 + p
        return st

    def read_state(self):
        """Copy the last output step's fields into host arrays on self.st (AoS, the
        reference's layout) and return it."""
        torch, st = self.torch, self.st
        self.join()
        s = self.stream()
        fs = torch.empty(self.N * 9, dtype=torch.float64, device=self.dev)
        self._to_aos(self.fstar_out, fs)
        feq = torch.empty_like(fs)
        ro, U = self.ro_out.double().contiguous(), self.U_out.double().contiguous()
        check(self.L.iblbm_feq(ptr(ro), ptr(U), self.N, self.case.incompressible, ptr(feq), s), "iblbm_feq")
        st.fstar = fs.reshape(self.N, 9).cpu().numpy()
        st.feq = feq.reshape(self.N, 9).cpu().numpy()
        st.ro = ro.cpu().numpy()
        st.U = U.reshape(self.N, 2).cpu().numpy()
        st.fib = self.band_fib_dense().cpu().numpy()
        if self.method == "DFC":
            st.dfc_force_lagr = self.d_dfc_force[: 2 * self.Lb].reshape(self.Lb, 2).cpu().numpy()
        if self.method == "MDF" and not self.no_ibm:
            st.mdf_iter_stats = self.mdf_stats()
        return st

    def fpost_aos(self):
        """Post-collision populations of the last completed step (AoS)."""
        torch = self.torch
        out = torch.empty(self.N * 9, dtype=torch.float64, device=self.dev)
        self._to_aos(self.f[self.parity], out)
        return out.reshape(self.N, 9).cpu().numpy()

    def _to_aos(self, soa, out):
        """Lattice SoA buffer -> FP64 AoS f[N, 9] (adds the weights back in the FP32 form)."""
        if self.f32:
            check(self.L.iblbm_from_shifted_f32(ptr(soa), self.geom, ptr(out), self.stream()),
                  "iblbm_from_shifted_f32")
        else:
            check(self.L.iblbm_soa_to_aos(ptr(soa), self.geom, ptr(out), self.stream()), "iblbm_soa_to_aos")
