"""GPU parity: the CUDA path against the reference's golden vectors and the CPU
oracle.  The FP64 plain form reproduces the reference's arithmetic operation for
operation, so populations, moments and forces are compared bit for bit
(`assert_array_equal`); Cd/Cl, which the engine reduces on the device in a
different summation order, are held to 1e-12 relative (the target is 1e-9)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def units():
    return dict(np.load(os.path.join(GOLD, "units.npz")))


def test_reference_shaped_kernels(torch, units):
    from iblbm_b200 import gpu_kernels as gk
    u = units
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    h = lambda t: t.cpu().numpy()
    np.testing.assert_array_equal(h(gk.feq_gpu(d(u["u_ro"]), d(u["u_U"]))), u["u_feq"])
    np.testing.assert_array_equal(h(gk.feq_gpu(d(u["u_ro"]), d(u["u_U"]), True)), u["u_feq_inc"])
    ro, U = gk.macroscopic_gpu(d(u["u_fstar"]))
    np.testing.assert_array_equal(h(ro), u["u_macro_ro"])
    np.testing.assert_array_equal(h(U), u["u_macro_U"])
    tau, taum = float(u["u_tau"][0]), float(u["u_tau_minus"][0])
    args = [d(u[k]) for k in ("u_fstar", "u_feq", "u_U", "u_fib")]
    np.testing.assert_array_equal(h(gk.collision_gpu(*args, tau, 1.0)), u["u_bgk"])
    np.testing.assert_array_equal(h(gk.collision_trt_gpu(*args, tau, taum, 1.0)), u["u_trt"])
    np.testing.assert_array_equal(h(gk.collision_cm_mrt_gpu(*args, u["u_S"], 1.0)), u["u_cmmrt"])
    nx, ny = int(u["g_nx"][0]), int(u["g_ny"][0])
    np.testing.assert_array_equal(h(gk.streaming_gpu(d(u["g_fold"]), d(u["g_fpost"]), nx, ny)), u["g_stream"])
    from oracle import harness as H
    U2 = d(u["u_U"]).clone()
    gk.velocity_correction_gpu(U2, d(u["u_fib"]), d(u["u_ro"]), 1.0)
    Uo = u["u_U"].copy()
    H.velocity_correction(Uo, u["u_fib"], u["u_ro"], 1.0)
    np.testing.assert_array_equal(h(U2), Uo)


@pytest.mark.parametrize("delta", ["hat", "peskin4pt"])
def test_reference_shaped_ibm_wrappers(torch, units, delta):
    """ibm_direct_forcing_gpu / compute_lambda_gpu / dfc_correction_gpu against
    the reference's own outputs on its inputs (bit for bit)."""
    from iblbm_b200 import gpu_kernels as gk
    u = units
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    nx, ny, dx = int(u["i_nx"][0]), int(u["i_ny"][0]), float(u["i_dx"][0])
    Lx, Ly, dv, La = d(u["i_Lx"]), d(u["i_Ly"]), d(u["i_dv"]), float(u["i_Larea"][0])
    Eux, Euy, Ro = (d(u[k].ravel()) for k in ("i_Eux", "i_Euy", "i_Ro"))
    for inc in (0, 1):
        fib, Lux, Luy = gk.ibm_direct_forcing_gpu(Lx, Ly, dv, Eux, Euy, Ro, dx, dx, 1.0, La, ny, nx, delta, True,
                                                  bool(inc))
        k = f"df_{delta}_{inc}"
        np.testing.assert_array_equal(fib.cpu().numpy(), u[k + "_fib"])
        np.testing.assert_array_equal(Lux.cpu().numpy(), u[k + "_Lux"])
        np.testing.assert_array_equal(Luy.cpu().numpy(), u[k + "_Luy"])
    Efx, Efy, _, _ = gk.ibm_direct_forcing_fields_gpu(Lx, Ly, dv, Eux, Euy, Ro, dx, dx, 1.0, La, ny, nx, delta)
    np.testing.assert_array_equal(Efx.cpu().numpy().ravel(), u[f"df_{delta}_0_fib"][:, 0])
    lam = gk.compute_lambda_gpu(Lx, Ly, 1.0, La, dx, dx, ny, nx, delta)
    np.testing.assert_array_equal(lam.cpu().numpy(), u[f"lam_{delta}"])
    lr = np.load(os.path.join(GOLD, "lambda_rho.npz"))
    for rho_f in (1.3, 0.7):  # lambda(k) = 1 / (2 rho_f ds W_sum), the reference's own outputs
        lam_r = gk.compute_lambda_gpu(Lx, Ly, rho_f, La, dx, dx, ny, nx, delta)
        np.testing.assert_array_equal(lam_r.cpu().numpy(), lr[f"lam_{delta}_{rho_f}"])
    fstar = d(u[f"dfc_{delta}_fstar"])
    corr, force = gk.dfc_correction_gpu(Lx, Ly, dv, fstar, lam, dx, dx, La, ny, nx, delta)
    np.testing.assert_array_equal((fstar + corr).cpu().numpy(), u[f"dfc_{delta}_fc"])
    np.testing.assert_allclose(force.cpu().numpy(), u[f"dfc_{delta}_force"], rtol=1e-13, atol=1e-18)


@pytest.mark.parametrize("delta", ["hat", "peskin4pt"])
def test_raw_df_kernel_handles(torch, units, delta):
    """_ibm_interp_force_kern and _ibm_spread_kern (the raw kernels the
    reference's per-particle DF closure launches, iblbm/ibm/forcing.py:185-231)
    with the reference's call convention: interpolated velocities equal to the
    reference's own, and the spread of the computed marker forces equal to the
    reference's DF field, bit for bit."""
    from iblbm_b200 import gpu_kernels as gk
    u = units
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    nx, ny, dx = int(u["i_nx"][0]), int(u["i_ny"][0]), float(u["i_dx"][0])
    Lx, Ly, dv, La = d(u["i_Lx"]), d(u["i_Ly"]), d(u["i_dv"]), float(u["i_Larea"][0])
    Eux, Euy, Ro = (d(u[k]).reshape(ny, nx) for k in ("i_Eux", "i_Euy", "i_Ro"))
    Lb = int(Lx.numel())
    for inc in (0, 1):
        Lfx, Lfy, Lux, Luy = (torch.empty(Lb, dtype=torch.float64, device="cuda") for _ in range(4))
        gk._ibm_interp_force_kern(gk._grid(Lb), (gk._BLOCK,),
                                  (Lx, Ly, dv, Eux, Euy, Ro, dx, dx, 1.0, nx, ny, Lb, gk._DELTA_TYPE_IDS[delta],
                                   gk._DELTA_STENCIL_A[delta], inc, Lfx, Lfy, Lux, Luy))
        k = f"df_{delta}_{inc}"
        np.testing.assert_array_equal(Lux.cpu().numpy(), u[k + "_Lux"])
        np.testing.assert_array_equal(Luy.cpu().numpy(), u[k + "_Luy"])
        Efx = torch.zeros(ny, nx, dtype=torch.float64, device="cuda")
        Efy = torch.zeros_like(Efx)
        gk._ibm_spread_kern(gk._grid(Lb), (gk._BLOCK,),
                            (Lfx, Lfy, Lx, Ly, dx, dx, La, nx, ny, Lb, gk._DELTA_TYPE_IDS[delta],
                             gk._DELTA_STENCIL_A[delta], Efx, Efy))
        np.testing.assert_array_equal(Efx.cpu().numpy().ravel(), u[k + "_fib"][:, 0])
        np.testing.assert_array_equal(Efy.cpu().numpy().ravel(), u[k + "_fib"][:, 1])


def _cfg(kw):
    from iblbm_b200.config import SimConfig
    kw = dict(kw)
    kw["cylinder_center"] = tuple(kw["cylinder_center"])
    if kw.get("particles_config"):
        kw["particles_config"] = [dict(p, center=tuple(p["center"])) for p in kw["particles_config"]]
    return SimConfig(**kw)


def _compare_runs(cfg, res, ref):
    assert res["engine"].status() == 0, f"device status {res['engine'].status()}"
    s, r = res["state"], ref["state"]
    for k in ("ro", "U", "fstar", "fib", "feq"):
        np.testing.assert_array_equal(getattr(s, k), getattr(r, k), err_msg=k)
    np.testing.assert_allclose(res["Cd_history"], ref["Cd_history"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(res["Cl_history"], ref["Cl_history"], rtol=1e-12, atol=1e-13)
    if r.particles is not None:
        for p, q in zip(s.particles, r.particles):
            np.testing.assert_array_equal(p.pos, q.pos)
            np.testing.assert_array_equal(p.vel, q.vel)
            np.testing.assert_array_equal(p.force, q.force)
            if cfg.enable_rotation:
                assert (p.omega, p.angle, p.torque) == (q.omega, q.angle, q.torque)
    if cfg.ibm_method == "DFC":
        np.testing.assert_allclose(s.dfc_force_lagr, r.dfc_force_lagr, rtol=1e-13, atol=1e-16)


from tests.golden.make_golden import RUN_CASES  # noqa: E402


@pytest.mark.parametrize("name", sorted(RUN_CASES))
def test_engine_matches_oracle_bitwise(torch, name):
    """Every golden configuration, run by the engine and by the oracle."""
    from iblbm_b200 import run
    from oracle import harness as H
    cfg = _cfg(RUN_CASES[name])
    ref = H.run(cfg)
    res = run(cfg, verbose=False)
    _compare_runs(cfg, res, ref)


def test_engine_matches_reference_golden(torch):
    """The engine against the reference's own end-to-end fixture (SHA-256)."""
    import hashlib
    from iblbm_b200 import run
    g = dict(np.load(os.path.join(GOLD, "run_c1_df_bgk_hat.npz")))
    kw = json.loads(bytes(g["config_json"]).decode())
    res = run(_cfg(kw), verbose=False)
    for k in ("ro", "U", "fib", "fstar"):
        a = np.ascontiguousarray(getattr(res["state"], k), dtype=np.float64)
        assert hashlib.sha256(a.tobytes()).hexdigest() == bytes(g[f"sha_{k}"]).hex(), k
    np.testing.assert_allclose(res["Cd_history"], g["Cd_history"], rtol=1e-12)


@pytest.mark.parametrize("collision", ["BGK", "TRT", "CM_MRT"])
@pytest.mark.parametrize("method,delta", [("DF", "hat"), ("MDF", "peskin4pt"), ("DFC", "peskin4pt")])
def test_method_matrix(torch, collision, method, delta):
    """3 collisions x 3 IB methods on a small Dirichlet-Neumann channel, 120 steps."""
    from iblbm_b200 import run
    from oracle import harness as H
    kw = dict(Re=40, NN=49, xmax=2, ymax=1, cylinder_center=(0.45, 0.5), cylinder_D_ratio=0.25, lattice_u=0.05,
              inflow_u=0.05, bc_type="dirichlet_neumann", delta_type=delta, ibm_method=method,
              collision_model=collision, trt_magic_param=0.1875, mdf_iterations=20, mdf_min_iterations=5,
              mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=120, use_convergence=False,
              check_interval=40)
    cfg = _cfg(kw)
    _compare_runs(cfg, run(cfg, verbose=False), H.run(cfg))


def test_taylor_green_tracks_the_analytic_vortex(torch):
    """The Taylor-Green run (no IBM step) stays within 2 % (L2) of the analytic
    decaying vortex after 300 steps (the oracle's error on this lattice: 1.0 %)."""
    from iblbm_b200 import run
    from iblbm_b200.physics import tg_base, tg_params
    cfg = _cfg(RUN_CASES["tg_lbm_bgk"])
    s = run(cfg, verbose=False)["state"]
    L, nu = tg_params(cfg)
    XX, YY = np.meshgrid(np.arange(s.nx) - (s.nx - 1) / 2.0, np.arange(s.ny) - (s.ny - 1) / 2.0)
    ux, uy = tg_base(XX.ravel(), YY.ravel(), cfg.tg_u0, L)
    d = np.exp(-2.0 * nu * (np.pi / L) ** 2 * cfg.max_steps)
    ana = np.stack([ux * d, uy * d], axis=1)
    assert np.sqrt(np.sum((s.U - ana) ** 2)) / np.sqrt(np.sum(ana ** 2)) < 0.02


def test_config1_full_geometry_1000_steps(torch):
    """Config 1 geometry (401 x 161, D = 20, DF + BGK + hat) for 1000 steps."""
    from iblbm_b200 import run
    from oracle import harness as H
    kw = dict(RUN_CASES["c1_df_bgk_hat"], max_steps=1000, check_interval=100)
    cfg = _cfg(kw)
    _compare_runs(cfg, run(cfg, verbose=False), H.run(cfg))


@pytest.mark.parametrize("name", ["C2", "C3", "C5"])
def test_benchmark_geometries_200_steps(torch, name):
    """Configurations 2 (1601 x 641, MDF + Peskin-4, TRT), 3 (1281 x 1281,
    oscillating DFC, open boundary) and 5 (321 x 1281, two settling discs,
    coupled MDF, CM-MRT) at full size for 200 steps: every field bit for bit
    against the oracle."""
    from iblbm_b200 import run
    from oracle import harness as H
    from tests.golden.make_golden import INIT_CASES
    kw = dict(INIT_CASES[name], max_steps=200, check_interval=50, use_convergence=False)
    if name == "C2":
        kw.update(mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6)
    cfg = _cfg(kw)
    _compare_runs(cfg, run(cfg, verbose=False), H.run(cfg))


def test_config1_full_geometry_10000_steps(torch):
    """Config 1 (401 x 161, D = 20, DF + BGK + hat) for its full 10 000 steps:
    every field bit for bit against the oracle, Cd/Cl to 1e-12."""
    from iblbm_b200 import run
    from oracle import harness as H
    kw = dict(RUN_CASES["c1_df_bgk_hat"], max_steps=10000, check_interval=500)
    cfg = _cfg(kw)
    _compare_runs(cfg, run(cfg, verbose=False), H.run(cfg))


@pytest.mark.parametrize("name", ["c2_mdf_trt_p4", "tg_ibm_mdf_trt_p4"])
def test_graph_and_eager_paths_agree(torch, name):
    """Replaying captured CUDA graphs gives the same bits as eager launches
    (for Taylor-Green the graphs carry the per-step decay factor update)."""
    from iblbm_b200.engine import Engine
    kw = dict(RUN_CASES[name], max_steps=60)
    e1, e2 = Engine(_cfg(kw)), Engine(_cfg(kw))
    e1.advance(60, outputs_last=True, use_graph=True)
    e2.advance(60, outputs_last=True, use_graph=False)
    torch.cuda.synchronize()
    s1, s2 = e1.read_state(), e2.read_state()
    for k in ("fstar", "U", "ro", "fib"):
        np.testing.assert_array_equal(getattr(s1, k), getattr(s2, k), err_msg=k)


@pytest.mark.parametrize("name", ["c3_dfc_bgk_p4_osc", "c2_mdf_cmmrt_p4", "vin_df_bgk_p4"])
def test_overlapped_schedule_matches_serial(torch, name):
    """Band kernel + box pass on a side stream concurrent with the bulk pass gives
    the same bits as the serial schedule (moving and fixed bodies)."""
    from iblbm_b200.engine import Engine
    kw = dict(RUN_CASES[name], max_steps=90)
    e1, e2 = Engine(_cfg(kw)), Engine(_cfg(kw))
    e2.overlap = False
    e1.advance(90, outputs_last=True, use_graph=True)
    e2.advance(90, outputs_last=True, use_graph=False)
    torch.cuda.synchronize()
    assert e1.status() == 0 and e2.status() == 0
    s1, s2 = e1.read_state(), e2.read_state()
    for k in ("fstar", "U", "ro", "fib"):
        np.testing.assert_array_equal(getattr(s1, k), getattr(s2, k), err_msg=k)
    np.testing.assert_array_equal(e1.fpost_aos(), e2.fpost_aos())


def test_step_io_matches_plain_steps(torch):
    """A fixed-body step driven with host I/O (markers in from pinned memory,
    the band force out, one graph per parity) gives the same bits as plain steps."""
    from iblbm_b200.engine import Engine
    kw = dict(RUN_CASES["c2_mdf_trt_p4"], max_steps=60)
    e1, e2 = Engine(_cfg(kw)), Engine(_cfg(kw))
    e1.advance(3, outputs_last=False)
    e2.advance(3, outputs_last=False)
    Lb = e1.Lb
    host_in = torch.empty(4 * Lb, dtype=torch.float64).pin_memory()
    host_in[:Lb] = torch.as_tensor(e1.st.Lx)
    host_in[Lb:2 * Lb] = torch.as_tensor(e1.st.Ly)
    host_in[2 * Lb:] = torch.as_tensor(e1.st.desired_velocity.reshape(-1))
    host_out = torch.empty(2, dtype=torch.float64).pin_memory()
    for _ in range(6):
        e1.step_io(host_in, host_out)
    e2.advance(6, outputs_last=False, use_graph=False)
    torch.cuda.synchronize()
    nb = int(e2.d_count.item())
    np.testing.assert_array_equal(host_out.numpy(), e2.d_fib[: 2 * nb].view(nb, 2).double().sum(0).cpu().numpy())
    np.testing.assert_array_equal(e1.fpost_aos(), e2.fpost_aos())
    assert e1.ttt == e2.ttt
    # one step ahead with two alternating buffer pairs
    ins = [host_in, torch.empty_like(host_in).pin_memory()]
    ins[1].copy_(host_in)
    outs = [host_out, torch.empty_like(host_out).pin_memory()]
    evs = [e1.step_io(ins[k % 2], outs[k % 2], wait=False) for k in range(5)]
    evs[-1].synchronize()
    e2.advance(5, outputs_last=False, use_graph=False)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(outs[0].numpy(), e2.d_fib[: 2 * nb].view(nb, 2).double().sum(0).cpu().numpy())
    np.testing.assert_array_equal(e1.fpost_aos(), e2.fpost_aos())


def test_step_io_taylor_green(torch):
    """Host-driven steps of a Taylor-Green case with markers (the decay factor's
    per-step update inside the captured step) give the same bits as plain steps."""
    from iblbm_b200.engine import Engine
    kw = dict(RUN_CASES["tg_ibm_mdf_trt_p4"], max_steps=20)
    e1, e2 = Engine(_cfg(kw)), Engine(_cfg(kw))
    e1.advance(2, outputs_last=False)
    e2.advance(2, outputs_last=False)
    Lb = e1.Lb
    host_in = torch.empty(4 * Lb, dtype=torch.float64).pin_memory()
    host_in.copy_(torch.cat([e1.d_Lx[:Lb], e1.d_Ly[:Lb], e1.d_dv[:2 * Lb]]).cpu())
    host_out = torch.empty(2, dtype=torch.float64).pin_memory()
    for _ in range(24):  # past the decay table sized for max_steps: it grows
        e1.step_io(host_in, host_out)
    e2.advance(24, outputs_last=False, use_graph=False)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(e1.fpost_aos(), e2.fpost_aos())
    assert int(e1.d_tg_step.item()) == int(e2.d_tg_step.item()) == e1.ttt


@pytest.mark.parametrize("method,spacing", [("DF", 0.5), ("MDF", 0.65), ("DFC", 0.5)])
def test_large_moving_body_keeps_lists_in_global_memory(torch, method, spacing):
    """An oscillating cylinder of 100 nodes diameter with Peskin-4 markers every
    0.5-0.65 dx (483-628 markers): its band layout exceeds the band kernel's
    shared memory, so the step keeps its contribution lists in global memory
    and rebuilds them there every step.  FP64, 20 steps, bit for bit against
    the oracle."""
    from iblbm_b200 import run
    from iblbm_b200._lib import DELTA_IDS
    from iblbm_b200.engine import Engine
    from oracle import harness as H
    cfg = _cfg(dict(Re=100, NN=401, xmax=1.5, ymax=1, cylinder_center=(0.75, 0.5), cylinder_D_ratio=0.25,
                    lattice_u=0.05, inflow_u=0.0, bc_type="open_boundary", delta_type="peskin4pt",
                    ibm_method=method, collision_model="TRT", motion_type="oscillating", KC=5.0,
                    nx_formula="simple", mdf_iterations=20, mdf_min_iterations=5, mdf_tolerance=1e-6,
                    marker_spacing_factor=spacing, max_steps=20, use_convergence=False, check_interval=10))
    eng = Engine(cfg, precision="f64")
    assert eng.L.iblbm_ibm_smem_bytes(eng.Lb, eng.B, DELTA_IDS[cfg.delta_type]) > 220 * 1024
    _compare_runs(cfg, run(cfg, verbose=False, engine=eng), H.run(cfg))
