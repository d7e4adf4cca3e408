"""Diagnostics against the reference's own functions (fixtures made by
tests/golden/make_golden_diag.py from iblbm.diagnostics)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "diag.npz")


@pytest.fixture(scope="module")
def diag():
    return dict(np.load(GOLD))


@pytest.mark.parametrize("name", ["signed", "rect_low", "rect_high"])
def test_strouhal_matches_reference(diag, name):
    from iblbm_b200.diagnostics import compute_strouhal
    ci, D, u = int(diag["st_ci"][0]), float(diag["st_D"][0]), float(diag["st_u"][0])
    cl = diag[f"st_{name}_cl"]
    steps = np.arange(1, len(cl) + 1) * ci
    uref = u * (8 if name == "rect_high" else 1)
    assert compute_strouhal(cl, steps, D, uref, ci) == float(diag[f"st_{name}"][0])


def test_diagnostic_markers_count():
    from iblbm_b200.diagnostics import diagnostic_markers
    Lx, Ly, th = diagnostic_markers(0.5, 0.5, 0.125, 81)
    assert len(Lx) == 126 and th[0] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("delta", ["hat", "peskin4pt"])
def test_slip_error_matches_reference(diag, delta):
    from iblbm_b200.diagnostics import compute_slip_error
    NN = 81
    dx = 1.0 / (NN - 1)
    r = compute_slip_error(diag["slip_Eux"], diag["slip_Euy"], dx, dx, 0.5, 0.5, 0.25, NN, delta, u_ref=0.05)
    np.testing.assert_allclose(r["per_marker"], diag[f"slip_{delta}_per_marker"], rtol=1e-13, atol=0)
    assert abs(r["mean"] - float(diag[f"slip_{delta}_mean"][0])) <= 1e-13 * abs(r["mean"])
    assert abs(r["max"] - float(diag[f"slip_{delta}_max"][0])) <= 1e-13 * abs(r["max"])


@pytest.mark.gpu
@pytest.mark.parametrize("delta", ["hat", "peskin4pt"])
def test_leakage_flux_matches_reference(diag, delta):
    """Normal flux through the diagnostic ring against the reference's
    compute_leakage_flux on the same field: per-marker normal velocities to
    1e-13 of the largest, the signed total (a sum with cancellation) to 1e-12."""
    from iblbm_b200.diagnostics import compute_leakage_flux
    NN = 81
    dx = 1.0 / (NN - 1)
    q = compute_leakage_flux(diag["slip_Eux"], diag["slip_Euy"], dx, dx, 0.5, 0.5, 0.25, NN, delta, u_ref=0.05)
    want = diag[f"leak_{delta}_per_marker"]
    scale = float(np.max(np.abs(want)))
    np.testing.assert_allclose(q["per_marker"], want, rtol=0, atol=1e-13 * scale)
    total, raw = diag[f"leak_{delta}_total"]
    assert abs(q["total"] - total) <= 1e-12 * scale
    assert abs(q["total_raw"] - raw) <= 1e-12 * scale * 0.05 * np.pi * 0.25


@pytest.mark.gpu
def test_run_reports_marker_slip():
    """run() adds the marker slip of the last output step (mean, max, RMS over
    U_ref), interpolated in the reference's order: equal to the oracle's
    interpolation of the same velocity field."""
    from iblbm_b200 import SimConfig, run
    from oracle import harness as H
    cfg = SimConfig(Re=20, NN=41, xmax=2.5, ymax=1, cylinder_center=(0.625, 0.5), cylinder_D_ratio=0.25,
                    lattice_u=0.05, inflow_u=0.05, bc_type="dirichlet_neumann", delta_type="hat", ibm_method="DF",
                    collision_model="BGK", marker_spacing_factor=1.0, max_steps=60, use_convergence=False,
                    check_interval=20)
    res = run(cfg, verbose=False)
    st = res["state"]
    Lux, Luy = H.ibm_df(st.Lx, st.Ly, np.zeros((st.Lb, 2)), np.ascontiguousarray(st.U[:, 0]),
                        np.ascontiguousarray(st.U[:, 1]), np.ones(st.nx * st.ny), st.dx, st.dy, 1.0, st.Larea,
                        st.ny, st.nx, "hat")[1:3]
    mag = np.sqrt(Lux ** 2 + Luy ** 2)
    assert res["slip"]["max"] == float(np.max(mag) / st.in_u)
    assert res["slip"]["mean"] == float(np.mean(mag) / st.in_u)
    assert res["slip"]["rms"] == float(np.sqrt(np.mean(mag ** 2)) / st.in_u)


@pytest.mark.parametrize("kind", ["signed", "rect_low", "rect_high"])
def test_tail_statistics_match_reference(diag, kind):
    """Tail index, tail mean (30 % and 50 %), half peak-to-peak and Cl amplitude
    of the reference's functions on the same series, bit for bit."""
    from iblbm_b200 import diagnostics as D
    cl = diag[f"st_{kind}_cl"]
    got = [D.tail_start_index(len(cl)), D.tail_mean(cl), D.tail_peak_to_peak_amp(cl), D.tail_mean(cl, 0.5),
           D.compute_cl_amplitude(cl)]
    np.testing.assert_array_equal(np.array(got), diag[f"tail_{kind}"])
    with pytest.raises(ValueError):
        D.tail_values([])


def test_convergence_and_recirculation_match_reference(diag):
    from iblbm_b200 import diagnostics as D
    NN = 81
    dx = 1.0 / (NN - 1)
    Eux, Euy = diag["slip_Eux"], diag["slip_Euy"]
    assert D.check_convergence(Eux, Euy, diag["conv_old"], Euy * 0.5) == diag["conv"][0]
    assert D.check_convergence(Eux, Euy, 0 * Eux, 0 * Euy) == 1.0
    w = diag["recirc_field"]
    got = [D.compute_recirculation_length(w, dx, dx, 0.5, 0.5, 0.25),
           D.compute_recirculation_length(np.abs(w), dx, dx, 0.5, 0.5, 0.25)]
    np.testing.assert_array_equal(np.array(got), diag["recirc"])


def test_internal_flow_matches_reference(diag):
    """Residual flow inside the body, and the momentum and angular momentum of
    the fluid inside a disc (two forms, one clipped at the lattice corner),
    against the reference's functions on the same fields, bit for bit."""
    from iblbm_b200 import diagnostics as D
    NN = 81
    dx = 1.0 / (NN - 1)
    Eux, Euy, ro = diag["slip_Eux"], diag["slip_Euy"], diag["inside_ro"]
    r = D.compute_inside_residual(Eux, Euy, dx, dx, 0.5, 0.5, 0.25, kappa=2.0, u_ref=0.05)
    got = [r["mean"], r["max"], r["n_points"], r["mean_normalized"], r["max_normalized"]]
    np.testing.assert_array_equal(np.array(got), diag["inside_residual"])
    assert D.compute_inside_residual(Eux, Euy, dx, dx, 0.5, 0.5, 0.01)["n_points"] == 0
    np.testing.assert_array_equal(np.array(D.compute_internal_momentum(Eux, Euy, ro, dx, dx, 0.5, 0.5, 0.125)),
                                  diag["internal_momentum"])
    assert D.compute_internal_angular_momentum(Eux, Euy, ro, dx, dx, 0.5, 0.5, 0.125) == \
        diag["internal_angular_momentum"][0]
    ny, nx = Eux.shape
    U = np.stack([Eux.ravel(), Euy.ravel()], axis=1)
    got = [D.compute_l_int_z(U, ro.ravel(), nx, ny, dx, 0.5, 0.5, 0.125),
           D.compute_l_int_z(U, ro.ravel(), nx, ny, dx, 0.02, 0.97, 0.125)]
    np.testing.assert_array_equal(np.array(got), diag["l_int_z"])


def test_surface_stress_force_matches_reference(diag):
    """Stress of a seeded D2Q9 state and the force it puts on a cylinder (one
    circle inside the lattice, one clamped at its edge), against the reference's
    surface functions, bit for bit."""
    import hashlib
    from iblbm_b200 import diagnostics as D
    NN = 81
    dx = 1.0 / (NN - 1)
    ro = diag["inside_ro"]
    ny, nx = ro.shape
    rng = np.random.default_rng(12)
    fst = (1.0 / 9.0) + 0.01 * rng.standard_normal((nx * ny, 9))
    feq = (1.0 / 9.0) + 0.01 * rng.standard_normal((nx * ny, 9))
    sig = D.compute_stress_tensor(fst, feq, ro.ravel(), 0.8, None, ny, nx)
    np.testing.assert_array_equal(sig.reshape(-1, 4)[::97], diag["stress_sample"])
    assert hashlib.sha256(np.ascontiguousarray(sig).tobytes()).digest() == bytes(diag["stress_sha"])
    got = np.stack([D.integrate_surface_force(sig, 0.5, 0.5, 0.125, dx, dx, nx, ny),
                    D.integrate_surface_force(sig, 0.05, 0.5, 0.125, dx, dx, nx, ny, 100)])
    np.testing.assert_array_equal(got, diag["surface_force"])
