"""The network oracle's gradient against central finite differences (CPU)."""
import numpy as np

from oracle import mlp_oracle as M


def _params(rng, npar):
    P = np.zeros(npar)
    P[0:64] = rng.standard_normal(64) * 0.1
    P[64:128] = 1.0 + 0.1 * rng.random(64)
    P[128:130] = [2.0, 0.5]
    P[M.HDR:] = rng.standard_normal(npar - M.HDR) * 0.15
    return P


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    npar = M.unpack(np.zeros(20000))[4]
    P = _params(rng, npar)
    X = rng.standard_normal((37, 64))
    T = rng.standard_normal((37, 2))
    L, g = M.loss_and_grad(P, X, T)
    assert np.all(g[:M.HDR] == 0.0)
    idx = rng.choice(np.arange(M.HDR, npar), size=60, replace=False)
    h = 1e-6
    for k in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        fd = (M.loss_and_grad(Pp, X, T)[0] - M.loss_and_grad(Pm, X, T)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-8, (k, fd, g[k])


def test_adam_first_step_is_a_sign_step():
    rng = np.random.default_rng(2)
    npar = M.unpack(np.zeros(20000))[4]
    P = _params(rng, npar)
    g = np.sign(rng.standard_normal(npar)) * (0.5 + rng.random(npar))
    P1, m, v = M.adam_step(P, g, np.zeros(npar), np.zeros(npar), 1, 1e-3)
    np.testing.assert_allclose(P1[M.HDR:] - P[M.HDR:], -1e-3 * np.sign(g[M.HDR:]), rtol=1e-6, atol=1e-9)
    np.testing.assert_array_equal(P1[:M.HDR], P[:M.HDR])


def test_tf32_rounding():
    """The oracle's TF32 rounding (cvt.rna.tf32.f32: 10 explicit mantissa bits,
    to nearest, ties away from zero) and the tensor-core mode's closeness to the
    exact one."""
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -10)
    assert M.tf32(one + ulp / 2) == one + ulp  # a tie rounds away from zero
    assert M.tf32(-(one + ulp / 2)) == -(one + ulp)
    assert M.tf32(one + ulp / 2 - np.float32(2.0 ** -20)) == one
    assert M.tf32(np.float32(3.0)) == 3.0
    rng = np.random.default_rng(3)
    npar = M.unpack(np.zeros(20000))[4]
    P = _params(rng, npar)
    X = rng.standard_normal((50, 64))
    ye, yt = M.predict(P, X), M.predict(P, X, tc=True)
    assert 0 < np.abs(ye - yt).max() <= 1e-2 * np.abs(ye).max()
