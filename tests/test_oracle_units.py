"""Analytic anchors of the oracle's pieces (independent of any fixture)."""
import numpy as np
import pytest

W = [4 / 9] + [1 / 9] * 4 + [1 / 36] * 4
EX = [0, 1, 0, -1, 0, 1, -1, -1, 1]
EY = [0, 0, 1, 0, -1, 1, 1, -1, -1]


@pytest.mark.parametrize("rho,ux,uy", [(1.0, 0.0, 0.0), (1.02, 0.05, -0.01), (0.97, -0.08, 0.03)])
def test_feq_moments(orc, rho, ux, uy):
    f = [orc.feq(k, rho, ux, uy) for k in range(9)]
    assert sum(f) == pytest.approx(rho, abs=1e-15)
    assert sum(e * v for e, v in zip(EX, f)) == pytest.approx(rho * ux, abs=1e-15)
    assert sum(e * v for e, v in zip(EY, f)) == pytest.approx(rho * uy, abs=1e-15)
    pxx = sum(e * e * v for e, v in zip(EX, f))
    assert pxx == pytest.approx(rho / 3 + rho * ux * ux, abs=1e-14)


def test_spline_interpolates_knots(orc):
    """Spline3_S returns f at both ends of its interval whatever the moments."""
    for fi_1, fi, m1, m2 in [(1.0, 2.0, 0.3, -0.7), (0.1, 0.1, 5.0, 5.0)]:
        assert orc.spline3_s(3.0, 3.0, 1.0, fi_1, fi, m1, m2) == pytest.approx(fi_1, abs=1e-15)
        assert orc.spline3_s(4.0, 3.0, 1.0, fi_1, fi, m1, m2) == pytest.approx(fi, abs=1e-15)


def test_spline_keeps_reference_constant(orc):
    """The reference writes 1/6 as 0.1666667 (assit_multi.h:128-131)."""
    mid = orc.spline3_s(0.5, 0.0, 1.0, 0.0, 0.0, 1.0, 1.0)
    # a + b + c + d with a = b = 0.125 c6, c = d = -0.5 c6, c6 = 0.1666667
    assert mid == pytest.approx(-0.75 * 0.1666667, rel=1e-15)


def test_gtsv_matches_dense_solve(orc):
    rng = np.random.default_rng(0)
    for n in (2, 3, 9, 81, 513):
        l = np.full(n, 0.5); m = np.full(n, 2.0); u = np.full(n, 0.5)
        l[0] = 0; u[n - 1] = 0
        u[0] = 0
        if n > 1: l[1] = 0
        if n >= 2: u[n - 2] = 0; l[n - 1] = 0
        A = np.diag(m) + np.diag(l[1:], -1) + np.diag(u[:-1], 1)
        B = rng.standard_normal((n, 12))
        X = orc.gtsv(l, m, u, B)
        np.testing.assert_allclose(A @ X, B, atol=1e-13)


def test_temporal_weights_are_lagrange(orc):
    for xm in (0.0, 0.25, 0.5, 0.75, 1.0):
        a = 0.5 * (xm - 1) * xm
        b = (xm - 1) * (xm + 1)
        c = 0.5 * xm * (xm + 1)
        assert a - b + c == pytest.approx(1.0, abs=1e-15)      # constants are kept
        assert -a + c == pytest.approx(xm, abs=1e-15)          # linear data on nodes -1, 0, 1


def test_oracle_thread_count_does_not_change_results(mb, orc):
    g = mb.geo_init(mb.layout_builtin("2_5"), mb.make_config(64, 32, 3, 15, 15))
    res = []
    for t in (1, 4):
        orc.set_threads(t)
        o = orc.Oracle(g)
        o.init()
        o.evolution(20)
        res.append(np.concatenate([o.fields(a)["F"].ravel() for a in range(5)]))
    orc.set_threads(0)
    assert np.array_equal(res[0], res[1])


def test_settle_step_and_strouhal():
    import mblbm
    x = [1.2, 1.1, 1.004, 0.997, 1.001, 1.0]
    assert mblbm.settle_step(x, 1.0) == 2
    assert mblbm.settle_step([1.0] * 4, 1.0) == 0
    assert mblbm.settle_step([1.0, 1.0, 1.1], 1.0) == 3
    t = np.arange(4000)
    cl = 0.3 * np.sin(2 * np.pi * t / 250.0 + 0.3)
    st = mblbm.strouhal(cl, D=20, U0=0.05)
    assert abs(st - 20 / (250.0 * 0.05)) < 1e-3
    assert mblbm.strouhal(np.zeros(100), 20, 0.05) is None


def test_unet_oracle_gradients_finite_differences():
    """The CPU oracle's backward pass against central differences of its own
    loss (exact arithmetic, BF16 rounding off), on sampled parameters."""
    import unet_ref
    unet_ref.ROUND = False
    try:
        rng = np.random.default_rng(5)
        N, H, W = 1, 8, 16
        parts = []
        for ci, co, _ in unet_ref.LAYERS:  # He-scaled, as the device initialisation
            parts += [rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)), 0.05 * rng.standard_normal(co)]
        parts += [rng.standard_normal(96) * np.sqrt(1.0 / 32), 0.05 * rng.standard_normal(3)]
        p = np.concatenate(parts)
        n = len(p)
        inp = rng.standard_normal((N, H, W, 4))
        tgt = rng.standard_normal((N, H, W, 3))
        mask = (rng.random((N, H, W)) > 0.3).astype(np.float64)
        _, loss, g = unet_ref.forward_backward(p, inp, tgt, mask)
        idx = rng.choice(n, 40, replace=False)
        idx = np.concatenate([idx, [n - 1, n - 50, 5, 16 * 9 * 32 + 3]])
        eps = 1e-6
        for i in idx:
            q = p.copy(); q[i] += eps
            lp = unet_ref.forward_backward(q, inp, tgt, mask)[1]
            q[i] -= 2 * eps
            lm = unet_ref.forward_backward(q, inp, tgt, mask)[1]
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)) + 1e-8, (i, fd, g[i])
    finally:
        unet_ref.ROUND = True
