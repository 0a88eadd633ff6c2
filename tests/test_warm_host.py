"""Learned warm start, host side: the oracle's network gradient against
finite differences, the kernel-rounded gradient against the exact one, the
Grad-13 seed against its own moments, and the case scalings."""
import math

import numpy as np
import pytest

from oracle import warm_oracle as W


def _batch(n=48, seed=0):
    rng = np.random.default_rng(seed)
    q = np.column_stack([rng.uniform(0, 1, n), rng.uniform(0, 1, n),
                         rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)])
    X = W.features(q)
    T = np.zeros((n, W.N_OUT), np.float32)
    T[:, :W.N_USED] = rng.normal(size=(n, W.N_USED))
    return X, T


def _params(seed=0):
    from alebgk4paper_b200.warmstart import init_params
    p = init_params(seed)
    p[W.B_OFF[0]:] = np.random.default_rng(seed + 1).normal(0, 0.1, W.N_PARAMS - W.B_OFF[0])
    p[W.B_OFF[4] + W.N_USED:] = 0
    return p


def test_parameter_layout_matches_the_library():
    from alebgk4paper_b200 import _abi
    assert W.N_PARAMS == _abi.load().alebgk_net_nparams() == 59920


def test_exact_gradient_matches_finite_differences():
    X, T = _batch()
    p = _params().astype(np.float64)
    w = np.linspace(0.5, 2.0, W.N_USED)
    g = W.grad_exact(p, X, T, w)
    rng = np.random.default_rng(3)
    picks = list(rng.choice(W.N_PARAMS, 40, replace=False)) + [W.B_OFF[l] + 3 for l in range(5)]
    for i in picks:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (W.loss_exact(pp, X, T, w) - W.loss_exact(pm, X, T, w)) / (2 * h) / len(X)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])


def test_rounded_gradient_is_close_to_exact():
    X, T = _batch(256)
    p = _params()
    loss, g = W.loss_grad(p, X, T)
    ge = W.grad_exact(p.astype(np.float64), W.bf16(X), T)
    for l, (i, o) in enumerate(W.LAYERS):
        a = g[W.W_OFF[l]:W.W_OFF[l] + i * o].astype(np.float64)
        b = ge[W.W_OFF[l]:W.W_OFF[l] + i * o]
        assert np.linalg.norm(a - b) <= 0.03 * np.linalg.norm(b), l
    assert math.isclose(loss, W.loss_exact(p.astype(np.float64), W.bf16(X), T), rel_tol=0.02)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0], np.float32)
    r = W.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0          # tie to even
    assert r[2] == 1.0 + 4 * 2 ** -8            # tie to even, upwards
    assert r[3] == 1.0 and r[4] == -2.5 and r[5] == 0.0


@pytest.mark.parametrize("Nv", [16, 20, 24])
def test_grad13_rows_reproduce_their_moments(Nv):
    vmin, dv, R = -1303.0, 2 * 1303.0 / (Nv - 1), 208.0
    m = np.array([[1.3, 3.0, -2.0, 271.5, 40.0, -25.0, 10.0, 3e3, -2e3],
                  [0.6, -0.5, 0.2, 269.0, -3.0, 1.0, 2.0, -50.0, 80.0]])
    g1, g2 = W.grad13_rows(m, Nv, vmin, dv, R)
    mm = W.moments13(g1, g2, Nv, vmin, dv, R)
    assert np.allclose(mm[:, 0], m[:, 0], rtol=1e-7)
    assert np.allclose(mm[:, 1:4], m[:, 1:4], rtol=1e-6, atol=1e-6)
    # the velocity grid's quadrature error of the stress and heat flux
    assert np.allclose(mm[:, 4:], m[:, 4:], rtol=2e-3, atol=1e-9 * abs(m[:, 4:]).max())


def test_grad13_of_an_equilibrium_is_the_maxwellian():
    Nv, vmin, dv, R = 16, -1303.0, 2 * 1303.0 / 15, 208.0
    m = np.array([[1.0, 2.0, -1.0, 270.0, 0, 0, 0, 0, 0]])
    g1, g2 = W.grad13_rows(m, Nv, vmin, dv, R)
    vx, vy = W.velocity_grid(Nv, vmin, dv)
    th = R * 270.0
    M = 1.0 / (2 * np.pi * th) * np.exp(-((vx - 2.0) ** 2 + (vy + 1.0) ** 2) / (2 * th))
    assert np.allclose(g1[0], M, rtol=1e-13, atol=0)
    assert np.allclose(g2[0], 0.5 * th * M, rtol=1e-13, atol=0)   # MLSBasis.hpp:99-104


def test_case_scalings_round_trip():
    from alebgk4paper_b200 import Case
    from alebgk4paper_b200 import warmstart as ws
    c = Case("cavity2d", Nx=12, Nv=8, lid_speed=4.0, rho0=2.0, tau=3.7142e-10 / 2)
    q = ws.case_inputs(c)
    assert q.shape == (c.N, 4)
    assert q[:, :2].min() >= 0 and q[:, :2].max() <= 1
    assert -1 <= q[0, 2] <= 1 and -1 <= q[0, 3] <= 1
    rng = np.random.default_rng(0)
    mom = np.column_stack([2 + 0.01 * rng.normal(size=c.N), rng.normal(size=(c.N, 2)),
                           270 + rng.normal(size=c.N), rng.normal(size=(c.N, 5))])
    t = ws.case_targets(c, mom)
    mu, sd = rng.normal(size=9), rng.uniform(0.5, 2, 9)
    scale, shift = ws.denormalise(c, mu, sd)
    back = shift + scale * ((t.astype(np.float64) - mu) / sd)
    assert np.allclose(back, mom, rtol=1e-6, atol=1e-6)
