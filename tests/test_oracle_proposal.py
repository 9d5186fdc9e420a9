"""CPU checks of the learned-proposal oracle: the hand-derived gradient against central finite
differences, reverse moves, BF16 rounding and the exact Hastings correction (detailed balance
of the learned-proposal transition matrix on a tiny lattice)."""

import numpy as np
import pytest

from oracle import lattice as olat
from oracle import proposal as P


def test_gradient_matches_finite_differences():
    Lx, Ly = 4, 5
    rng = np.random.default_rng(0)
    s = olat.random_configs(rng, 3, Lx * Ly, 6, 7)
    th = P.init_params(1, 0.3).astype(np.float64)
    lq = P.log_q(s, th, Lx, Ly)
    mv = [int(rng.choice(np.flatnonzero(np.isfinite(r)))) for r in lq]
    w = np.array([0.3, 1.0, 0.7])
    _, g = P.loss_and_grad(s, mv, w, th, Lx, Ly)
    eps = 1e-5
    for k in rng.choice(P.PARAM_COUNT, 40, replace=False):
        tp, tm = th.copy(), th.copy()
        tp[k] += eps
        tm[k] -= eps
        fd = (P.loss_and_grad(s, mv, w, tp, Lx, Ly)[0] - P.loss_and_grad(s, mv, w, tm, Lx, Ly)[0])
        fd /= 2 * eps
        assert abs(fd - g[k]) < 1e-6 + 1e-5 * abs(g[k]), (k, fd, g[k])


def test_reverse_move_and_masks():
    Lx, Ly = 3, 4
    rng = np.random.default_rng(1)
    s = olat.random_configs(rng, 5, Lx * Ly, 4, 5)
    th = P.init_params(2, 0.2)
    for n_dirs in (4, 8):
        lq = P.log_q(s, th, Lx, Ly, n_dirs)
        assert np.allclose(np.exp(lq).sum(1), 1.0)
        mv = [int(rng.choice(np.flatnonzero(np.isfinite(r)))) for r in lq]
        sp, _, _ = P.apply_move(s, mv, Lx, Ly)
        rm = P.reverse_move(mv, Lx, Ly)
        assert np.isfinite(P.log_q(sp, th, Lx, Ly, n_dirs)[np.arange(5), rm]).all()
        s2, _, _ = P.apply_move(sp, rm, Lx, Ly)
        assert np.array_equal(s2, s)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -3.3e-5, 7.0e12], np.float32)
    r = P.round_bf16(x)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0**-8)
    assert r[1] == 1.0 and r[2] == 1.015625  # ties to even


def test_learned_transition_satisfies_detailed_balance():
    """T(s -> s') = q(m | s) min(1, |psi'|^2 q(m' | s') / (|psi|^2 q(m | s))) satisfies
    |psi(s)|^2 T(s -> s') = |psi(s')|^2 T(s' -> s) for every pair, for any network."""
    Lx, Ly, nu, nd = 3, 3, 1, 2
    N = Lx * Ly
    basis = []
    for up in range(N):
        for d1 in range(N):
            for d2 in range(d1 + 1, N):
                c = -np.ones(2 * N, np.int8)
                c[up] = 1
                c[N + d1] = c[N + d2] = 1
                basis.append(c)
    basis = np.array(basis)
    index = {b.tobytes(): k for k, b in enumerate(basis)}
    rng = np.random.default_rng(3)
    logpsi = rng.normal(size=len(basis))
    th = P.init_params(4, 0.5)
    lq = P.log_q(basis, th, Lx, Ly)
    T = np.zeros((len(basis), len(basis)))
    for a in range(len(basis)):
        for m in np.flatnonzero(np.isfinite(lq[a])):
            sp, _, _ = P.apply_move(basis[a : a + 1], [m], Lx, Ly)
            b = index[sp[0].tobytes()]
            rm = P.reverse_move([m], Lx, Ly)[0]
            ratio = np.exp(2 * (logpsi[b] - logpsi[a]) + lq[b, rm] - lq[a, m])
            T[a, b] += np.exp(lq[a, m]) * min(1.0, ratio)
    p = np.exp(2 * logpsi)
    flux = p[:, None] * T
    assert np.allclose(flux, flux.T, rtol=1e-12, atol=1e-15)
