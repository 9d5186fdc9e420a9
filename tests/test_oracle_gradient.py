"""The FP64 oracle's per-sample Jacobian of log|psi| against central finite differences of the
oracle's own amplitude (CPU only).  The oracle restates the backward of
``code/backflow/models.py:198-211`` link by link (Pfaffian adjoint, the custom VJP of
``pf_kernel.py:354-365``, ``build_wtilde``'s backward, the CNN backward, the projection)."""

import numpy as np
import pytest

from oracle import backflow as ob
from oracle import gradient as og
from oracle import lattice as olat
from oracle import pfaffian as opf
from oracle import projection as oproj


def small_params(Lx, Ly, C, layers, std, seed):
    rng = np.random.default_rng(seed)
    conv_w, conv_b, cin = [], [], 2
    for _ in range(layers):
        conv_w.append(rng.normal(0, std, (C, cin, 3, 3)))
        conv_b.append(rng.normal(0, std, (C,)))
        cin = C
    d = C // 2
    W = rng.normal(0, 1, (3, Lx * Ly, d)) / np.sqrt(d)
    return dict(conv_w=conv_w, conv_b=conv_b, W=W, theta=0.55, Lx=Lx, Ly=Ly)


@pytest.mark.parametrize("symm", [False, True])
def test_jacobian_matches_finite_differences(symm):
    p = small_params(4, 4, 8, 3, 0.4, 1)
    s = olat.random_configs(np.random.default_rng(2), 3, 16, 7, 7)
    sg, la, J = og.log_jacobian(s, p, symm=symm)
    s0, l0 = oproj.projected_amplitude(s, p, symm=symm)
    assert np.array_equal(sg, s0) and np.allclose(la, l0, atol=1e-12)
    assert J.shape == (3, og.param_count(p))
    vec = og.flatten_params(p)
    rng = np.random.default_rng(5)
    cols = list(rng.choice(len(vec), 40, replace=False)) + [0, len(vec) - 2, len(vec) - 1]
    h = 1e-5
    for k in cols:
        vp, vm = vec.copy(), vec.copy()
        vp[k] += h
        vm[k] -= h
        lp = oproj.projected_amplitude(s, og.unflatten_params(vp, p), symm=symm)[1]
        lm = oproj.projected_amplitude(s, og.unflatten_params(vm, p), symm=symm)[1]
        fd = (lp - lm) / (2 * h)
        scale = max(1e-3, np.max(np.abs(J[:, k])))
        assert np.max(np.abs(fd - J[:, k])) < 1e-6 * max(1.0, scale), (k, fd, J[:, k])


def test_slogpf_adjoint_directional_derivative():
    rng = np.random.default_rng(7)
    A = rng.normal(size=(4, 10, 10))
    A = A - np.swapaxes(A, 1, 2)
    E = rng.normal(size=(4, 10, 10))
    E = E - np.swapaxes(E, 1, 2)
    G = og.slogpf_adjoint(A)
    h = 1e-6
    fd = (opf.slogpf(A + h * E)[1] - opf.slogpf(A - h * E)[1]) / (2 * h)
    assert np.allclose(np.einsum("bpq,bpq->b", G, E), fd, rtol=1e-6, atol=1e-8)


def test_pairing_vjp_is_the_adjoint_of_the_gather():
    """<G, dF> = <dY, dY_dir> + <dWt, dWt_dir> for random directions (linearisation)."""
    Lx = Ly = 4
    rng = np.random.default_rng(3)
    s = olat.random_configs(rng, 2, 16, 7, 7)
    idx = ob.fermion_idx(s)
    Y = rng.normal(size=(2, 14, 4))
    Wt = ob.build_wtilde(rng.normal(size=(3, 16, 4)), 0.3, Lx, Ly)
    G = rng.normal(size=(2, 14, 14))
    dY, dWt = og.pairing_occ_vjp(Y, idx, Wt, G, Lx, Ly)
    vY = rng.normal(size=Y.shape)
    vW = rng.normal(size=Wt.shape)
    h = 1e-6
    Fp = ob.pairing_occ(Y + h * vY, idx, Wt + h * vW, Lx, Ly)
    Fm = ob.pairing_occ(Y - h * vY, idx, Wt - h * vW, Lx, Ly)
    lhs = np.einsum("bpq,bpq->b", G, (Fp - Fm) / (2 * h))
    rhs = np.einsum("bpa,bpa->b", dY, vY) + np.einsum("bkra,kra->b", dWt, vW)
    assert np.allclose(lhs, rhs, rtol=1e-7, atol=1e-9)
