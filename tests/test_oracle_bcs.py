"""The BCS-backflow oracle (``code/backflow/models.py:214-302``) against the Pfaffian oracle:
the BCS amplitude is the Pfaffian of [[0, F], [-F^T, 0]], i.e. the Pfaffian state whose
same-spin pairing blocks vanish (CPU only)."""

import numpy as np
import pytest

from oracle import backflow as ob
from oracle import bcs
from oracle import lattice as olat
from oracle import pfaffian as opf
from oracle import projection as oproj


def params(L, seed, delta_d):
    rng = np.random.default_rng(seed)
    conv_w, conv_b, cin = [], [], 2
    for _ in range(3):
        conv_w.append(rng.normal(0, 0.3, (16, cin, 3, 3)))
        conv_b.append(rng.normal(0, 0.3, (16,)))
        cin = 16
    W = rng.normal(0, 1, (L * L, 8)) / np.sqrt(8)
    return dict(conv_w=conv_w, conv_b=conv_b, W=W, theta=0.55, delta_d=delta_d, Lx=L, Ly=L)


@pytest.mark.parametrize("symm", [False, True])
def test_bcs_equals_pfaffian_with_vanishing_same_spin_blocks(symm):
    p = params(4, 1, 0.0)
    s = olat.random_configs(np.random.default_rng(2), 6, 16, 7, 7)
    s1, l1 = bcs.projected_amplitude(s, p, symm=symm)
    s2, l2 = oproj.projected_amplitude(s, bcs.as_pfaffian_params(p), symm=symm)
    assert np.array_equal(s1, s2)
    assert np.allclose(l1, l2, atol=1e-10)


def test_bcs_dwave_term_as_block_pfaffian():
    p = params(4, 3, 0.37)
    L, N = 4, 16
    s = olat.random_configs(np.random.default_rng(4), 5, N, 7, 7)
    sg, la = bcs.amplitude(s, p)
    y = ob.cnn_forward(s, p["conv_w"], p["conv_b"], L, L)
    Wud = bcs.wt_ud(p["W"], p["theta"], L, L)
    for b in range(5):
        iu = np.nonzero(s[b, :N] > 0)[0]
        idn = np.nonzero(s[b, N:] > 0)[0]
        F = bcs.occupied_block(y[b : b + 1, 0][:, iu], iu[None], y[b : b + 1, 1][:, idn],
                               idn[None], Wud, 0.37, L, L)[0]
        n = F.shape[0]
        big = np.zeros((2 * n, 2 * n))
        big[:n, n:] = F
        big[n:, :n] = -F.T
        s0, l0 = opf.slogpf(big)
        assert np.isclose(l0, la[b], atol=1e-10)
        assert s0 * ob.fermion_inverse_sign(s[b : b + 1])[0] == sg[b]
