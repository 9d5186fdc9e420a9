"""The compiled CPU restatement (oracle/c/nh_port.c, the CPU baseline of bench.py) against the
numpy oracle: same signs, log|psi| within 1e-9, projected and unprojected."""

import shutil

import numpy as np
import pytest

from oracle import lattice as olat
from oracle import port
from oracle import projection as oproj


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
@pytest.mark.parametrize("L,symm", [(4, True), (4, False), (8, True), (8, False)])
def test_port_matches_numpy_oracle(L, symm):
    rng = np.random.default_rng(L)
    N = L * L
    ne = 7 * N // 16
    C = 32
    conv_w = [rng.normal(size=(C, 2 if l == 0 else C, 3, 3)) * 0.3 for l in range(4)]
    conv_b = [rng.normal(size=C) * 0.3 for _ in range(4)]
    params = dict(conv_w=conv_w, conv_b=conv_b, W=rng.normal(size=(3, N, C // 2)) / 4.0,
                  theta=0.55, Lx=L, Ly=L)
    s = olat.random_configs(rng, 5, N, ne, ne)
    s0, l0 = oproj.projected_amplitude(s, params, symm=symm)
    s1, l1 = port.projected_amplitude(s, params, symm=symm, threads=2)
    assert np.array_equal(s1, s0)
    assert np.max(np.abs(l1 - l0)) < 1e-9, np.max(np.abs(l1 - l0))
