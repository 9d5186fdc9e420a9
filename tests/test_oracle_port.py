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


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_port_fp32_build_close_to_fp64():
    """The FP32 build (the arithmetic of the reference's own path) computes the same amplitudes
    to FP32 accuracy: same signs, log|psi| within 1e-3 on well-conditioned 4x4 and 8x8 cases
    with the benchmark's weight scale."""
    for L in (4, 8):
        rng = np.random.default_rng(10 + L)
        N = L * L
        ne = 7 * N // 16
        C = 32
        conv_w = [rng.normal(size=(C, 2 if l == 0 else C, 3, 3)) * 0.02 for l in range(4)]
        conv_b = [rng.normal(size=C) * 0.02 for _ in range(4)]
        params = dict(conv_w=conv_w, conv_b=conv_b, W=rng.normal(size=(3, N, C // 2)) / 4.0,
                      theta=0.55, Lx=L, Ly=L)
        s = olat.random_configs(rng, 6, N, ne, ne)
        s0, l0 = port.projected_amplitude(s, params, symm=True, threads=2)
        s1, l1 = port.projected_amplitude(s, params, symm=True, threads=2, fp32=True)
        assert np.array_equal(s1, s0)
        nz = s0 != 0  # the projection can vanish exactly on small lattices (logabs -inf)
        assert np.max(np.abs(l1[nz] - l0[nz])) < 1e-3, np.max(np.abs(l1[nz] - l0[nz]))
