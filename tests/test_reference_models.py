"""The oracle's pairing matrices and d-wave form factor against vectors computed by the
reference's own einsum paths (``code/backflow/models.py:69-84,163-196,272-281``), generated by
``tests/golden/make_models_golden.py`` (CPU only).  The reference stores the pair distances in
FP32, so the envelope agrees with the oracle's FP64 one to ~1e-8 relative; the form factor and
the feature split agree exactly."""

import os

import numpy as np
import pytest

from oracle import backflow as obf
from oracle import bcs as obcs
from oracle import lattice as olat

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "models_golden.npz"))
CASES = [tuple(int(v) for v in c) for c in G["cases"]]


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("k", range(len(CASES)))
def test_pair_tables(k):
    LX, LY, _ = CASES[k]
    disp, _, dist = olat.displacement_tables(LX, LY)
    assert np.array_equal(dist[disp].astype(np.float32), G[f"dist_{k}"])
    # F^d: -1 on x bonds, +1 on y bonds, as a function of i - j
    assert np.array_equal(obcs.dwave_factor(LX, LY)[disp], G[f"fd_{k}"])
    assert np.count_nonzero(G[f"fd_{k}"]) > 0


@pytest.mark.parametrize("k", range(len(CASES)))
def test_pfaffian_einsum_path(k):
    """Network output x (2 d, LX, LY) -> features: channels [0, d) spin up, [d, 2 d) down, site
    x Ly + y; then the (2N, 2N) antisymmetric matrix of the einsum path."""
    LX, LY, d = CASES[k]
    N = LX * LY
    for b, x in enumerate(G[f"x_{k}"]):
        y = np.swapaxes(x.reshape(2, d, N), 1, 2)
        F = obf.pairing_matrix_einsum(y, G[f"W_{k}"], float(G[f"theta_{k}"]), LX, LY)
        assert rel(F, G[f"Fpf_{k}"][b]) < 1e-7


def test_oracle_cnn_split_matches_reference_split():
    """The oracle's network output -> feature split is the reference's (a one-layer network
    with a centre-tap kernel, whose output is known in closed form)."""
    LX, LY, d = 4, 4, 8
    rng = np.random.default_rng(5)
    s = olat.random_configs(rng, 2, LX * LY, 7, 7)
    w = np.zeros((2 * d, 2, 3, 3))
    w[:, :, 1, 1] = rng.normal(size=(2 * d, 2))
    b = rng.normal(size=2 * d)
    img = s.reshape(2, 2, LX, LY).astype(np.float64)
    x = b[None, :, None, None] + np.einsum("oi,bixy->boxy", w[:, :, 1, 1], img)
    y = obf.cnn_forward(s, [w], [b], LX, LY)
    assert np.allclose(y, np.swapaxes(x.reshape(2, 2, d, LX * LY), 2, 3), rtol=0, atol=1e-13)


@pytest.mark.parametrize("k", range(len(CASES)))
def test_bcs_einsum_path(k):
    LX, LY, d = CASES[k]
    N = LX * LY
    Wud = obcs.wt_ud(G[f"Wb_{k}"], float(G[f"thetab_{k}"]), LX, LY)
    sites = np.arange(N)[None]
    for b, y in enumerate(G[f"y_{k}"]):
        F = obcs.occupied_block(y[0][None], sites, y[1][None], sites, Wud,
                                float(G[f"delta_{k}"]), LX, LY)[0]
        assert rel(F, G[f"Fbcs_{k}"][b]) < 1e-7
