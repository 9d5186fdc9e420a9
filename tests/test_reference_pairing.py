"""The oracle's pairing tables and occupied gathers against vectors computed by the reference's
own functions (``code/backflow/pf_kernel.py:83-124,368-401``, ``code/backflow/bcs_kernel.py:
63-71,293-315``), run in FP64 by ``tests/golden/make_pairing_golden.py`` (CPU only).  The GPU
kernels are checked against this oracle in ``test_gpu_parity.py`` and ``test_gpu_bcs.py``.

The reference keeps the minimum-image distances D_r in FP32 (``pf_kernel.py:95``) and the
oracle in FP64, so the envelope tables agree to ~1e-8 relative; the gathers are compared on the
reference's own tables, where they agree to rounding."""

import os

import numpy as np
import pytest

from oracle import backflow as obf
from oracle import bcs as obcs
from oracle import lattice as olat

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "pairing_golden.npz"))
CASES = [tuple(int(v) for v in c) for c in G["cases"]]


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("k", range(len(CASES)))
def test_displacement_tables(k):
    LX, LY = CASES[k][:2]
    disp, neg, dist = olat.displacement_tables(LX, LY)
    assert np.array_equal(disp, G[f"disp_{k}"])
    assert np.array_equal(neg, G[f"neg_{k}"])
    assert np.array_equal(dist.astype(np.float32), G[f"dist_{k}"])


@pytest.mark.parametrize("k", range(len(CASES)))
def test_wtilde_tables(k):
    LX, LY = CASES[k][:2]
    W, theta = G[f"W_{k}"], float(G[f"theta_{k}"])
    Wt = G[f"Wt_{k}"]
    assert rel(obf.build_wtilde(W, theta, LX, LY), Wt) < 1e-7
    assert rel(obcs.wt_ud(W[0], theta, LX, LY), G[f"Wud_{k}"]) < 1e-7
    # the reference's table is exactly antisymmetric: Wt[2 sq + sp, -r] = -Wt[2 sp + sq, r]
    neg = G[f"neg_{k}"]
    for sp in (0, 1):
        for sq in (0, 1):
            assert np.array_equal(Wt[2 * sq + sp][neg], -Wt[2 * sp + sq])


@pytest.mark.parametrize("k", range(len(CASES)))
def test_pfaffian_gather(k):
    LX, LY = CASES[k][:2]
    N = LX * LY
    s, y, F = G[f"s_{k}"], G[f"y_{k}"], G[f"F_{k}"]
    idx = np.stack([np.flatnonzero(c > 0) for c in s])
    assert np.array_equal(idx, obf.fermion_idx(s))
    Y = obf.occupied_features(y.reshape(len(s), 2 * N, -1), idx)
    assert rel(obf.pairing_occ(Y, idx, G[f"Wt_{k}"], LX, LY), F) < 1e-13
    # the oracle end to end (its own FP64 envelope) and its einsum twin of models.py:169-196
    Wt = obf.build_wtilde(G[f"W_{k}"], float(G[f"theta_{k}"]), LX, LY)
    assert rel(obf.pairing_occ(Y, idx, Wt, LX, LY), F) < 1e-7
    for b in range(len(s)):
        full = obf.pairing_matrix_einsum(y[b], G[f"W_{k}"], float(G[f"theta_{k}"]), LX, LY)
        assert rel(full[np.ix_(idx[b], idx[b])], F[b]) < 1e-7


@pytest.mark.parametrize("k", range(len(CASES)))
def test_bcs_gather(k):
    LX, LY = CASES[k][:2]
    N = LX * LY
    s, y, Fud = G[f"s_{k}"], G[f"y_{k}"], G[f"Fud_{k}"]
    iu = np.stack([np.flatnonzero(c[:N] > 0) for c in s])
    idn = np.stack([np.flatnonzero(c[N:] > 0) for c in s])
    Yu = np.take_along_axis(y[:, 0], iu[:, :, None], axis=1)
    Yd = np.take_along_axis(y[:, 1], idn[:, :, None], axis=1)
    got = obcs.occupied_block(Yu, iu, Yd, idn, G[f"Wud_{k}"], 0.0, LX, LY)
    assert rel(got, Fud) < 1e-13
