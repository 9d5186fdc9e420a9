"""The library's envelope table and occupied gather (``nh_build_wtilde``, ``nh_pairing_occ``)
against vectors computed by the reference's own ``build_wtilde`` and ``pairing_matrix_occ``
(``code/backflow/pf_kernel.py:107-124,384-401``; generated in FP64 by
``tests/golden/make_pairing_golden.py``).  The reference keeps the distances D_r in FP32, so
the FP64 table agrees to ~1e-8 relative; the FP32 outputs agree to FP32 rounding."""

import os

import numpy as np
import pytest
import torch

import neuralhubbard_b200 as nh

pytestmark = pytest.mark.gpu
DEV = "cuda"
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "pairing_golden.npz"))
CASES = [tuple(int(v) for v in c) for c in G["cases"]]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("k", range(len(CASES)))
def test_wtilde_and_gather_against_reference_vectors(k):
    LX, LY, d, n_up, n_dn = CASES[k]
    N = LX * LY
    geom = nh.PairGeometry(LX, LY, d, n_up, n_dn)
    W = torch.from_numpy(G[f"W_{k}"].astype(np.float32)).to(DEV)
    theta = float(G[f"theta_{k}"])
    Wt, Wt64 = nh.build_wtilde(W, theta, geom, fp64=True)
    # the inputs were rounded to FP32 here; the reference ran on the FP64 values
    assert rel(Wt.cpu().numpy(), G[f"Wt_{k}"]) < 1e-6
    assert rel(Wt64.cpu().numpy(), G[f"Wt_{k}"]) < 1e-6
    s, y, F0 = G[f"s_{k}"], G[f"y_{k}"], G[f"F_{k}"]
    idx = np.stack([np.flatnonzero(c > 0) for c in s]).astype(np.int32)
    Y = np.take_along_axis(y.reshape(len(s), 2 * N, d), idx[:, :, None].astype(np.int64), 1)
    F = nh.pairing_occ(torch.from_numpy(Y.astype(np.float32)).to(DEV),
                       torch.from_numpy(idx).to(DEV), Wt, geom).cpu().numpy()
    assert np.array_equal(F, -np.swapaxes(F, 1, 2))
    assert rel(F, F0) < 1e-5
