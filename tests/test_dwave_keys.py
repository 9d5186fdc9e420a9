"""The packed d-wave key orders against the reference's own ``dwave_keys`` and
``string_sites`` (``code/measure/observables.py:96-154``), through the golden fixture that
``tests/golden/make_dwave_keys.py`` generated from the reference (CPU only).  The GPU kernel's
term binning is checked against ``oracle.observables`` in ``test_gpu_observables.py``; this file
pins that oracle's bond orientation, and the host-side key lists, to the reference."""

import os

import numpy as np
import pytest

from neuralhubbard_b200.observables import PackedDwave
from oracle import observables as oobs

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "dwave_keys.npz"))
CASES = [tuple(int(v) for v in c) for c in GOLDEN["cases"]]


@pytest.mark.parametrize("k", range(len(CASES)))
def test_packed_dwave_keys_match_reference(k):
    LX, LY, rx, ry, primary = CASES[k]
    dw = PackedDwave(LX, LY, R=(rx, ry), primary_only=bool(primary))
    F = np.array([(*bl, oL, *br, oR) for bl, oL, br, oR in dw.F_keys], np.int32)
    G = np.array([(*i, *j, "ud".index(s)) for i, j, s in dw.G_keys], np.int32)
    assert np.array_equal(F, GOLDEN[f"F_{k}"])
    assert np.array_equal(G, GOLDEN[f"G_{k}"])
    assert np.array_equal(np.array(dw.left_bonds, np.int32), GOLDEN[f"left_{k}"])


@pytest.mark.parametrize("k", range(len(CASES)))
def test_pair_term_orientation_matches_reference(k):
    """Term t = 2 bond + o = 4 site + 2 axis + o is A+(bond, o) with the reference's
    (c+_up site, c+_dn site); the left-bond operators of ``PackedDwave.measure`` use the same
    orientation."""
    LX, LY, rx, ry, primary = CASES[k]
    strings = GOLDEN[f"strings_{k}"]
    assert np.array_equal(np.array(oobs.bond_pairs(LX, LY), np.int32), strings)
    dw = PackedDwave(LX, LY, R=(rx, ry), primary_only=bool(primary))
    for bl in dw.left_bonds:
        lo, hi = dw.bond_sites(bl)
        t = 2 * (2 * dw.index(bl[:2]) + bl[2])
        assert (dw.index(lo), dw.index(hi)) == tuple(strings[t])
        assert (dw.index(hi), dw.index(lo)) == tuple(strings[t + 1])
