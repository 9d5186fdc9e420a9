"""Packed observables on the connected-configuration engine (``code/measure/transverse_spin.py``,
``code/measure/dwave_packed.py``, keys of ``code/measure/observables.py:120-150``).

Each call evaluates one operator family O = sum_t O_t in one C-ABI call (``nh_observable``): the
connections of every term are generated on the GPU, their amplitudes go through the same
pipeline as the local energy, and the local values are binned by term and averaged over the
samples.  ``transverse_terms`` gives T[0, r] = <S+_a S-_{a+r}>, T[1, r] = <S-_a S+_{a+r}> of a
reference site; ``PackedDwave`` the d-wave F and G terms of main-text Eq. (2) in the reference's
key order.
"""

from __future__ import annotations

import ctypes
from typing import Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .backflow import stream_ptr, workspace
from .state import Samples, Variational, as_spins

SPINS = ("u", "d")


def observable(state: Variational, samples: Samples, kind: int, arg0: int,
               arg1: int = 0) -> torch.Tensor:
    """Sample means (FP64 device tensor) of the terms of one family: kind ``OBS_TRANSVERSE_SPIN``
    (arg0 = reference site; (2, N)), ``OBS_PAIR`` (arg0, arg1 = sites of c+_up c+_dn; (4 N) over
    the bonds 4 site + 2 axis + orientation) or ``OBS_HOP`` (arg0 = site, arg1 = spin; (N))."""
    spins = as_spins(samples.spins, state.device)
    psi = samples.psi if samples.psi is not None else state(spins)
    B = spins.shape[0]
    N = state.N
    n_out = {_lib.OBS_TRANSVERSE_SPIN: 2 * N, _lib.OBS_PAIR: 4 * N, _lib.OBS_HOP: N}[kind]
    out = torch.empty(n_out, dtype=torch.float64, device=state.device)
    p = state.model.c_params()
    nbytes = _lib.load().nh_observable_workspace_bytes(B, state.n_symm, kind, ctypes.byref(p))
    ws = workspace(nbytes, state.device, "observable")
    _lib.call("nh_observable", spins.data_ptr(), psi.sign.contiguous().data_ptr(),
              psi.logabs.contiguous().data_ptr(), B, state.n_symm, ctypes.byref(p), kind,
              int(arg0), int(arg1), out.data_ptr(), ws.data_ptr(), ws.numel(),
              stream_ptr(state.device))
    return out.reshape(2, N) if kind == _lib.OBS_TRANSVERSE_SPIN else out


def transverse_terms(state: Variational, samples: Samples, ref: Tuple[int, int]) -> torch.Tensor:
    """(2, N): T[0, r] = <S+_a S-_{a+r}>, T[1, r] = <S-_a S+_{a+r}> for the reference site
    a = ref, r = 0 holding n_up (1 - n_dn) and n_dn (1 - n_up) at a (``transverse_spin.py:
    109-119``)."""
    Ly = state.model.geom.LY
    return observable(state, samples, _lib.OBS_TRANSVERSE_SPIN, int(ref[0]) * Ly + int(ref[1]))


class PackedDwave:
    """F and G terms of the d-wave measurement at R (``dwave_packed.py:33-103``): left bonds
    touching R (+x and +y with ``primary_only``), all right bonds and sites.  F[bl, oL, br, oR] =
    <A+(bl, oL) A(br, oR)> with A+(bond, o) = c+_{a up} c+_{b dn}, (a, b) the (lower, upper)
    ends for o = 0 and swapped for o = 1; G[i, j, s] = <c+_{i s} c_{j s}>."""

    DIRS = ((1, 0), (-1, 0), (0, 1), (0, -1))

    def __init__(self, LX: int, LY: int, R: Sequence[int] = (0, 0), primary_only: bool = True):
        self.LX, self.LY = LX, LY
        dirs = self.DIRS[::2] if primary_only else self.DIRS
        self.left_bonds = sorted({self._canon_bond(tuple(R), d) for d in dirs})
        self.left_sites = sorted({s for b in self.left_bonds for s in self.bond_sites(b)})
        sites = [(x, y) for x in range(LX) for y in range(LY)]
        all_bonds = [(x, y, ax) for (x, y) in sites for ax in (0, 1)]
        self.F_keys = [(bl, oL, br, oR) for bl in self.left_bonds for oL in (0, 1)
                       for br in all_bonds for oR in (0, 1)]
        self.G_keys = [(i, j, s) for i in self.left_sites for j in sites for s in SPINS]

    def _wrap(self, site):
        return (site[0] % self.LX, site[1] % self.LY)

    def _canon_bond(self, site, d):
        if d[0] + d[1] < 0:
            site = (site[0] + d[0], site[1] + d[1])
        return (*self._wrap(site), 0 if d[0] != 0 else 1)

    def bond_sites(self, bond):
        x, y, axis = bond
        return (x, y), self._wrap((x + 1, y) if axis == 0 else (x, y + 1))

    def index(self, site) -> int:
        return int(site[0]) * self.LY + int(site[1])

    def measure(self, state: Variational, samples: Samples):
        """(F, G) sample means in the order of F_keys, G_keys (numpy FP64)."""
        if samples.psi is None:
            samples = Samples(samples.spins, state(samples.spins))
        F = []
        for bl in self.left_bonds:
            lo, hi = self.bond_sites(bl)
            for oL in (0, 1):
                a, b = (lo, hi) if oL == 0 else (hi, lo)
                F.append(observable(state, samples, _lib.OBS_PAIR, self.index(a),
                                    self.index(b)).cpu().numpy())
        G = []
        for i in self.left_sites:
            gu = observable(state, samples, _lib.OBS_HOP, self.index(i), 0).cpu().numpy()
            gd = observable(state, samples, _lib.OBS_HOP, self.index(i), 1).cpu().numpy()
            G.append(np.stack([gu, gd], axis=1).reshape(-1))
        return np.concatenate(F), np.concatenate(G)
