"""Hubbard local energy, FP64 oracle.

H = - sum_{<ij>, sigma} t_ij (c+_{i sigma} c_{j sigma} + h.c.) + U sum_i n_{i up} n_{i down}
with t_ij = t on the 4 nearest and t' on the 4 next-nearest neighbours of the periodic
lattice (``Hubbard(U=8, t=[1.0, t'], n_neighbor=[1, 2])``, ``code/states.py:244-247``).

E_loc(s) = sum_s' <s|H|s'> psi(s') / psi(s)  (``H.Oloc``, ``code/quick_start.py:33``).
The connected s' move one sigma-electron from occupied mode m to an empty neighbouring
mode m'; <s|H|s'> = -t_d (-1)^(number of occupied modes strictly between m and m'), the
Jordan-Wigner sign of the ordering |s> = c+_{m1} ... c+_{mk}|0>, m1 < ... < mk.
Connections are enumerated by occupied mode (ascending), then by hop direction in the order
of ``lattice.HOP_DIRS``.
"""

from __future__ import annotations

import itertools

import numpy as np

from . import lattice


def hops(s: np.ndarray, Lx: int, Ly: int, t: float, tp: float, n_dirs: int = 8):
    """Connections of one configuration: arrays (from_mode, to_mode, h) in enumeration
    order; h = <s|H|s'> for s' = s with the electron at from_mode moved to to_mode."""
    N = Lx * Ly
    nbr = lattice.neighbour_table(Lx, Ly)
    amp = lattice.hop_amplitudes(t, tp, n_dirs)
    occ = np.asarray(s) > 0
    cum = np.concatenate([[0], np.cumsum(occ)])
    fr, to, hv = [], [], []
    for m in np.flatnonzero(occ):
        sigma, i = divmod(int(m), N)
        for d in range(n_dirs):
            mj = sigma * N + int(nbr[i, d])
            if occ[mj]:
                continue
            lo, hi = (m, mj) if m < mj else (mj, m)
            between = cum[hi] - cum[lo + 1]
            fr.append(int(m))
            to.append(mj)
            hv.append(-amp[d] * (1.0 if between % 2 == 0 else -1.0))
    return np.array(fr, np.int64), np.array(to, np.int64), np.array(hv, np.float64)


def hop_counts(s: np.ndarray, Lx: int, Ly: int, n_dirs: int = 8) -> np.ndarray:
    """(B,) number of connections of each configuration."""
    N = Lx * Ly
    nbr = lattice.neighbour_table(Lx, Ly)
    occ = np.asarray(s) > 0
    cnt = np.zeros(occ.shape[0], np.int64)
    for sigma in range(2):
        o = occ[:, sigma * N : (sigma + 1) * N]
        for d in range(n_dirs):
            cnt += (o & ~o[:, nbr[:, d]]).sum(1)
    return cnt


def apply_hop(s: np.ndarray, fr: int, to: int) -> np.ndarray:
    out = np.array(s, copy=True)
    out[fr] = -1
    out[to] = 1
    return out


def double_occupancy(s: np.ndarray, N: int) -> np.ndarray:
    s = np.asarray(s)
    return ((s[..., :N] > 0) & (s[..., N:] > 0)).sum(-1)


def local_energy(s: np.ndarray, amp_fn, Lx: int, Ly: int, t: float, tp: float, U: float,
                 n_dirs: int = 8, psi=None):
    """E_loc of each configuration in s (B, 2N).  ``amp_fn(configs) -> (sign, logabs)``."""
    s = np.asarray(s)
    N = Lx * Ly
    if psi is None:
        psi = amp_fn(s)
    sg0, la0 = psi
    E = U * double_occupancy(s, N).astype(np.float64)
    for b in range(s.shape[0]):
        fr, to, hv = hops(s[b], Lx, Ly, t, tp, n_dirs)
        if len(fr) == 0:
            continue
        conn = np.repeat(s[b][None], len(fr), axis=0)
        conn[np.arange(len(fr)), fr] = -1
        conn[np.arange(len(fr)), to] = 1
        sg, la = amp_fn(conn)
        E[b] += np.sum(hv * sg * sg0[b] * np.exp(la - la0[b]))
    return E


# ---------------------------------------------------------------- Fock-space brute force


def _apply_annihilate(bits: int, m: int):
    if not (bits >> m) & 1:
        return None, 0
    sign = -1 if bin(bits & ((1 << m) - 1)).count("1") % 2 else 1
    return bits & ~(1 << m), sign


def _apply_create(bits: int, m: int):
    if (bits >> m) & 1:
        return None, 0
    sign = -1 if bin(bits & ((1 << m) - 1)).count("1") % 2 else 1
    return bits | (1 << m), sign


def fock_basis(N: int, n_up: int, n_dn: int) -> np.ndarray:
    """All (n_up, n_dn) configurations as (D, 2N) int8 +-1."""
    out = []
    for up in itertools.combinations(range(N), n_up):
        for dn in itertools.combinations(range(N), n_dn):
            s = -np.ones(2 * N, np.int8)
            s[list(up)] = 1
            s[[N + j for j in dn]] = 1
            out.append(s)
    return np.array(out)


def hamiltonian_matrix(basis: np.ndarray, Lx: int, Ly: int, t: float, tp: float, U: float):
    """Dense <s|H|s'> on ``basis`` from explicit fermion operators (mode m is bit m, and
    c_m anticommutes past the occupied modes below m)."""
    N = Lx * Ly
    D = basis.shape[0]
    key = {}
    bits_of = []
    for a, s in enumerate(basis):
        b = 0
        for m in np.flatnonzero(s > 0):
            b |= 1 << int(m)
        key[b] = a
        bits_of.append(b)
    x, y = lattice.site_xy(Lx, Ly)
    bonds = []
    for (dx, dy, amp) in [(1, 0, t), (0, 1, t), (1, 1, tp), (1, -1, tp)]:
        if amp == 0:
            continue
        j = ((x + dx) % Lx) * Ly + (y + dy) % Ly
        for i in range(N):
            bonds.append((i, int(j[i]), amp))
    H = np.zeros((D, D))
    for a, b in enumerate(bits_of):
        H[a, a] += U * sum(((b >> i) & 1) and ((b >> (N + i)) & 1) for i in range(N))
        for (i, j, amp) in bonds:
            for sigma in range(2):
                for (p, q) in ((i, j), (j, i)):
                    mp, mq = sigma * N + p, sigma * N + q
                    b1, s1 = _apply_annihilate(b, mq)
                    if b1 is None:
                        continue
                    b2, s2 = _apply_create(b1, mp)
                    if b2 is None:
                        continue
                    H[key[b2], a] += -amp * s1 * s2
    return H
