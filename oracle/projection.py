"""Symmetry projection onto the trivial representation of Flip(0) @ Flip(1) @ SpinInverse()
(``code/states.py:274-279``), FP64 oracle.

With |s> = c+_{m1} ... c+_{mk} |0>, m1 < ... < mk, a mode permutation g acts as
U_g |s> = eta_g(s) |g s>, eta_g(s) the parity of the permutation that sorts
(g(m1), ..., g(mk)).  Every element is an involution, so

    psi_P(s) = (1/|G|) sum_g eta_g(s) psi(g s).

The 1/|G| normalisation and the sign convention of SpinInverse are quantax-internal and not
executable here (parity unpinned); they change log|psi_P| by a constant and leave local
energies and Metropolis ratios unchanged.
"""

from __future__ import annotations

import numpy as np

from . import backflow, lattice


def image_configs(s: np.ndarray, maps: np.ndarray) -> np.ndarray:
    """(B, 2N), (G, 2N) -> (B, G, 2N) with s_g[g(m)] = s[m]."""
    B, M = s.shape
    G = maps.shape[0]
    out = np.empty((B, G, M), dtype=s.dtype)
    for g in range(G):
        out[:, g, maps[g]] = s
    return out


def image_signs(s: np.ndarray, maps: np.ndarray) -> np.ndarray:
    """(B, G) fermionic reordering signs eta_g(s)."""
    B = s.shape[0]
    G = maps.shape[0]
    idx = backflow.fermion_idx(s)
    out = np.empty((B, G))
    n = idx.shape[1]
    upper = np.triu(np.ones((n, n), bool), 1)[None]
    for g in range(G):
        img = maps[g][idx]  # (B, n)
        inv = ((img[:, :, None] > img[:, None, :]) & upper).sum((1, 2))
        out[:, g] = np.where(inv % 2 == 0, 1.0, -1.0)
    return out


def signed_logsumexp(sign: np.ndarray, logabs: np.ndarray, axis: int = -1):
    """(sign, log|.|) of sum_i sign_i exp(logabs_i) along ``axis``."""
    m = np.max(np.where(sign != 0, logabs, -np.inf), axis=axis, keepdims=True)
    m = np.where(np.isfinite(m), m, 0.0)
    tot = np.sum(sign * np.exp(logabs - m), axis=axis)
    m = np.squeeze(m, axis)
    with np.errstate(divide="ignore"):
        return np.sign(tot), np.log(np.abs(tot)) + m


def projected_amplitude(s: np.ndarray, params: dict, symm: bool = True):
    """(sign, logabs) of psi_P(s) (or of psi(s) when ``symm`` is False)."""
    s = np.asarray(s)
    if not symm:
        return backflow.amplitude(s, params)
    Lx, Ly = params["Lx"], params["Ly"]
    maps = lattice.symmetry_mode_maps(Lx, Ly)
    G = maps.shape[0]
    imgs = image_configs(s, maps)  # (B, G, 2N)
    eta = image_signs(s, maps)
    sg, la = backflow.amplitude(imgs.reshape(-1, s.shape[1]), params)
    sg = sg.reshape(-1, G) * eta
    la = la.reshape(-1, G)
    sgn, lab = signed_logsumexp(sg, la, axis=1)
    return sgn, lab - np.log(G)
