"""Lattice tables of the periodic Lx x Ly Hubbard lattice (oracle, FP64).

Site index ``i = x * Ly + y``; mode index ``m = sigma * N + i`` with sigma = 0 (up), 1 (down)
(``README.md`` conventions of the reference; ``code/backflow/models.py:31-32``).
"""

from __future__ import annotations

import numpy as np

# Hop directions: 4 nearest neighbours (amplitude t) then 4 next-nearest (amplitude t').
# Direction order is the enumeration order of connected configurations everywhere.
HOP_DIRS = np.array(
    [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (1, -1), (-1, 1), (-1, -1)], dtype=np.int64
)


def site_xy(Lx: int, Ly: int):
    """(x, y) of every site in row-major order."""
    return np.divmod(np.arange(Lx * Ly), Ly)


def displacement_tables(Lx: int, Ly: int):
    """(disp (N, N), neg (N,), dist (N,)) as in ``code/backflow/pf_kernel.py:83-96``.

    ``disp[i, j]`` is the displacement index r of ``i - j`` taken periodically,
    ``neg[r]`` the index of ``-r`` and ``dist[r]`` the minimum-image length of r (FP64).
    """
    x, y = site_xy(Lx, Ly)
    disp = ((x[:, None] - x[None, :]) % Lx) * Ly + (y[:, None] - y[None, :]) % Ly
    neg = ((-x) % Lx) * Ly + (-y) % Ly
    mx = np.minimum(x, Lx - x)
    my = np.minimum(y, Ly - y)
    dist = np.sqrt((mx * mx + my * my).astype(np.float64))
    return disp.astype(np.int64), neg.astype(np.int64), dist


def neighbour_table(Lx: int, Ly: int) -> np.ndarray:
    """(N, 8) site reached from each site along each of ``HOP_DIRS``."""
    x, y = site_xy(Lx, Ly)
    nx = (x[:, None] + HOP_DIRS[None, :, 0]) % Lx
    ny = (y[:, None] + HOP_DIRS[None, :, 1]) % Ly
    return nx * Ly + ny


def hop_amplitudes(t: float, tp: float, n_dirs: int = 8) -> np.ndarray:
    """t_d for each direction: t for the 4 nearest, t' for the 4 next-nearest."""
    amp = np.array([t] * 4 + [tp] * 4, dtype=np.float64)
    return amp[:n_dirs]


def symmetry_mode_maps(Lx: int, Ly: int) -> np.ndarray:
    """(8, 2N) mode permutations of Flip(axis=0)^a Flip(axis=1)^b SpinInverse()^c.

    Element g = a + 2 b + 4 c.  Flip(axis=0) maps x -> (-x) mod Lx, Flip(axis=1) maps
    y -> (-y) mod Ly, SpinInverse swaps the up and down modes of a site.  All elements are
    involutions and commute.  (The quantax group is built at ``code/states.py:274-279``;
    the choice of reflection centre is immaterial for translation-invariant networks.)
    """
    N = Lx * Ly
    x, y = site_xy(Lx, Ly)
    maps = np.empty((8, 2 * N), dtype=np.int64)
    for g in range(8):
        fx, fy, si = g & 1, (g >> 1) & 1, (g >> 2) & 1
        xs = (-x) % Lx if fx else x
        ys = (-y) % Ly if fy else y
        site = xs * Ly + ys
        for sigma in range(2):
            maps[g, sigma * N : (sigma + 1) * N] = (sigma ^ si) * N + site
    return maps


def random_configs(rng: np.random.Generator, batch: int, N: int, n_up: int, n_dn: int):
    """(batch, 2N) int8 +-1 configurations with exactly n_up / n_dn occupied sites,
    uniform without replacement per spin half."""
    s = -np.ones((batch, 2 * N), dtype=np.int8)
    for b in range(batch):
        s[b, rng.choice(N, n_up, replace=False)] = 1
        s[b, N + rng.choice(N, n_dn, replace=False)] = 1
    return s
