"""Metropolis hop sampler, counter-based random numbers and chain statistics (oracle).

Random numbers: Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random
numbers: as easy as 1, 2, 3", SC'11), restated here so that the CUDA sampler's draws can be
reproduced bit for bit.  Counter = (step_lo, chain, stream, step_hi), key = (seed_lo, seed_hi).

Plain uniform-hop proposal (the ParticleHop analogue of ``code/states.py:397-408``): pick an
occupied mode uniformly (rank e among the k occupied modes, ascending), pick one of the
``n_dirs`` hop directions uniformly; if the target mode of the same spin is empty the move
is proposed, otherwise the step is a null move.  The proposal is symmetric, so a move is
accepted when u < |psi(s') / psi(s)|^2.

Site exchange (the SiteExchange analogue of ``code/states.py:397-408``): pick a site i
uniformly (word 0 of the draw) and one of the ``n_dirs`` directions (word 1); the site j it
reaches swaps its occupation (up and down) with i.  Equal occupations are a null move; an up and
a down electron may move in one step.  The reverse move (j and the opposite direction) has the
same probability, so the proposal is symmetric.  The mixed sampler (``MixSampler`` of a
ParticleHop and a SiteExchange sampler) runs hops on chains b < first_exchange and exchanges on
the others.
"""

from __future__ import annotations

import numpy as np

from . import lattice

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32(counter, key, rounds: int = 10):
    """Vectorised Philox4x32: counter (4, ...) uint32-valued ints, key (2,) -> (4, ...)."""
    c = [np.asarray(ci, dtype=np.uint64) & MASK for ci in counter]
    k0 = np.uint64(key[0] & MASK)
    k1 = np.uint64(key[1] & MASK)
    for _ in range(rounds):
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & np.uint64(MASK)
        hi1, lo1 = p1 >> np.uint64(32), p1 & np.uint64(MASK)
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(W0)) & np.uint64(MASK)
        k1 = (k1 + np.uint64(W1)) & np.uint64(MASK)
    return [ci.astype(np.uint32) for ci in c]


def uniform_from_u32(x):
    """u = (x >> 8) * 2^-24 in [0, 1), exact in FP32 and FP64."""
    return (np.asarray(x, np.uint32) >> np.uint32(8)).astype(np.float64) * (2.0 ** -24)


def draws(seed: int, step: int, chains: np.ndarray, stream: int = 0):
    """The 4 uint32 draws of each chain at ``step``."""
    chains = np.asarray(chains, np.uint64)
    z = np.zeros_like(chains)
    lo, hi = step & MASK, (step >> 32) & MASK
    return philox4x32([z + lo, chains, z + stream, z + hi], (seed & MASK, (seed >> 32) & MASK))


def propose_uniform(s: np.ndarray, r0, r1, Lx: int, Ly: int, n_dirs: int = 8):
    """Plain proposal for each chain: (from_mode, to_mode, valid)."""
    N = Lx * Ly
    nbr = lattice.neighbour_table(Lx, Ly)
    B = s.shape[0]
    fr = np.zeros(B, np.int64)
    to = np.zeros(B, np.int64)
    ok = np.zeros(B, bool)
    for b in range(B):
        occ = np.flatnonzero(s[b] > 0)
        k = len(occ)
        e = (int(r0[b]) * k) >> 32
        dr = (int(r1[b]) * n_dirs) >> 32
        m = int(occ[e])
        sigma, i = divmod(m, N)
        mj = sigma * N + int(nbr[i, dr])
        fr[b], to[b] = m, mj
        ok[b] = s[b, mj] < 0
    return fr, to, ok


def propose_exchange(s: np.ndarray, r0, r1, Lx: int, Ly: int, n_dirs: int = 8):
    """Site-exchange proposal for each chain: a list of (from_mode, to_mode) hops (0, 1 or 2)
    and valid (at least one hop)."""
    N = Lx * Ly
    nbr = lattice.neighbour_table(Lx, Ly)
    moves, ok = [], np.zeros(s.shape[0], bool)
    for b in range(s.shape[0]):
        i = (int(r0[b]) * N) >> 32
        j = int(nbr[i, (int(r1[b]) * n_dirs) >> 32])
        hops = []
        for sigma in range(2):
            oi, oj = s[b, sigma * N + i] > 0, s[b, sigma * N + j] > 0
            if oi != oj:
                src, dst = (i, j) if oi else (j, i)
                hops.append((sigma * N + src, sigma * N + dst))
        moves.append(hops)
        ok[b] = len(hops) > 0
    return moves, ok


def metropolis_accept(log_ratio2: np.ndarray, r2) -> np.ndarray:
    """Accept when u < exp(log_ratio2), compared as log(u) < log_ratio2 (FP64)."""
    u = uniform_from_u32(r2)
    with np.errstate(divide="ignore"):
        return np.log(u) < log_ratio2


def metropolis_steps(s, psi, amp_fn, Lx, Ly, seed, step0, nsteps, n_dirs=8,
                     first_exchange=None):
    """Run ``nsteps`` Metropolis steps on every chain: hops on chains b < first_exchange (all
    chains when None), site exchanges on the others.  Returns (s, sign, logabs, accepted count
    per chain)."""
    s = np.array(s, copy=True)
    sign, logabs = (np.array(a, dtype=np.float64, copy=True) for a in psi)
    B = s.shape[0]
    fx = B if first_exchange is None else int(first_exchange)
    chains = np.arange(B)
    acc = np.zeros(B, np.int64)
    for t in range(step0, step0 + nsteps):
        r = draws(seed, t, chains)
        fr, to, ok = propose_uniform(s, r[0], r[1], Lx, Ly, n_dirs)
        moves = [[(int(fr[b]), int(to[b]))] for b in range(B)]
        if fx < B:
            mx, okx = propose_exchange(s[fx:], r[0][fx:], r[1][fx:], Lx, Ly, n_dirs)
            moves[fx:] = mx
            ok[fx:] = okx
        idx = np.flatnonzero(ok)
        if len(idx) == 0:
            continue
        sp = s[idx].copy()
        for k, b in enumerate(idx):
            for m_from, m_to in moves[b]:
                sp[k, m_from] = -1
                sp[k, m_to] = 1
        sg2, la2 = amp_fn(sp)
        a = metropolis_accept(2.0 * (la2 - logabs[idx]), r[2][idx]) & (sg2 != 0)
        sel = idx[a]
        s[sel] = sp[a]
        sign[sel] = sg2[a]
        logabs[sel] = la2[a]
        acc[sel] += 1
    return s, sign, logabs, acc


def tau_int(x: np.ndarray, c: float = 5.0) -> float:
    """Integrated autocorrelation time of a series (T,) or chains (T, B) with Sokal's
    automatic window (smallest W with W >= c tau(W)); tau = 1/2 + sum_{t=1}^W rho(t)."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = x[:, None]
    T = x.shape[0]
    xc = x - x.mean(0, keepdims=True)
    f = np.fft.rfft(xc, n=2 * T, axis=0)
    acf = np.fft.irfft(f * np.conj(f), axis=0)[:T].mean(1)
    if acf[0] <= 0:
        return 0.5
    rho = acf / acf[0]
    tau = 0.5
    for W in range(1, T):
        tau += rho[W]
        if W >= c * tau:
            break
    return float(max(tau, 0.5))


def jackknife_mean(x: np.ndarray, blocks=(1, 2, 4, 8), min_blocks: int = 8):
    """Mean and block-jackknife error of a series (``code/measure/assemble.py:48-84``)."""
    x = np.asarray(x, np.float64)
    val = x.mean()
    errs = []
    for b in blocks:
        nb = x.shape[0] // b
        if nb < min_blocks:
            continue
        xb = x[: nb * b].reshape(nb, b).mean(1)
        reps = (xb.sum() - xb) / (nb - 1)
        errs.append(np.sqrt(nb - 1) * reps.std())
    return float(val), float(max(errs)) if errs else float("nan")
