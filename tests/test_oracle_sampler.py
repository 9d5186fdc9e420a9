"""The site-exchange proposal of the oracle (the restatement the GPU sampler is replayed
against): symmetric, particle-number conserving, and, with Metropolis acceptance, in detailed
balance with |psi|^2 on a small lattice (exact enumeration of the proposal's transition
matrix)."""

import itertools

import numpy as np

from oracle import lattice as olat
from oracle import sampler as osam


def _apply(s, hops):
    t = s.copy()
    for m_from, m_to in hops:
        t[m_from] = -1
        t[m_to] = 1
    return t


def _proposal_matrix(configs, Lx, Ly, n_dirs):
    """P[a, b]: probability that the exchange proposal from configs[a] proposes configs[b]
    (null moves on the diagonal), by enumerating the (site, direction) draws."""
    N = Lx * Ly
    index = {c.tobytes(): k for k, c in enumerate(configs)}
    P = np.zeros((len(configs), len(configs)))
    for a, s in enumerate(configs):
        for site, d in itertools.product(range(N), range(n_dirs)):
            # draws that select this site and direction exactly
            r0 = np.array([((site << 32) + N - 1) // N], np.uint64)
            r1 = np.array([((d << 32) + n_dirs - 1) // n_dirs], np.uint64)
            moves, ok = osam.propose_exchange(s[None], r0, r1, Lx, Ly, n_dirs)
            b = index[_apply(s, moves[0]).tobytes()] if ok[0] else a
            P[a, b] += 1.0 / (N * n_dirs)
    return P


def test_exchange_proposal_symmetric_and_balanced():
    Lx, Ly, nu, nd = 3, 3, 2, 2
    N = Lx * Ly
    configs = []
    for up in itertools.combinations(range(N), nu):
        for dn in itertools.combinations(range(N), nd):
            s = -np.ones(2 * N, np.int8)
            s[list(up)] = 1
            s[[N + i for i in dn]] = 1
            configs.append(s)
    configs = np.array(configs)
    for n_dirs in (4, 8):
        P = _proposal_matrix(configs, Lx, Ly, n_dirs)
        assert np.allclose(P.sum(1), 1.0)
        off = P - np.diag(np.diag(P))
        assert np.allclose(off, off.T)  # symmetric proposal
        # Metropolis with a random |psi|^2: detailed balance pi_a T_ab = pi_b T_ba
        pi = np.random.default_rng(n_dirs).random(len(configs)) + 0.1
        T = off * np.minimum(1.0, pi[None, :] / pi[:, None])
        flow = pi[:, None] * T
        assert np.allclose(flow, flow.T)
    # exchanges move at most one electron of each spin and conserve both particle numbers
    s = olat.random_configs(np.random.default_rng(1), 64, N, nu, nd)
    r = osam.draws(9, 3, np.arange(64))
    moves, ok = osam.propose_exchange(s, r[0], r[1], Lx, Ly, 8)
    for b in range(64):
        t = _apply(s[b], moves[b])
        assert (t[:N] > 0).sum() == nu and (t[N:] > 0).sum() == nd
        assert len(moves[b]) <= 2 and ok[b] == (len(moves[b]) > 0)
