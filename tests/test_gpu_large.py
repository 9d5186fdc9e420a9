"""GPU tests of the large-lattice path: 24x24 (n = 504) and 32x32 (n = 896), where the Pfaffian
triangle lives in global memory (1024 threads, one row each) and, at 32x32, the CNN's activation
planes too.

The all-FP64 path (cond_tau = 1) must match the FP64 oracle to 1e-8; the default mixed path keeps
signs exact and log|psi| within 1e-3 (FP32 round-off of a 504- or 896-dimensional elimination).
The ragged local energy is checked against the sum over its connected configurations built from
the hop list, and the learned-proposal sampler by a replay of its parts.
"""

import numpy as np
import pytest
import torch

import neuralhubbard_b200 as nh
from oracle import lattice as olat
from oracle import projection as oproj
from oracle import sampler as osam

pytestmark = pytest.mark.gpu
DEV = "cuda"


def host_params(params, L):
    return dict(conv_w=[np.asarray(w, np.float64) for w in params["conv_w"]],
                conv_b=[np.asarray(b, np.float64) for b in params["conv_b"]],
                W=np.asarray(params["W"], np.float64), theta=float(params["theta"]), Lx=L, Ly=L)


@pytest.mark.parametrize("L,symm", [(24, True), (32, False)])
def test_amplitude_large_lattice(L, symm):
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=32, std=0.02, seed=21)
    s = olat.random_configs(np.random.default_rng(L), 2, N, ne, ne)
    s0, l0 = oproj.projected_amplitude(s, host_params(params, L), symm=symm)
    m64 = nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=1.0)
    sg, la = nh.Variational(m64, symm=symm)(s).numpy()
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < 1e-8, np.max(np.abs(la - l0))
    m = nh.PfaffianBackflow(L, L, ne, ne, params=params)
    psi = nh.Variational(m, symm=symm)(s)
    sg, la = psi.numpy()
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < 1e-3, np.max(np.abs(la - l0))


def test_local_energy_large_lattice():
    """24x24: E_loc from the ragged pipeline equals U docc + sum_s' h(s, s') psi(s') / psi(s)
    evaluated from the explicit connected configurations of the hop list."""
    L = 24
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=32, std=0.02, seed=22)
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params)
    state = nh.Variational(model, symm=False)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    s = torch.from_numpy(olat.random_configs(np.random.default_rng(23), 3, N, ne, ne)).to(DEV)
    psi = state(s)
    e = H.Oloc(state, nh.Samples(s, psi), chunk_configs=1024).cpu().numpy()
    counts, offsets, rec, hval = H.hop_list(s, L, L)
    owner = torch.repeat_interleave(torch.arange(3, device=DEV), counts.long())
    conn = s[owner].clone()
    rows = torch.arange(conn.shape[0], device=DEV)
    conn[rows, rec[:, 0].long()] = -1
    conn[rows, rec[:, 1].long()] = 1
    phi = state(conn)
    ratio = (phi.sign.double() * psi.sign.double()[owner]
             * torch.exp(phi.logabs - psi.logabs[owner]))
    kin = torch.zeros(3, dtype=torch.float64, device=DEV).index_add_(0, owner, hval * ratio)
    docc = ((s[:, :N] > 0) & (s[:, N:] > 0)).sum(1).double()
    e0 = (kin + 8.0 * docc).cpu().numpy()
    assert np.max(np.abs(e - e0) / np.abs(e0)) < 1e-9


def test_learned_metropolis_32x32_replay():
    """32x32 (n = 896): the learned-proposal sampler equals a replay from its proposal draws
    and the amplitudes of the proposed configurations."""
    L = 32
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=32, std=0.02, seed=24)
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params)
    state = nh.Variational(model, symm=False)
    q = nh.HopProposal(L, L, 8, seed=25, std=0.2)
    s0 = olat.random_configs(np.random.default_rng(26), 6, N, ne, ne)
    smp = nh.LearnedHop(state, 6, q, initial_spins=s0, seed=99)
    s = torch.from_numpy(s0).to(DEV)
    logabs = state(s).logabs.clone()
    steps = 3
    for t in range(steps):
        fr, to, ok, lqr = q.sample(s, 99, t)
        idx = torch.nonzero(ok).flatten()
        sp = s[idx].clone()
        r = torch.arange(len(idx), device=DEV)
        sp[r, fr[idx].long()] = -1
        sp[r, to[idx].long()] = 1
        phi = state(sp)
        u = osam.draws(99, t, idx.cpu().numpy())[2]
        lr2 = 2.0 * (phi.logabs - logabs[idx]).cpu().numpy() + lqr[idx].double().cpu().numpy()
        a = torch.from_numpy(osam.metropolis_accept(lr2, u) & (phi.sign.cpu().numpy() != 0))
        a = a.to(DEV)
        s[idx[a]] = sp[a]
        logabs[idx[a]] = phi.logabs[a]
    smp.run(steps)
    assert torch.equal(smp.spins, s)
    assert torch.equal(smp.psi.logabs, logabs)


@pytest.mark.parametrize("symm", [False, True])
def test_local_energy_24x24_against_fp64_path(symm):
    """24x24 E_loc of the default mixed-precision path against the all-FP64 path (cond_tau = 1:
    FP64 network, gather and Pfaffian for every image, itself equal to the FP64 oracle to 1e-8 in
    test_amplitude_large_lattice), unprojected and projected: the batch mean within 1e-5 t per
    site, every sample within 1e-4 relative."""
    L = 24
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=32, std=0.02, seed=27)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    s = torch.from_numpy(olat.random_configs(np.random.default_rng(28), 4, N, ne, ne)).to(DEV)
    out = []
    for tau in (nh.backflow.DEFAULT_COND_TAU, 1.0):
        state = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=tau),
                               symm=symm)
        out.append(H.Oloc(state, nh.Samples(s, state(s)), chunk_configs=2048).cpu().numpy())
    e, e64 = out
    assert abs(e.mean() - e64.mean()) / N < 1e-5, (e.mean(), e64.mean())
    assert np.max(np.abs(e - e64) / np.maximum(1.0, np.abs(e64))) < 1e-4, (e, e64)
