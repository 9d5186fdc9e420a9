"""GPU tests of the learned hop proposal against the FP64 oracle.

Forward logits, loss and gradient, the Adam step and the proposal draw (move and Hastings
log-ratio) are compared with ``oracle.proposal`` evaluated on the same BF16-rounded weights;
the fused learned-proposal Metropolis step is replayed bit for bit from its parts; and on a 3x3
lattice the chains' histogram is compared with the exact |psi|^2.
"""

import numpy as np
import pytest
import torch

import neuralhubbard_b200 as nh
from oracle import lattice as olat
from oracle import proposal as oprop
from oracle import sampler as osam

pytestmark = pytest.mark.gpu
DEV = "cuda"


def make_proposal(L, std=0.3, seed=0, n_dirs=8):
    th = oprop.init_params(seed, std)
    q = nh.HopProposal(L, L, n_dirs=n_dirs, params=th, device=DEV)
    return q, oprop.round_bf16(th).astype(np.float64)


@pytest.mark.parametrize("L,ne", [(6, 10), (16, 112)])
def test_logits_vs_oracle(L, ne):
    q, th = make_proposal(L, seed=1)
    s = olat.random_configs(np.random.default_rng(L), 4, L * L, ne, ne)
    z = q.logits(s).cpu().numpy()
    z0 = oprop.logits(s, th, L, L)
    assert np.max(np.abs(z - z0)) < 1e-4 * max(1.0, np.abs(z0).max())


@pytest.mark.parametrize("L,ne,n_dirs", [(6, 10, 8), (8, 28, 4), (24, 252, 8), (32, 448, 8)])
def test_loss_and_gradient_vs_oracle(L, ne, n_dirs):
    """24x24 and 32x32 exceed shared memory: the backward keeps its activation planes in
    per-CTA global slices of the workspace."""
    q, th = make_proposal(L, seed=2, n_dirs=n_dirs)
    rng = np.random.default_rng(5)
    s = olat.random_configs(rng, 12, L * L, ne, ne)
    lq = oprop.log_q(s, th, L, L, n_dirs)
    mv = np.array([rng.choice(np.flatnonzero(np.isfinite(r))) for r in lq], np.int32)
    w = rng.random(12).astype(np.float32)
    loss, grad = q.loss_grad(torch.from_numpy(s), torch.from_numpy(mv), torch.from_numpy(w))
    l0, g0 = oprop.loss_and_grad(s, mv, w.astype(np.float64), th, L, L, n_dirs)
    assert abs(loss.item() - l0) < 1e-5 * max(1.0, abs(l0))
    g = grad.cpu().numpy()
    assert np.max(np.abs(g - g0)) < 1e-4 * np.abs(g0).max(), np.max(np.abs(g - g0))


def test_gradient_is_deterministic_and_skips_invalid_moves():
    L, ne = 6, 10
    q, _ = make_proposal(L, seed=3)
    rng = np.random.default_rng(6)
    s = torch.from_numpy(olat.random_configs(rng, 300, L * L, ne, ne))
    mv = torch.from_numpy(rng.integers(0, 16 * L * L, 300).astype(np.int32))
    w = torch.ones(300)
    l1, g1 = q.loss_grad(s, mv, w)
    l2, g2 = q.loss_grad(s, mv, w)
    assert torch.equal(g1, g2) and torch.equal(l1, l2)
    # records whose move is invalid carry no gradient: same result with their weight zeroed
    ok = nh.proposal.valid_moves(s.to(DEV), L, L)[torch.arange(300), mv.long().to(DEV)].cpu()
    l3, g3 = q.loss_grad(s, mv, torch.where(ok, w, torch.zeros_like(w)))
    assert torch.allclose(g1, g3, atol=1e-7) and torch.allclose(l1, l3, atol=1e-7)


def test_adam_step_vs_oracle():
    L = 6
    q, _ = make_proposal(L, seed=4)
    th0 = q.numpy().astype(np.float64)
    rng = np.random.default_rng(7)
    grads = [rng.normal(size=oprop.PARAM_COUNT).astype(np.float32) for _ in range(3)]
    m = np.zeros_like(th0)
    v = np.zeros_like(th0)
    th = th0
    for t, g in enumerate(grads, 1):
        q.adam_step(torch.from_numpy(g).to(DEV), lr=1e-2)
        th, m, v = oprop.adam_step(th, m, v, g.astype(np.float64), t, 1e-2)
    assert np.max(np.abs(q.numpy() - th)) < 1e-5
    w = q.weights.float().cpu().numpy()
    assert np.array_equal(w, oprop.round_bf16(q.numpy()))


@pytest.mark.parametrize("L,ne,n_dirs", [(6, 10, 8), (16, 112, 8), (8, 28, 4)])
def test_proposal_draw_vs_oracle(L, ne, n_dirs):
    """The drawn move lies where the oracle's CDF puts the Philox uniform (up to FP32 rounding of
    the CDF) and log q(reverse | s') - log q(move | s) matches the oracle."""
    q, th = make_proposal(L, seed=5, n_dirs=n_dirs)
    B = 64
    s = olat.random_configs(np.random.default_rng(8), B, L * L, ne, ne)
    seed, step = 99, 7
    fr, to, ok, lqr = (x.cpu().numpy() for x in q.sample(s, seed, step))
    assert ok.all()
    r = osam.draws(seed, step, np.arange(B))
    u = osam.uniform_from_u32(r[0])
    lq = oprop.log_q(s, th, L, L, n_dirs)
    N = L * L
    nbr = olat.neighbour_table(L, L)
    for b in range(B):
        p = np.exp(lq[b])
        cdf = np.cumsum(p)
        sg, i = divmod(int(fr[b]), N)
        j = int(to[b]) - sg * N
        d = int(np.flatnonzero(nbr[i] == j)[0])
        m = (sg * 8 + d) * N + i
        assert np.isfinite(lq[b, m])
        lo = cdf[m] - p[m]
        assert lo - 1e-5 <= u[b] <= cdf[m] + 1e-5, (b, lo, u[b], cdf[m])
        sp, _, _ = oprop.apply_move(s[b : b + 1], [m], L, L)
        rm = oprop.reverse_move([m], L, L)[0]
        lr0 = oprop.log_q(sp, th, L, L, n_dirs)[0, rm] - lq[b, m]
        assert abs(lqr[b] - lr0) < 1e-4, (b, lqr[b], lr0)


def test_learned_metropolis_replays_from_parts():
    """The fused learned-proposal steps equal a replay from the proposal draws, the amplitudes of
    the proposed configurations and the Hastings rule log u < 2 dlog|psi| + log q ratio."""
    L = 6
    N = L * L
    params = nh.init_params(L, L, channels=32, std=0.3, seed=9)
    model = nh.PfaffianBackflow(L, L, 10, 10, params=params)
    state = nh.Variational(model, symm=True)
    q, _ = make_proposal(L, seed=6, std=0.2)  # logits of O(1) spread: moves get accepted
    s0 = olat.random_configs(np.random.default_rng(10), 40, N, 10, 10)
    smp = nh.LearnedHop(state, 40, q, initial_spins=s0, seed=321)
    s = torch.from_numpy(s0).to(DEV)
    psi = state(s)
    sign, logabs = psi.sign.clone(), psi.logabs.clone()
    acc = torch.zeros(40, dtype=torch.int32, device=DEV)
    steps = 20
    for t in range(steps):
        fr, to, ok, lqr = q.sample(s, 321, t)
        idx = torch.nonzero(ok).flatten()
        sp = s[idx].clone()
        rows = torch.arange(len(idx), device=DEV)
        sp[rows, fr[idx].long()] = -1
        sp[rows, to[idx].long()] = 1
        phi = state(sp)
        r = osam.draws(321, t, idx.cpu().numpy())
        lr2 = 2.0 * (phi.logabs - logabs[idx]).cpu().numpy() + lqr[idx].double().cpu().numpy()
        a = osam.metropolis_accept(lr2, r[2]) & (phi.sign.cpu().numpy() != 0)
        sel = idx[torch.from_numpy(a).to(DEV)]
        keep = torch.from_numpy(a).to(DEV)
        s[sel] = sp[keep]
        sign[sel] = phi.sign[keep]
        logabs[sel] = phi.logabs[keep]
        acc[sel] += 1
    smp.run(steps)
    assert torch.equal(smp.spins, s)
    assert torch.equal(smp.psi.logabs, logabs) and torch.equal(smp.psi.sign, sign)
    assert torch.equal(smp.accepted, acc)
    assert acc.sum().item() > 0.05 * 40 * steps


def _transition(basis, lq, logp, Lx, Ly, hastings):
    """Exact Metropolis transition matrix of the learned proposal on a 1 + 1 electron basis."""
    N = Lx * Ly
    T = np.zeros((len(basis), len(basis)))
    for a in range(len(basis)):
        for m in np.flatnonzero(np.isfinite(lq[a])):
            sp, _, _ = oprop.apply_move(basis[a : a + 1], [m], Lx, Ly)
            b = int(np.argmax(sp[0, :N])) * N + int(np.argmax(sp[0, N:]))
            lr = logp[b] - logp[a]
            if hastings:
                lr += lq[b, oprop.reverse_move([m], Lx, Ly)[0]] - lq[a, m]
            T[a, b] += np.exp(lq[a, m]) * min(1.0, np.exp(lr))
        T[a, a] += 1.0 - T[a].sum()
    return T


def test_learned_sampler_samples_psi_squared_3x4():
    """Learned-proposal chains on the 144 states of a 3x4 lattice with 1 + 1 electrons.  The
    GPU histogram over steps (burn, burn + steps] is compared with its exact expectation, the
    uniform start propagated by the oracle's transition matrix: only sampling noise separates
    them.  The same expectation without the Hastings factor (a mistake planted in the oracle)
    is far from the histogram, and the corrected matrix leaves |psi|^2 invariant."""
    Lx, Ly = 3, 4
    N = Lx * Ly
    params = nh.init_params(Lx, Ly, channels=32, std=0.3, seed=11)
    model = nh.PfaffianBackflow(Lx, Ly, 1, 1, params=params)
    state = nh.Variational(model, symm=False)
    basis = -np.ones((N * N, 2 * N), np.int8)
    for up in range(N):
        for dn in range(N):
            basis[up * N + dn, up] = 1
            basis[up * N + dn, N + dn] = 1
    la = state(basis).logabs.cpu().numpy()
    logp = 2 * (la - la.max())
    p = np.exp(logp) / np.exp(logp).sum()
    th = oprop.init_params(12, 0.25)
    q = nh.HopProposal(Lx, Ly, 8, params=th, device=DEV)
    th = oprop.round_bf16(th).astype(np.float64)
    # 65536 chains: the histogram's noise (TV ~ 0.008 at tau_int ~ 20) sits well under the bound
    B, burn, steps = 65536, 40, 240
    smp = nh.LearnedHop(state, B, q, seed=2024)
    smp.run(burn)
    hist = torch.zeros(N * N, dtype=torch.float64, device=DEV)
    for _ in range(steps):
        smp.run(1)
        k = smp.spins[:, :N].argmax(1) * N + smp.spins[:, N:].argmax(1)
        hist += torch.bincount(k, minlength=N * N).double()
    emp = (hist / hist.sum()).cpu().numpy()
    assert smp.acceptance > 0.05
    lq = oprop.log_q(basis, th, Lx, Ly)
    expect = {}
    for hastings in (True, False):
        T = _transition(basis, lq, logp, Lx, Ly, hastings)
        mu = np.full(N * N, 1.0 / (N * N)) @ np.linalg.matrix_power(T, burn)
        acc = np.zeros(N * N)
        for _ in range(steps):
            mu = mu @ T
            acc += mu
        expect[hastings] = acc / steps
        if hastings:
            assert np.allclose(p @ T, p, atol=1e-12)
    tv = 0.5 * np.abs(emp - expect[True]).sum()
    tv_wrong = 0.5 * np.abs(emp - expect[False]).sum()
    assert tv < 0.02, tv
    assert tv_wrong > 5 * tv, (tv, tv_wrong)


def test_training_learns_a_local_target():
    """The training kernels learn: on records whose weight is 1 for hops of down-spin electrons
    in direction +x and 0.02 otherwise, 300 Adam steps move the network's expected weight
    E_q[w] on held-out configurations from the untrained ~0.1 to above 0.5."""
    L = 6
    N = L * L
    rng = np.random.default_rng(40)
    q = nh.HopProposal(L, L, 8, params=np.zeros(oprop.PARAM_COUNT, np.float32), device=DEV)

    def records(n, seed):
        s = torch.from_numpy(olat.random_configs(np.random.default_rng(seed), n, N, 15, 15)).to(DEV)
        ok = nh.proposal.valid_moves(s, L, L)
        g = torch.Generator(device=DEV)
        g.manual_seed(seed)
        m = torch.rand(ok.shape, generator=g, device=DEV).masked_fill_(~ok, -1.0).argmax(1)
        c = m // N
        w = torch.where(c == 8 + 0, 1.0, 0.02).float()  # spin down (8..15), direction 0 (+x)
        return s, m.to(torch.int32), w, ok

    def expected_weight(s, ok):
        z = q.logits(s).reshape(s.shape[0], -1)
        z = z.masked_fill(~ok, -float("inf"))
        p = torch.softmax(z, 1)
        wmap = torch.full((16, N), 0.02, device=DEV)
        wmap[8] = 1.0
        return float((p * wmap.reshape(1, -1)).sum(1).mean().item())

    train = records(8192, 41)
    s_test, _, _, ok_test = records(512, 42)
    before = expected_weight(s_test, ok_test)
    losses = q.train(train[:3], 300, batch=512, lr=1e-2, seed=int(rng.integers(1 << 30)))
    after = expected_weight(s_test, ok_test)
    assert before < 0.2, before
    assert after > 0.5, (before, after)
    assert np.mean(losses[-20:]) < np.mean(losses[:20])


def test_learned_sampler_against_plain_8x8():
    """A/B on the 8x8 lattice (projected amplitudes): the proposal trained on plain-chain records
    raises the acceptance per step over the plain uniform hop (it never proposes a null move),
    and both samplers give the same energy per site within 3 sigma (the Hastings correction
    keeps |psi|^2)."""
    L = 8
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=32, std=0.3, seed=0)
    state = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params), symm=True)
    B = 1024
    plain = nh.ParticleHop(state, B, n_neighbor=(1, 2), seed=1)
    plain.run(1500)  # equilibrate: both samplers must start from |psi|^2 for the energy A/B
    snaps = []
    for _ in range(16):
        plain.run(1)
        snaps.append(plain.spins.clone())
    start = plain.spins.clone()
    rec = nh.training_records(state, torch.cat(snaps), seed=2, weight="barker")
    q = nh.HopProposal(L, L, 8, seed=3, std=0.05)
    q.train(rec, 300, batch=512, lr=3e-3)
    learned = nh.LearnedHop(state, B, q, initial_spins=start, seed=4)
    a_p0, a_l0 = plain.accepted.sum().item(), learned.accepted.sum().item()
    plain.run(600)
    learned.run(600)
    acc_p = (plain.accepted.sum().item() - a_p0) / (B * 600)
    acc_l = (learned.accepted.sum().item() - a_l0) / (B * 600)
    assert acc_l > 1.2 * acc_p, (acc_l, acc_p)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    e = []
    for smp in (plain, learned):
        el = H.Oloc(state, nh.Samples(smp.spins[:512].contiguous(), smp.psi[:512])).cpu().numpy()
        el = el / N
        e.append((el.mean(), el.std(ddof=1) / np.sqrt(len(el))))
    (m0, s0), (m1, s1) = e
    assert abs(m0 - m1) < 3 * np.hypot(s0, s1), e
