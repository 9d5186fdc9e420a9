"""GPU parity tests: every CUDA entry point against the FP64 oracle on the same inputs.

Bars: configuration bookkeeping, hop enumeration and Pfaffian signs bit-exact; log|psi| within
1e-4 absolute of FP64 on the FP32 path; batch-mean local energy within 1e-5 t per site.
"""

import numpy as np
import pytest
import torch

import neuralhubbard_b200 as nh
from neuralhubbard_b200 import _lib
from oracle import backflow as obf
from oracle import hubbard as ohub
from oracle import lattice as olat
from oracle import pfaffian as opf
from oracle import projection as oproj
from oracle import sampler as osam

pytestmark = pytest.mark.gpu
DEV = "cuda"
LOG_TOL = 1e-4


def host_params(model):
    p = model.host_params
    return dict(conv_w=[np.asarray(w, np.float64) for w in p["conv_w"]],
                conv_b=[np.asarray(b, np.float64) for b in p["conv_b"]],
                W=np.asarray(p["W"], np.float64), theta=float(p["theta"]),
                Lx=model.geom.LX, Ly=model.geom.LY)


def make_model(L, std=0.02, seed=0, channels=32):
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=channels, std=std, seed=seed)
    return nh.PfaffianBackflow(L, L, ne, ne, params=params)


def rand_skew32(rng, n, batch):
    A = rng.normal(size=(batch, n, n)).astype(np.float32)
    return A - np.swapaxes(A, 1, 2)


@pytest.mark.parametrize("n", [2, 4, 56, 100, 224, 236, 248, 256, 400, 1024])
def test_slogpf_random(n):
    """Gaussian antisymmetric matrices (condition ~ n^2): plain FP32, and with the FP64
    recompute of the matrices whose pivot ratio exceeds the default cond_tau (5).  Beyond shared
    memory (FP32 n > 256, FP64 n > 236) the triangles live in the workspace; cond_tau = 1
    recomputes every matrix in FP64."""
    rng = np.random.default_rng(n)
    A = rand_skew32(rng, n, 6 if n <= 400 else 3)
    s0, l0 = opf.slogpf(A.astype(np.float64))
    sg, la, fl = nh.slogpf(torch.from_numpy(A).to(DEV), cond_tau=0.0)
    assert np.array_equal(sg.cpu().numpy(), s0)
    assert np.max(np.abs(la.cpu().numpy() - l0)) < (1e-4 if n <= 100 else 1e-3)
    sg, la, fl = nh.slogpf(torch.from_numpy(A).to(DEV))
    fl = fl.cpu().numpy()
    assert np.array_equal(sg.cpu().numpy(), s0)
    err = np.abs(la.cpu().numpy() - l0)
    refined = (fl & _lib.FLAG_REFINED) != 0
    assert np.array_equal(refined, (fl & _lib.FLAG_GROWTH) != 0)
    assert np.all(err[refined] < 1e-9)
    assert np.max(err) < 1e-4  # the default refinement threshold leaves only well-conditioned
    # matrices in FP32
    if n >= 236:
        sg, la, fl = nh.slogpf(torch.from_numpy(A).to(DEV), cond_tau=1.0)
        assert np.all(fl.cpu().numpy() & _lib.FLAG_REFINED)
        assert np.array_equal(sg.cpu().numpy(), s0)
        assert np.max(np.abs(la.cpu().numpy() - l0)) < 1e-9


def test_slogpf_near_nodal():
    """Near-nodal matrices (one pivot scaled to ~1e-6 of the others, condition ~1e6) are flagged
    and recomputed in FP64; sign mismatches must be 0."""
    rng = np.random.default_rng(77)
    n, B = 224, 16
    Q = np.linalg.qr(rng.normal(size=(B, n, n)))[0]  # orthogonal: condition ~ pivot ratio
    blocks = np.zeros((B, n, n))
    a = rng.uniform(0.5, 2.0, size=(B, n // 2)) * rng.choice([-1, 1], size=(B, n // 2))
    a[:, 7] *= 1e-6
    for k in range(n // 2):
        blocks[:, 2 * k, 2 * k + 1], blocks[:, 2 * k + 1, 2 * k] = a[:, k], -a[:, k]
    A = np.einsum("bji,bjk,bkl->bil", Q, blocks, Q).astype(np.float32)
    A = 0.5 * (A - np.swapaxes(A, 1, 2))
    s0, l0 = opf.slogpf(A.astype(np.float64))
    sg, la, fl = nh.slogpf(torch.from_numpy(A).to(DEV))
    fl = fl.cpu().numpy()
    assert np.all(fl & _lib.FLAG_REFINED)
    assert np.array_equal(sg.cpu().numpy(), s0)
    assert np.max(np.abs(la.cpu().numpy() - l0)) < 1e-6


def test_slogpf_singular_and_deterministic():
    rng = np.random.default_rng(1)
    A = rand_skew32(rng, 56, 4)
    A[1] = 0.0
    A[2, :, 7] = 0.0
    A[2, 7, :] = 0.0
    t = torch.from_numpy(A).to(DEV)
    sg, la, fl = nh.slogpf(t)
    sg, la, fl = sg.cpu().numpy(), la.cpu().numpy(), fl.cpu().numpy()
    assert sg[1] == 0 and la[1] == -np.inf and fl[1] & _lib.FLAG_ZERO_PIVOT
    assert sg[2] == 0 and fl[2] & _lib.FLAG_ZERO_PIVOT
    sg2, la2, _ = nh.slogpf(t)
    assert np.array_equal(sg2.cpu().numpy(), sg) and np.array_equal(la2.cpu().numpy(), la)


def test_wtilde_and_pairing():
    model = make_model(8, std=0.3)
    g = model.geom
    Wt0 = obf.build_wtilde(model.host_params["W"], float(model.theta), 8, 8, np.float32)
    Wt = model.Wt.cpu().numpy()
    assert np.allclose(Wt, Wt0, rtol=1e-6, atol=0)
    Wt64 = obf.build_wtilde(model.host_params["W"].astype(np.float64), float(model.theta), 8, 8)
    assert np.allclose(model.Wt64.cpu().numpy(), Wt64, rtol=1e-13, atol=0)
    rng = np.random.default_rng(3)
    s = olat.random_configs(rng, 5, g.N, g.n_up, g.n_dn)
    y = model.features(torch.from_numpy(s).to(DEV))
    idx = obf.fermion_idx(s)
    Y = np.take_along_axis(y.cpu().numpy().reshape(5, 2 * g.N, g.d), idx[:, :, None], 1)
    F = nh.pairing_occ(torch.from_numpy(Y).to(DEV), torch.from_numpy(idx.astype(np.int32)).to(DEV),
                       model.Wt, g).cpu().numpy()
    assert np.array_equal(F, -np.swapaxes(F, 1, 2))  # exactly antisymmetric
    F0 = obf.pairing_occ(Y.astype(np.float64), idx, Wt.astype(np.float64), 8, 8)
    assert np.allclose(F, F0, rtol=1e-5, atol=1e-6 * np.abs(F0).max())


@pytest.mark.parametrize("L", [8, 16])
def test_cnn_features(L):
    model = make_model(L, std=0.3, seed=L)
    g = model.geom
    s = olat.random_configs(np.random.default_rng(L), 4, g.N, g.n_up, g.n_dn)
    y = model.features(torch.from_numpy(s).to(DEV)).cpu().numpy()
    hp = host_params(model)
    y0 = obf.cnn_forward(s, hp["conv_w"], hp["conv_b"], L, L)
    assert np.max(np.abs(y - y0)) < 2e-5 * max(1.0, np.abs(y0).max())


@pytest.mark.parametrize("L,B,symm", [(8, 16, False), (8, 8, True), (16, 4, False), (16, 2, True)])
def test_amplitude(L, B, symm):
    model = make_model(L, std=0.3, seed=1)
    g = model.geom
    s = olat.random_configs(np.random.default_rng(10 + L), B, g.N, g.n_up, g.n_dn)
    state = nh.Variational(model, symm=symm)
    psi = state(s)
    sg, la = psi.numpy()
    s0, l0 = oproj.projected_amplitude(s, host_params(model), symm=symm)
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < LOG_TOL


@pytest.mark.parametrize("L,symm", [(8, True), (16, False)])
def test_amplitude_all_fp64(L, symm):
    """cond_tau = 1 flags every item, so the whole batch takes the FP64 recompute path."""
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=32, std=0.3, seed=5)
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=1.0)
    s = olat.random_configs(np.random.default_rng(31), 3, N, ne, ne)
    psi = nh.Variational(model, symm=symm)(s)
    sg, la = psi.numpy()
    assert np.all(psi.flags.cpu().numpy() & _lib.FLAG_REFINED)
    s0, l0 = oproj.projected_amplitude(s, host_params(model), symm=symm)
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < 1e-9


@pytest.mark.parametrize("std,symm", [(0.3, False), (0.02, True)])
def test_amplitude_tensor_core_cnn(std, symm):
    """tcgen05 CNN.  BF16 x3 (mode 2) carries ~16 significant bits per feature: it meets the
    1e-4 bar with the benchmark's weights (std 0.02) and stays within 1e-3 with rough test weights
    (std 0.3); BF16 (mode 1) is the low-precision form.  Signs must match the oracle."""
    L, ne = 16, 112
    params = nh.init_params(L, L, channels=32, std=std, seed=6)
    s = olat.random_configs(np.random.default_rng(52), 3, L * L, ne, ne)
    m0 = nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=0)
    s0, l0 = oproj.projected_amplitude(s, host_params(m0), symm=symm)
    for mode, tol in ((2, LOG_TOL if std < 0.1 else 1e-3), (1, 5e-2 if std < 0.1 else 0.5)):
        m = nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=mode)
        psi = nh.Variational(m, symm=symm)(s)
        sg, la = psi.numpy()
        assert not (psi.flags.cpu().numpy() & _lib.FLAG_NONFINITE).any()
        assert np.array_equal(sg, s0), mode
        assert np.max(np.abs(la - l0)) < tol, (mode, np.max(np.abs(la - l0)))


@pytest.mark.parametrize("L,ne,std,symm", [(8, 14, 0.3, True), (10, 25, 0.3, False),
                                           (12, 63, 0.3, False), (12, 65, 0.3, True),
                                           (16, 112, 0.02, True), (16, 128, 0.3, False)])
def test_amplitude_tensor_memory_pfaffian(L, ne, std, symm):
    """pf_mode 1 (optional): matrix in tensor memory, 3xTF32 tcgen05 trailing updates.  n = 28 ...
    256 covers one 128-row tile (NP = 32, 64, 128) and two (NP = 160, 224, 256).  Signs exact.
    The tensor cores' accumulation into the FP32 matrix does not round like an FMA, so this mode
    carries its own measured bar, 3e-4 in log|psi| after the FP64 recompute (the CUDA-core
    kernel of the default path meets 1e-4).  Without the recompute it stays close to the
    CUDA-core FP32 kernel."""
    params = nh.init_params(L, L, channels=32, std=std, seed=7)
    s = olat.random_configs(np.random.default_rng(60 + L + ne), 3, L * L, ne, ne)
    m1 = nh.PfaffianBackflow(L, L, ne, ne, params=params, pf_mode=1)
    psi = nh.Variational(m1, symm=symm)(s)
    sg, la = psi.numpy()
    assert not (psi.flags.cpu().numpy() & _lib.FLAG_NONFINITE).any()
    s0, l0 = oproj.projected_amplitude(s, host_params(m1), symm=symm)
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < 3e-4, np.max(np.abs(la - l0))
    # FP32 only: the two FP32 kernels agree to their own rounding error
    m0 = nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=0.0, pf_mode=0)
    m1f = nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=0.0, pf_mode=1)
    a0 = nh.Variational(m0, symm=False)(s)
    a1 = nh.Variational(m1f, symm=False)(s)
    assert torch.equal(a0.sign, a1.sign)
    assert torch.max(torch.abs(a0.logabs - a1.logabs)).item() < 1e-2


def test_chosen_forms_16x16():
    """The benchmark's chosen form (tcgen05 BF16x3 CNN, CUDA-core Pfaffian) meets the 1e-4 bar at
    the benchmark's initialisation; with the tensor-memory Pfaffian (pf_mode 1) it meets that
    mode's 3e-4 bar.  Signs exact in both."""
    L, ne = 16, 112
    params = nh.init_params(L, L, channels=32, std=0.02, seed=0)
    s = olat.random_configs(np.random.default_rng(8), 2, L * L, ne, ne)
    for pf_mode, tol in ((0, LOG_TOL), (1, 3e-4)):
        m = nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=2, pf_mode=pf_mode)
        sg, la = nh.Variational(m, symm=True)(s).numpy()
        if pf_mode == 0:
            s0, l0 = oproj.projected_amplitude(s, host_params(m), symm=True)
        assert np.array_equal(sg, s0)
        assert np.max(np.abs(la - l0)) < tol, (pf_mode, np.max(np.abs(la - l0)))


def test_local_energy_tensor_memory_pfaffian():
    L, ne = 8, 28
    params = nh.init_params(L, L, channels=32, std=0.3, seed=2)
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params, pf_mode=1)
    s = olat.random_configs(np.random.default_rng(22), 3, L * L, ne, ne)
    e = nh.Hubbard(8.0, [1.0, -0.2], [1, 2]).Oloc(nh.Variational(model, symm=False),
                                                   nh.Samples(s)).cpu().numpy()
    hp = host_params(model)
    e0 = ohub.local_energy(s, lambda c: oproj.projected_amplitude(c, hp, symm=False), L, L,
                           1.0, -0.2, 8.0)
    # amplitude ratios carry the mode's ~3e-4 log|psi| bar, so 1e-4 relative per sample
    assert np.max(np.abs(e - e0) / np.abs(e0)) < 1e-4


def test_amplitude_baseline_init_16x16():
    """The benchmark's own initialisation (weights N(0, 0.02)) at 16x16, 8 images."""
    model = make_model(16, std=0.02, seed=0)
    g = model.geom
    s = olat.random_configs(np.random.default_rng(5), 2, g.N, g.n_up, g.n_dn)
    sg, la = nh.Variational(model, symm=True)(s).numpy()
    s0, l0 = oproj.projected_amplitude(s, host_params(model), symm=True)
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < LOG_TOL


def test_unfused_path_is_bitwise_equal():
    """features -> gather -> slogpf equals the fused amplitude entry point bit for bit."""
    model = make_model(8, std=0.3, seed=4)
    g = model.geom
    s = olat.random_configs(np.random.default_rng(6), 6, g.N, g.n_up, g.n_dn)
    ts = torch.from_numpy(s).to(DEV)
    y = model.features(ts)
    idx = torch.from_numpy(obf.fermion_idx(s).astype(np.int32)).to(DEV)
    Y = torch.gather(y.reshape(6, 2 * g.N, g.d), 1, idx.long()[:, :, None].expand(-1, -1, g.d))
    F = nh.pairing_occ(Y.contiguous(), idx, model.Wt, g)
    sg, la, _ = nh.slogpf(F, cond_tau=0.0)
    model.cond_tau = 0.0
    model.refine_tau = 0.0
    psi = nh.Variational(model, symm=False)(ts)
    assert torch.equal(psi.sign, sg) and torch.equal(psi.logabs, la)


@pytest.mark.parametrize("L,n_dirs", [(8, 8), (16, 8), (16, 4)])
def test_hop_list_bit_exact(L, n_dirs):
    N = L * L
    ne = 7 * N // 16
    s = olat.random_configs(np.random.default_rng(L + n_dirs), 12, N, ne, ne)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2]) if n_dirs == 8 else nh.Hubbard(8.0, 1.0, 1)
    counts, offsets, rec, hval = H.hop_list(torch.from_numpy(s).to(DEV), L, L)
    counts, offsets, rec, hval = (x.cpu().numpy() for x in (counts, offsets, rec, hval))
    assert np.array_equal(counts, ohub.hop_counts(s, L, L, n_dirs))
    for b in range(12):
        fr, to, hv = ohub.hops(s[b], L, L, 1.0, -0.2 if n_dirs == 8 else 0.0, n_dirs)
        sl = slice(offsets[b], offsets[b + 1])
        assert np.array_equal(rec[sl, 0], fr) and np.array_equal(rec[sl, 1], to)
        assert np.array_equal(hval[sl], hv)


def test_local_energy_against_fock_hamiltonian():
    """4x4, 2 + 2 electrons: GPU E_loc equals sum_s' H[s, s'] psi(s') / psi(s) with H from
    explicit fermion operators (golden fixture)."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "hubbard_4x4.npz"))
    params = nh.init_params(4, 4, channels=16, std=0.3, seed=9)
    model = nh.PfaffianBackflow(4, 4, 2, 2, params=params)
    for symm in (False, True):
        state = nh.Variational(model, symm=symm)
        H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
        spins = g["spins"]
        e = H.Oloc(state, nh.Samples(spins)).cpu().numpy()
        sg_all, la_all = state(g["conn"]).numpy()
        sg0, la0 = state(spins).numpy()
        sgo, _ = oproj.projected_amplitude(spins, host_params(model), symm=symm)
        off = 0
        checked = 0
        for b, cnt in enumerate(g["counts"]):
            sl = slice(off, off + cnt)
            off += cnt
            # symmetry-forbidden: psi_P(s) = 0 (exactly, or to rounding: the images then cancel
            # completely and the FP64 recompute may return 0 where the oracle keeps a residue)
            if sgo[b] == 0 or sg0[b] == 0:
                continue
            terms = g["vals"][sl] * sg_all[sl] * sg0[b] * np.exp(la_all[sl] - la0[b])
            # near-forbidden samples cancel terms of ~1e7 down to O(1): bound by sum |terms|
            assert abs(e[b] - terms.sum()) <= 1e-12 * np.abs(terms).sum() + 1e-9
            checked += 1
        assert checked >= 40


def test_local_energy_vs_oracle():
    L = 8
    model = make_model(L, std=0.3, seed=2)
    g = model.geom
    s = olat.random_configs(np.random.default_rng(21), 3, g.N, g.n_up, g.n_dn)
    state = nh.Variational(model, symm=False)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    e = H.Oloc(state, nh.Samples(s)).cpu().numpy()
    hp = host_params(model)

    def amp(c):
        return oproj.projected_amplitude(c, hp, symm=False)

    e0 = ohub.local_energy(s, amp, L, L, 1.0, -0.2, 8.0)
    # weights N(0, 0.3) give |E_loc| ~ 100-1000 t: relative bar per sample
    assert np.max(np.abs(e - e0) / np.abs(e0)) < 2e-5


@pytest.mark.parametrize("L,B", [(8, 16), (16, 2)])
def test_local_energy_baseline_init(L, B):
    """The benchmark's initialisation (N(0, 0.02)): batch-mean E_loc within 1e-5 t per site."""
    model = make_model(L, std=0.02, seed=0)
    g = model.geom
    s = olat.random_configs(np.random.default_rng(40 + L), B, g.N, g.n_up, g.n_dn)
    state = nh.Variational(model, symm=False)
    e = nh.Hubbard(8.0, [1.0, -0.2], [1, 2]).Oloc(state, nh.Samples(s)).cpu().numpy()
    hp = host_params(model)
    e0 = ohub.local_energy(s, lambda c: oproj.projected_amplitude(c, hp, symm=False), L, L,
                           1.0, -0.2, 8.0)
    assert abs(e.mean() - e0.mean()) / g.N < 1e-5


def test_metropolis_bookkeeping_replay():
    """The GPU sampler's chains equal an oracle replay that uses the same Philox draws and the
    GPU amplitudes of the proposed configurations (bookkeeping bit-exact)."""
    L = 8
    model = make_model(L, std=0.3, seed=3)
    g = model.geom
    state = nh.Variational(model, symm=False)
    s0 = olat.random_configs(np.random.default_rng(7), 48, g.N, g.n_up, g.n_dn)
    smp = nh.ParticleHop(state, 48, n_neighbor=(1, 2), initial_spins=s0, seed=1234)
    psi0 = (smp.psi.sign.cpu().numpy().astype(np.float64), smp.psi.logabs.cpu().numpy())
    smp.run(25)
    s_gpu = smp.spins.cpu().numpy()

    def amp(c):
        sg, la = state(c).numpy()
        return sg.astype(np.float64), la

    s_ref, sg_ref, la_ref, acc = osam.metropolis_steps(s0, psi0, amp, L, L, 1234, 0, 25)
    assert np.array_equal(s_gpu, s_ref)
    assert np.array_equal(smp.accepted.cpu().numpy(), acc)
    assert np.array_equal(smp.psi.logabs.cpu().numpy(), la_ref)
    # particle numbers conserved
    assert np.all((s_gpu[:, : g.N] > 0).sum(1) == g.n_up)
    assert np.all((s_gpu[:, g.N :] > 0).sum(1) == g.n_dn)


def test_mixed_sampler_bookkeeping_replay():
    """MixSampler([ParticleHop, SiteExchange]) (code/states.py:397-408): hop steps on the first
    half of the chains, site exchanges on the second; the chains equal an oracle replay with the
    same Philox draws and the GPU amplitudes of the proposed configurations, bit for bit."""
    L = 8
    model = make_model(L, std=0.3, seed=5)
    g = model.geom
    state = nh.Variational(model, symm=False)
    s0 = olat.random_configs(np.random.default_rng(17), 48, g.N, g.n_up, g.n_dn)
    hop = nh.ParticleHop(state, 24, n_neighbor=(1, 2))
    exc = nh.SiteExchange(state, 24, n_neighbor=(1, 2))
    smp = nh.MixSampler([hop, exc], initial_spins=s0, seed=4321)
    assert smp.first_exchange == 24 and smp.nsamples == 48
    psi0 = (smp.psi.sign.cpu().numpy().astype(np.float64), smp.psi.logabs.cpu().numpy())
    smp.run(30)
    s_gpu = smp.spins.cpu().numpy()

    def amp(c):
        sg, la = state(c).numpy()
        return sg.astype(np.float64), la

    s_ref, sg_ref, la_ref, acc = osam.metropolis_steps(s0, psi0, amp, L, L, 4321, 0, 30,
                                                       first_exchange=24)
    assert np.array_equal(s_gpu, s_ref)
    assert np.array_equal(smp.accepted.cpu().numpy(), acc)
    assert np.array_equal(smp.psi.logabs.cpu().numpy(), la_ref)
    assert acc[24:].sum() > 0  # exchanges were accepted
    assert np.all((s_gpu[:, : g.N] > 0).sum(1) == g.n_up)
    assert np.all((s_gpu[:, g.N :] > 0).sum(1) == g.n_dn)


@pytest.mark.parametrize("symm", [False, True])
def test_local_energy_in_cuda_graph(symm):
    """Without the connection count the local energy never waits for the GPU: recorded once in
    a CUDA graph it replays on new configurations and equals the direct call bit for bit."""
    L = 8
    model = make_model(L, std=0.3, seed=12)
    g = model.geom
    state = nh.Variational(model, symm=symm)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    rng = np.random.default_rng(70)
    s1 = torch.from_numpy(olat.random_configs(rng, 24, g.N, g.n_up, g.n_dn)).to(DEV)
    s2 = torch.from_numpy(olat.random_configs(rng, 24, g.N, g.n_up, g.n_dn)).to(DEV)
    ref = [H.Oloc(state, nh.Samples(s, state(s)), chunk_configs=512) for s in (s1, s2)]
    assert H.last_n_conn > 0
    spins = s1.clone()
    psi = state(spins)
    sign, logabs = psi.sign.clone(), psi.logabs.clone()
    samples = nh.Samples(spins, nh.LogArray(sign, logabs))
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # warm-up off the capture: workspace and kernel attributes
        H.Oloc(state, samples, chunk_configs=512, count_connections=False)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        out = H.Oloc(state, samples, chunk_configs=512, count_connections=False)
    assert H.last_n_conn is None
    for s, e_ref in zip((s1, s2), ref):
        p = state(s)
        spins.copy_(s)
        sign.copy_(p.sign)
        logabs.copy_(p.logabs)
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, e_ref)


def test_local_energy_chunk_autotune():
    L = 8
    model = make_model(L, std=0.3, seed=13)
    g = model.geom
    state = nh.Variational(model, symm=False)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    s = olat.random_configs(np.random.default_rng(71), 64, g.N, g.n_up, g.n_dn)
    smp = nh.Samples(torch.from_numpy(s).to(DEV))
    ref = H.Oloc(state, smp, chunk_configs=4096)
    best = H.autotune(state, smp, candidates=(1024, 4096, 16384), repeats=1)
    assert best in (1024, 4096, 16384)
    e = H.Oloc(state, smp)  # uses the tuned chunk
    assert torch.allclose(e, ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("symm", [False, True])
def test_local_energy_persistent_equals_chunked(symm):
    """The persistent pass (one fused launch over every (configuration, image, connection) item,
    refinement with features recomputed in the kernel) computes the same arithmetic as the
    chunked pipeline: local energies equal bit for bit; and its launch count does not depend on
    the number of samples (a fixed launch sequence)."""
    L = 8
    model = make_model(L, std=0.3, seed=14)
    g = model.geom
    state = nh.Variational(model, symm=symm)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    s = torch.from_numpy(olat.random_configs(np.random.default_rng(72), 40, g.N, g.n_up,
                                              g.n_dn)).to(DEV)
    samples = nh.Samples(s, state(s))
    e_chunk = H.Oloc(state, samples, chunk_configs=512)
    e_pers = H.Oloc(state, samples, chunk_configs=0)
    assert torch.equal(e_pers, e_chunk)
    launches = []
    for B in (8, 40):
        sb = nh.Samples(s[:B].contiguous(), state(s[:B]))
        torch.cuda.synchronize()
        _lib.profile_read()
        _lib.profile_enable(True)
        H.Oloc(state, sb, chunk_configs=0, count_connections=False)
        torch.cuda.synchronize()
        _lib.profile_enable(False)
        launches.append(sum(n for _, n in _lib.profile_read().values()))
    assert launches[0] == launches[1], launches


@pytest.mark.parametrize("cnn_mode", [0, 2])
def test_accuracy_at_scale_16x16(cnn_mode):
    """Both default forms (plain: FP32 CNN; chosen: tcgen05 BF16x3 CNN) on 1024 projected 16x16
    configurations with the benchmark's weights (N(0, 0.02)): log|psi_P| within 1e-4 of the
    all-FP64 path (cond_tau = 1, itself equal to the FP64 oracle to 1e-9) on every
    configuration, and no sign mismatch.  The default policy: FP64 features and an FP64
    refinement with the FP32 pivot order for the images whose share of psi_P times pivot ratio
    exceeds cond_tau, and for every image carrying more than 2% of a configuration whose images
    cancel by more than cancel_tau."""
    L, ne, B = 16, 112, 1024
    params = nh.init_params(L, L, channels=32, std=0.02, seed=0)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(2024), B, L * L, ne, ne)).to(DEV)
    ref = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=1.0),
                         symm=True, max_parallel=B)(s)
    psi = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=cnn_mode),
                         symm=True, max_parallel=B)(s)
    assert torch.equal(psi.sign, ref.sign)
    err = (psi.logabs - ref.logabs).abs().max().item()
    assert err < 1e-4, err


def test_cancellation_recompute():
    """cancel_tau: in configurations whose 8 images cancel, the images carrying more than 2% of
    |psi_P| are recomputed in FP64; those configurations then agree with the all-FP64 result to
    1e-4 (the FP32 images left carry < 2% weight), the others are unchanged."""
    L, ne = 16, 112
    params = nh.init_params(L, L, channels=32, std=0.02, seed=0)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(1000), 512, L * L, ne, ne)).to(DEV)
    ref = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=1.0),
                         symm=True)(s)
    base = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cancel_tau=0.0),
                          symm=True)(s)
    m = nh.PfaffianBackflow(L, L, ne, ne, params=params, cancel_tau=8.0)
    psi = nh.Variational(m, symm=True)(s)
    fl = psi.flags.cpu().numpy()
    cancel = (fl & _lib.FLAG_CANCEL) != 0
    assert 0 < cancel.sum() < len(fl)
    assert np.all(fl[cancel] & _lib.FLAG_REFINED)
    la, l0, lb = psi.logabs.cpu().numpy(), ref.logabs.cpu().numpy(), base.logabs.cpu().numpy()
    assert np.max(np.abs(la[cancel] - l0[cancel])) < 1e-4
    assert np.array_equal(la[~cancel], lb[~cancel])
    assert torch.equal(psi.sign, ref.sign)
    assert np.abs(la - l0).max() <= np.abs(lb - l0).max()
    # the flag reports the cancellation factor of the final amplitude
    assert not (base.flags.cpu().numpy() & _lib.FLAG_CANCEL).any()
