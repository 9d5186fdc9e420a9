"""GPU parity of the residual backflow network (the released states' ResConv, net =
NH_NET_RESCONV) against the FP64 oracle, and the end-to-end pin of the conventions: the
projected local energy of the released 16x16 state (t' = -0.2) on its own equilibrated chains
against the published E/N = -0.74533(1), sigma^2/N = 0.0272(5).

The released files come from tests/golden/fetch_released.py (git-ignored copies); the tests
that need them skip when they are absent.
"""

import os

import numpy as np
import pytest
import torch

import neuralhubbard_b200 as nh
from neuralhubbard_b200 import checkpoint
from neuralhubbard_b200.backflow import DEFAULT_COND_TAU
from oracle import projection as oproj
from oracle import resconv as orc
from oracle import lattice as olat

pytestmark = pytest.mark.gpu
DEV = "cuda"
RELEASED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "released")
NAME = "tpm02_L16_pfaffian"


def random_resconv(L, blocks, seed, std=0.04):
    """Random residual-network parameters (LeCun-normal-sized 3x3 convolutions)."""
    rng = np.random.default_rng(seed)
    C, N, d = 64, L * L, 32
    return dict(net="resconv",
                embed=rng.normal(size=(C, 4)).astype(np.float32),
                conv_w=[(rng.normal(size=(C, C, 3, 3)) * std).astype(np.float32)
                        for _ in range(2 * blocks)],
                conv_b=[(rng.normal(size=C) * 0.1).astype(np.float32) for _ in range(2 * blocks)],
                W=(rng.normal(size=(3, N, d)) / np.sqrt(d)).astype(np.float32),
                theta=float(np.float32(0.55)))  # the C ABI takes theta in FP32


def oracle_params(params, L):
    """The oracle forms the pairing table's antisymmetrised blocks in the dtype of W: FP64 here,
    as the library's FP64 table does."""
    return dict(params, Lx=L, Ly=L, W=np.asarray(params["W"], np.float64))


def released():
    eqx = os.path.join(RELEASED, NAME + ".eqx")
    if not os.path.exists(eqx):
        pytest.skip("released weights not fetched (tests/golden/fetch_released.py)")
    params = checkpoint.load_pfaffian_backflow(eqx, 16)
    spins = checkpoint.load_spins(os.path.join(RELEASED, NAME + "_spins.npz"), 256)
    return params, spins


@pytest.mark.parametrize("L,blocks", [(4, 3), (8, 4), (16, 2)])
def test_resconv_features(L, blocks):
    """Features (2, N, d) against the oracle."""
    N = L * L
    ne = 7 * N // 16
    params = random_resconv(L, blocks, seed=L)
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params)
    s = olat.random_configs(np.random.default_rng(L + 1), 3, N, ne, ne)
    y = model.features(torch.from_numpy(s).to(DEV)).cpu().numpy()
    y0 = orc.resconv_forward(s, params["embed"], params["conv_w"], params["conv_b"], L, L)
    assert y.shape == y0.shape
    assert np.max(np.abs(y - y0)) < 2e-5 * np.max(np.abs(y0))


@pytest.mark.parametrize("symm", [True, False])
def test_resconv_amplitude(symm):
    """8x8, 4 blocks: signs exact; FP64 path within 1e-8, default path within 1e-4."""
    L, N = 8, 64
    ne = 7 * N // 16
    params = random_resconv(L, 4, seed=7)
    s = olat.random_configs(np.random.default_rng(8), 6, N, ne, ne)
    s0, l0 = oproj.projected_amplitude(s, oracle_params(params, L), symm=symm)
    for tau, tol in [(1.0, 1e-8), (DEFAULT_COND_TAU, 1e-4)]:
        model = nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=tau)
        sg, la = nh.Variational(model, symm=symm)(s).numpy()
        assert np.array_equal(sg, s0)
        assert np.max(np.abs(la - l0)) < tol, (tau, np.max(np.abs(la - l0)))


def test_resconv_amplitude_large_lattice():
    """24x24 (N = 576): the FP32 planes live in global memory; unprojected amplitudes."""
    L, N = 24, 576
    ne = 7 * N // 16
    params = random_resconv(L, 1, seed=24)
    s = olat.random_configs(np.random.default_rng(25), 2, N, ne, ne)
    s0, l0 = oproj.projected_amplitude(s, oracle_params(params, L), symm=False)
    for tau, tol in [(1.0, 1e-8), (DEFAULT_COND_TAU, 1e-3)]:
        model = nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=tau)
        sg, la = nh.Variational(model, symm=False)(s).numpy()
        assert np.array_equal(sg, s0)
        assert np.max(np.abs(la - l0)) < tol, (tau, np.max(np.abs(la - l0)))


def test_released_state_amplitudes():
    """Projected amplitudes of stored chains of the released state: the all-FP64 path equals
    the oracle to 1e-8, the default path to 1e-3 (FP32 through 32 convolutions whose
    activations grow to ~30)."""
    params, spins = released()
    s = spins[:6]
    s0, l0 = oproj.projected_amplitude(s, oracle_params(params, 16))
    ne = 7 * 256 // 16
    for tau, tol in [(1.0, 1e-8), (DEFAULT_COND_TAU, 1e-3)]:
        model = nh.PfaffianBackflow(16, 16, ne, ne, params=params, cond_tau=tau)
        sg, la = nh.Variational(model)(s).numpy()
        assert np.array_equal(sg, s0)
        assert np.max(np.abs(la - l0)) < tol, (tau, np.max(np.abs(la - l0)))


def test_released_state_energy():
    """E/N of the released tpm02_L16_pfaffian state on 256 of its stored chains (projected
    amplitudes, U = 8, t' = -0.2) within 4 standard errors of the published -0.74533, and the
    per-site variance near the published 0.0272: pins the occupation embedding, the network,
    the mode order, the fermionic image signs and the hopping signs together."""
    params, spins = released()
    info = checkpoint.RELEASED[NAME]
    ne = 7 * 256 // 16
    model = nh.PfaffianBackflow(16, 16, ne, ne, params=params)
    state = nh.Variational(model)
    H = nh.Hubbard(8.0, [1.0, info.tprime], [1, 2])
    s = torch.from_numpy(spins[:256]).to(DEV)
    e = H.Oloc(state, nh.Samples(s, state(s))).cpu().numpy() / 256
    mean, err = e.mean(), e.std(ddof=1) / np.sqrt(len(e))
    var = e.var(ddof=1) * 256
    assert abs(mean - info.energy) < 4 * err, (mean, err)
    assert 0.5 * info.variance < var < 1.5 * info.variance, var


@pytest.mark.parametrize("blocks", [1, 3])
def test_resconv_tc_amplitude(blocks):
    """16x16 on the tensor cores (cnn_mode 2, BF16 x3 products) with the default FP64 recompute
    of ill-conditioned images: signs exact, log|psi| within 1e-3 of the FP64 oracle (about 2e-4
    on the released state)."""
    L, N = 16, 256
    ne = 7 * N // 16
    params = random_resconv(L, blocks, seed=30 + blocks)
    s = olat.random_configs(np.random.default_rng(40 + blocks), 4, N, ne, ne)
    for symm in (False, True):
        s0, l0 = oproj.projected_amplitude(s, oracle_params(params, L), symm=symm)
        model = nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=2)
        sg, la = nh.Variational(model, symm=symm)(s).numpy()
        assert np.array_equal(sg, s0)
        assert np.max(np.abs(la - l0)) < 1e-3, (symm, np.max(np.abs(la - l0)))


def test_released_state_energy_tensor_cores():
    """The tensor-core network (cnn_mode 2) gives the released state's E/N on 256 stored chains
    within 4 standard errors of the published value as well."""
    params, spins = released()
    info = checkpoint.RELEASED[NAME]
    ne = 7 * 256 // 16
    state = nh.Variational(nh.PfaffianBackflow(16, 16, ne, ne, params=params, cnn_mode=2))
    H = nh.Hubbard(8.0, [1.0, info.tprime], [1, 2])
    s = torch.from_numpy(spins[256:512]).to(DEV)
    e = H.Oloc(state, nh.Samples(s, state(s))).cpu().numpy() / 256
    mean, err = e.mean(), e.std(ddof=1) / np.sqrt(len(e))
    assert abs(mean - info.energy) < 4 * err, (mean, err)


def test_released_L24_state_energy():
    """The released 24x24 state tpm02_L24_pfaffian (n = 504: the large-lattice Pfaffian and the
    residual network with its activation planes in global memory) on 64 of its stored chains:
    projected E/N within 4 standard errors of the published -0.74585(1) (code/states.py:118-119;
    standard error from the published sigma^2/N = 0.0257)."""
    name, L = "tpm02_L24_pfaffian", 24
    eqx = os.path.join(RELEASED, name + ".eqx")
    if not os.path.exists(eqx):
        pytest.skip("released weights not fetched (tests/golden/fetch_released.py)")
    info = checkpoint.RELEASED[name]
    N = L * L
    ne = 7 * N // 16
    params = checkpoint.load_pfaffian_backflow(eqx, L, expect_md5=info.md5)
    spins = checkpoint.load_spins(os.path.join(RELEASED, name + "_spins.npz"), N, ne, ne)
    state = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params))
    H = nh.Hubbard(8.0, [1.0, info.tprime], [1, 2])
    s = torch.from_numpy(spins[:64]).to(DEV)
    e = H.Oloc(state, nh.Samples(s, state(s)), chunk_configs=2048).cpu().numpy() / N
    err = np.sqrt(info.variance / N / len(e))
    assert abs(e.mean() - info.energy) < 4 * err, (e.mean(), err)
