"""GPU parity of the amplitude's backward against the FP64 oracle (``oracle/gradient.py``, itself
checked against finite differences on the CPU): the Pfaffian adjoint (the derivative of
``fermix.slogpf``, ``code/backflow/models.py:210``), the custom VJP of the occupied gather
(``code/backflow/pf_kernel.py:193-320,354-365``) and the per-sample Jacobian of log|psi| that
SR / AdamSR consume (``code/train_pfaffian_16x16_tpm02.py:100-101``).

Everything on the GPU runs in FP32 (the reference's own precision for these cotangents), so the
bars are relative to each quantity's scale: 1e-5 for the gather's VJP (no inverse involved),
and for the inverse-based quantities a bound set by FP32 times the matrices' conditioning.
"""

import numpy as np
import pytest
import torch

import neuralhubbard_b200 as nh
from neuralhubbard_b200 import _lib
from oracle import backflow as obf
from oracle import gradient as og
from oracle import lattice as olat

pytestmark = pytest.mark.gpu
DEV = "cuda"


def host_params(model):
    p = model.host_params
    return dict(conv_w=[np.asarray(w, np.float64) for w in p["conv_w"]],
                conv_b=[np.asarray(b, np.float64) for b in p["conv_b"]],
                W=np.asarray(p["W"], np.float64), theta=float(p["theta"]),
                Lx=model.geom.LX, Ly=model.geom.LY)


def make_model(L, std, seed=0, channels=32, layers=4):
    N = L * L
    ne = 7 * N // 16
    params = nh.init_params(L, L, channels=channels, layers=layers, std=std, seed=seed)
    return nh.PfaffianBackflow(L, L, ne, ne, params=params)


@pytest.mark.parametrize("n", [2, 14, 56, 100, 224])
def test_pfaffian_adjoint_random(n):
    rng = np.random.default_rng(n)
    A = rng.normal(size=(24, n, n))
    A = (A - np.swapaxes(A, 1, 2)).astype(np.float32)
    G, fl = nh.slogpf_adjoint(torch.from_numpy(A).to(DEV))
    G = G.cpu().numpy()
    G0 = og.slogpf_adjoint(A.astype(np.float64))
    assert np.all(fl.cpu().numpy() == 0)
    cond = np.linalg.cond(A.astype(np.float64))
    for b in range(A.shape[0]):
        scale = np.max(np.abs(G0[b]))
        assert np.max(np.abs(G[b] - G0[b])) <= 2e-6 * cond[b] * scale + 1e-6 * scale, b


def test_pfaffian_adjoint_singular_flagged():
    rng = np.random.default_rng(1)
    A = rng.normal(size=(3, 56, 56))
    A = (A - np.swapaxes(A, 1, 2)).astype(np.float32)
    A[1, 7, :] = 0.0
    A[1, :, 7] = 0.0
    G, fl = nh.slogpf_adjoint(torch.from_numpy(A).to(DEV))
    fl = fl.cpu().numpy()
    assert fl[0] == 0 and fl[2] == 0 and fl[1] == _lib.FLAG_ZERO_PIVOT
    assert np.all(G[1].cpu().numpy() == 0.0)
    G0 = og.slogpf_adjoint(A[[0, 2]].astype(np.float64))
    assert np.allclose(G[[0, 2]].cpu().numpy(), G0, atol=1e-3 * np.abs(G0).max())


@pytest.mark.parametrize("L", [4, 8, 16])
def test_pairing_occ_vjp(L):
    N = L * L
    ne = 7 * N // 16
    rng = np.random.default_rng(L)
    s = olat.random_configs(rng, 5, N, ne, ne)
    idx = obf.fermion_idx(s)
    n = idx.shape[1]
    d = 16
    Y = rng.normal(size=(5, n, d)).astype(np.float32)
    W = (rng.normal(size=(3, N, d)) / 4).astype(np.float32)
    geom = nh.PairGeometry(L, L, d, ne, ne)
    Wt = nh.build_wtilde(torch.from_numpy(W).to(DEV), 0.55, geom)
    G = rng.normal(size=(5, n, n)).astype(np.float32)
    dY, dWt = nh.pairing_occ_vjp(torch.from_numpy(Y).to(DEV),
                                 torch.from_numpy(idx.astype(np.int32)).to(DEV), Wt,
                                 torch.from_numpy(G).to(DEV), geom)
    dY0, dWt0 = og.pairing_occ_vjp(Y.astype(np.float64), idx, Wt.cpu().numpy().astype(np.float64),
                                   G.astype(np.float64), L, L)
    assert np.max(np.abs(dY.cpu().numpy() - dY0)) < 1e-5 * np.abs(dY0).max()
    assert np.max(np.abs(dWt.cpu().numpy() - dWt0)) < 1e-5 * np.abs(dWt0).max()


def jac_error(J, J0):
    """Largest deviation of each row relative to that row's largest entry."""
    return np.max(np.abs(J - J0), axis=1) / np.max(np.abs(J0), axis=1)


@pytest.mark.parametrize("symm", [False, True])
@pytest.mark.parametrize("std", [0.3, 0.02])
def test_log_jacobian_8x8(symm, std):
    model = make_model(8, std, seed=3)
    state = nh.Variational(model, symm=symm)
    s = olat.random_configs(np.random.default_rng(11), 12, 64, 28, 28)
    psi, J = state.jacobian(s)
    hp = host_params(model)
    sg0, la0, J0 = og.log_jacobian(s, hp, symm=symm)
    assert J.shape == (12, og.param_count(hp)) == (12, model.param_count)
    sg, la = psi.numpy()
    assert np.array_equal(sg, sg0)
    assert np.max(np.abs(la - la0)) < 1e-4
    err = jac_error(J.cpu().numpy(), J0)
    assert np.all(err < 2e-3), err
    assert np.median(err) < 2e-4, err
    # the amplitude returned on the way equals the plain amplitude call
    ref = state(s)
    assert np.array_equal(ref.sign.cpu().numpy(), sg)
    assert np.max(np.abs(ref.logabs.cpu().numpy() - la)) < 1e-9


def test_log_jacobian_16x16_projected():
    """The benchmark lattice (n = 224) with the benchmark weights (std 0.02), projected."""
    model = make_model(16, 0.02, seed=0)
    state = nh.Variational(model, symm=True)
    s = olat.random_configs(np.random.default_rng(5), 3, 256, 112, 112)
    psi, J = state.jacobian(s)
    sg0, la0, J0 = og.log_jacobian(s, host_params(model), symm=True, chunk=1)
    assert np.array_equal(psi.sign.cpu().numpy(), sg0)
    err = jac_error(J.cpu().numpy(), J0)
    assert np.all(err < 1e-2), err


def test_log_jacobian_chunks_and_repeat():
    """More samples than one workspace chunk, and bit-identical results on a repeat call."""
    model = make_model(4, 0.3, seed=2, channels=16, layers=3)
    state = nh.Variational(model, symm=True)
    s = olat.random_configs(np.random.default_rng(9), 700, 16, 7, 7)
    _, J1 = state.jacobian(s)
    _, J2 = state.jacobian(s)
    assert torch.equal(J1, J2)
    _, J0 = state.jacobian(s[:64], max_parallel=16)
    assert torch.equal(J1[:64], J0)
    sg0, la0, Jo = og.log_jacobian(s[:40], host_params(model), symm=True)
    assert np.all(jac_error(J1[:40].cpu().numpy(), Jo) < 2e-3)
