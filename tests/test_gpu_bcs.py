"""GPU parity of the BCS-backflow ansatz (``code/backflow/models.py:214-302``,
``code/backflow/bcs_kernel.py``) against the FP64 oracle ``oracle/bcs.py``, which is itself
checked against the Pfaffian oracle on the CPU (the BCS amplitude is the Pfaffian of
[[0, F], [-F^T, 0]]).  Bars: signs bit-exact; log|psi| within 1e-4 on the FP32 path with the
default recompute policy, within 1e-9 on the all-FP64 form."""

import numpy as np
import pytest
import torch

import neuralhubbard_b200 as nh
from oracle import bcs as obcs
from oracle import hubbard as ohub
from oracle import lattice as olat

pytestmark = pytest.mark.gpu


def bcs_params(L, std, seed, delta_d, channels=32, layers=4):
    p = nh.init_params(L, L, channels=channels, layers=layers, std=std, seed=seed)
    p["W"] = p["W"][0]
    p["delta_d"] = delta_d
    return p


def host(p, L):
    return dict(conv_w=[np.asarray(w, np.float64) for w in p["conv_w"]],
                conv_b=[np.asarray(b, np.float64) for b in p["conv_b"]],
                W=np.asarray(p["W"], np.float64), theta=float(p["theta"]),
                delta_d=float(p["delta_d"]), Lx=L, Ly=L)


@pytest.mark.parametrize("L", [4, 8])
@pytest.mark.parametrize("symm", [False, True])
def test_bcs_amplitude(L, symm):
    N = L * L
    ne = 7 * N // 16
    p = bcs_params(L, 0.3, 1, 0.37)
    model = nh.BCSBackflow(L, L, ne, ne, params=p)
    s = olat.random_configs(np.random.default_rng(L), 16, N, ne, ne)
    sg, la = nh.Variational(model, symm=symm)(s).numpy()
    s0, l0 = obcs.projected_amplitude(s, host(p, L), symm=symm)
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < 1e-4
    # all-FP64 form
    m64 = nh.BCSBackflow(L, L, ne, ne, params=p, cond_tau=1.0)
    sg, la = nh.Variational(m64, symm=symm)(s).numpy()
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < 1e-9


def test_bcs_equals_pfaffian_state_without_dwave():
    """delta_d = 0: the BCS state is the Pfaffian state with W = [W_ud, 0, 0]."""
    L, ne = 8, 28
    p = bcs_params(L, 0.3, 2, 0.0)
    s = olat.random_configs(np.random.default_rng(3), 32, 64, ne, ne)
    b = nh.Variational(nh.BCSBackflow(L, L, ne, ne, params=p, cond_tau=1.0), symm=True)(s)
    pf = dict(p)
    pf["W"] = np.stack([p["W"], np.zeros_like(p["W"]), np.zeros_like(p["W"])])
    pf.pop("delta_d")
    q = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=pf, cond_tau=1.0), symm=True)(s)
    assert torch.equal(b.sign, q.sign)
    assert torch.max(torch.abs(b.logabs - q.logabs)).item() < 1e-9


def test_bcs_16x16_projected():
    """The benchmark lattice (n_up = 112) with the benchmark weights, default policy."""
    L, ne = 16, 112
    p = bcs_params(L, 0.02, 0, 0.1)
    model = nh.BCSBackflow(L, L, ne, ne, params=p)
    s = olat.random_configs(np.random.default_rng(7), 4, 256, ne, ne)
    sg, la = nh.Variational(model, symm=True)(s).numpy()
    s0, l0 = obcs.projected_amplitude(s, host(p, L), symm=True)
    assert np.array_equal(sg, s0)
    assert np.max(np.abs(la - l0)) < 1e-4


def test_bcs_local_energy_and_sampler():
    L, ne = 4, 7
    p = bcs_params(L, 0.3, 4, 0.25, channels=32, layers=2)
    model = nh.BCSBackflow(L, L, ne, ne, params=p, cond_tau=1.0)
    state = nh.Variational(model, symm=False)
    s = olat.random_configs(np.random.default_rng(5), 6, 16, ne, ne)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    e = H.Oloc(state, nh.Samples(s)).cpu().numpy()
    hp = host(p, L)
    e0 = ohub.local_energy(s, lambda c: obcs.amplitude(c, hp), L, L, 1.0, -0.2, 8.0)
    assert np.max(np.abs(e - e0) / np.maximum(1.0, np.abs(e0))) < 1e-8
    smp = nh.ParticleHop(nh.Variational(model, symm=True), 64, n_neighbor=(1, 2),
                         initial_spins=olat.random_configs(np.random.default_rng(6), 64, 16, ne, ne),
                         seed=9)
    smp.run(20)
    sp = smp.spins
    assert torch.all((sp[:, :16] > 0).sum(1) == ne) and torch.all((sp[:, 16:] > 0).sum(1) == ne)
    ref = nh.Variational(model, symm=True)(sp)
    assert torch.equal(ref.sign, smp.psi.sign)
    assert torch.max(torch.abs(ref.logabs - smp.psi.logabs)).item() < 1e-12
