"""GPU parity of the packed observables (``code/measure/transverse_spin.py:44-119``,
``code/measure/dwave_packed.py:24-103``) against the FP64 oracle ``oracle/observables.py`` (itself
checked against exact Fock-space expectation values on the CPU).  The all-FP64 amplitude form is
compared at 1e-9, the default form at 1e-4 of each family's scale."""

import numpy as np
import pytest

import neuralhubbard_b200 as nh
from neuralhubbard_b200 import _lib
from neuralhubbard_b200.observables import PackedDwave, observable, transverse_terms
from oracle import lattice as olat
from oracle import observables as oobs
from oracle import projection as oproj

pytestmark = pytest.mark.gpu


def host(model, L):
    p = model.host_params
    return dict(conv_w=[np.asarray(w, np.float64) for w in p["conv_w"]],
                conv_b=[np.asarray(b, np.float64) for b in p["conv_b"]],
                W=np.asarray(p["W"], np.float64), theta=float(p["theta"]), Lx=L, Ly=L)


KINDS = [(_lib.OBS_TRANSVERSE_SPIN, "transverse", 5, 0), (_lib.OBS_PAIR, "pair", 5, 6),
         (_lib.OBS_PAIR, "pair", 9, 5), (_lib.OBS_HOP, "hop", 3, 0), (_lib.OBS_HOP, "hop", 10, 1)]


@pytest.mark.parametrize("symm", [False, True])
@pytest.mark.parametrize("cond_tau,tol", [(1.0, 1e-9), (None, 1e-4)])
def test_observables_4x4(symm, cond_tau, tol):
    L, ne = 4, 7
    params = nh.init_params(L, L, channels=32, layers=2, std=0.3, seed=5)
    kw = {} if cond_tau is None else {"cond_tau": cond_tau}
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params, **kw)
    state = nh.Variational(model, symm=symm)
    s = olat.random_configs(np.random.default_rng(1), 24, 16, ne, ne)
    hp = host(model, L)
    amp = lambda c: oproj.projected_amplitude(c, hp, symm=symm)  # noqa: E731
    psi0 = amp(s)
    samples = nh.Samples(s)
    for kind, name, a0, a1 in KINDS:
        got = observable(state, samples, kind, a0, a1).cpu().numpy().ravel()
        ref = oobs.packed_mean(s, amp, name, L, L, a0, a1, psi=psi0)
        assert np.max(np.abs(got - ref)) <= tol * max(1.0, np.max(np.abs(ref))), (name, a0, a1)


def test_packed_dwave_key_order_and_transverse_8x8():
    L, ne = 8, 28
    params = nh.init_params(L, L, std=0.3, seed=2)
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=1.0)
    state = nh.Variational(model, symm=True)
    s = olat.random_configs(np.random.default_rng(3), 8, 64, ne, ne)
    samples = nh.Samples(s)
    hp = host(model, L)
    amp = lambda c: oproj.projected_amplitude(c, hp, symm=True)  # noqa: E731
    psi0 = amp(s)
    T = transverse_terms(state, samples, (2, 3)).cpu().numpy()
    Tref = oobs.packed_mean(s, amp, "transverse", L, L, 2 * L + 3, psi=psi0).reshape(2, -1)
    assert np.max(np.abs(T - Tref)) < 1e-9
    dw = PackedDwave(L, L, R=(1, 2))
    F, G = dw.measure(state, samples)
    assert len(F) == len(dw.F_keys) and len(G) == len(dw.G_keys)
    # spot-check keys against the oracle
    for k in (0, 5, 77, len(dw.F_keys) - 1):
        bl, oL, br, oR = dw.F_keys[k]
        lo, hi = dw.bond_sites(bl)
        a, b = (lo, hi) if oL == 0 else (hi, lo)
        t = (dw.index(br[:2]) * 2 + br[2]) * 2 + oR
        ref = oobs.packed_mean(s, amp, "pair", L, L, dw.index(a), dw.index(b), psi=psi0)[t]
        assert abs(F[k] - ref) < 1e-9, k
    for k in (0, 3, len(dw.G_keys) - 1):
        i, j, sp = dw.G_keys[k]
        ref = oobs.packed_mean(s, amp, "hop", L, L, dw.index(i), "ud".index(sp), psi=psi0)
        assert abs(G[k] - ref[dw.index(j)]) < 1e-9, k
