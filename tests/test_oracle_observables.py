"""The packed-observable oracle (``code/measure/transverse_spin.py``, ``dwave_packed.py``)
against exact expectation values on a small Fock space: for any amplitude psi,
<psi|O|psi> / <psi|psi> = sum_s |psi(s)|^2 O_loc(s) / sum_s |psi(s)|^2, where the exact side
applies O itself (not its adjoint) to every basis state (CPU only)."""

import numpy as np
import pytest

from oracle import hubbard as ohub
from oracle import observables as oobs


def exact_and_estimated(kind, Lx, Ly, a0, a1, n_up, n_dn, seed):
    N = Lx * Ly
    basis = ohub.fock_basis(N, n_up, n_dn)
    rng = np.random.default_rng(seed)
    psi = rng.normal(size=len(basis))
    key = {oobs._bits(s): k for k, s in enumerate(basis)}

    def amp(configs):
        v = np.array([psi[key[oobs._bits(c)]] for c in configs])
        return np.sign(v), np.log(np.abs(v))

    w = psi ** 2 / np.sum(psi ** 2)
    terms = oobs.terms(kind, Lx, Ly, a0, a1)
    # exact: <psi|O_t|psi> with O_t applied to |s'> (operators of O right to left)
    exact = np.zeros(len(terms))
    for t, (k, ops, diag) in enumerate(terms):
        if ops is None:
            continue
        # O_t^dag's operators act on s in this order; O_t = (O_t^dag)^dag acts on s' with the
        # reversed list and each operator conjugated.
        o_ops = [(m, not cr) for m, cr in reversed(ops)]
        for a, s in enumerate(basis):
            nb, c = oobs._apply(oobs._bits(s), o_ops)
            if nb is None or nb not in key:
                continue
            exact[k] += psi[key[nb]] * c * psi[a]
    exact /= np.sum(psi ** 2)
    # estimate: the per-sample local values weighted by |psi|^2
    est = np.zeros(len(terms))
    for a, s in enumerate(basis):
        loc = oobs.packed_mean(s[None], amp, kind, Lx, Ly, a0, a1)
        est += w[a] * loc
    diag_bins = [k for k, ops, d in terms if ops is None]
    return exact, est, diag_bins


@pytest.mark.parametrize("kind,a0,a1", [("transverse", 4, 0), ("pair", 0, 1), ("pair", 3, 2),
                                        ("hop", 5, 0), ("hop", 1, 1)])
def test_packed_estimator_matches_exact_expectation(kind, a0, a1):
    exact, est, diag_bins = exact_and_estimated(kind, 3, 2, a0, a1, 2, 3, 7)
    off = np.setdiff1d(np.arange(len(exact)), diag_bins)
    assert np.allclose(est[off], exact[off], atol=1e-12)
    assert np.max(np.abs(exact[off])) > 1e-3  # the check is not vacuous
