"""Oracle Pfaffian: known-answer tests from mathematics and the golden matchings sums."""

import os

import numpy as np
import pytest

from oracle import pfaffian

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rand_skew(rng, n, batch=None):
    shape = (n, n) if batch is None else (batch, n, n)
    A = rng.normal(size=shape)
    return A - np.swapaxes(A, -1, -2)


def test_golden_matchings():
    g = np.load(os.path.join(GOLDEN, "pfaffian_kat.npz"))
    for A8, n, pf in zip(g["A"], g["n"], g["pf"]):
        A = A8[:n, :n]
        s, la = pfaffian.slogpf(A)
        assert s * np.exp(la) == pytest.approx(pf, rel=1e-12, abs=1e-14)
        assert pfaffian.pf_bruteforce(A) == pytest.approx(pf, rel=1e-12, abs=1e-14)


@pytest.mark.parametrize("n", [2, 4, 10, 32, 56])
def test_pf_squared_is_det(n):
    rng = np.random.default_rng(n)
    A = rand_skew(rng, n)
    s, la = pfaffian.slogpf(A)
    sd, ld = np.linalg.slogdet(A)
    assert sd > 0
    assert 2 * la == pytest.approx(ld, abs=1e-9)


@pytest.mark.parametrize("n", [4, 12, 40])
def test_congruence(n):
    """pf(B^T A B) = det(B) pf(A): pins the sign."""
    rng = np.random.default_rng(100 + n)
    A = rand_skew(rng, n)
    B = rng.normal(size=(n, n))
    s1, l1 = pfaffian.slogpf(B.T @ A @ B)
    s0, l0 = pfaffian.slogpf(A)
    sb, lb = np.linalg.slogdet(B)
    assert s1 == s0 * sb
    assert l1 == pytest.approx(l0 + lb, abs=1e-9)


def test_block_diagonal_and_swap():
    a = np.array([1.5, -0.25, 3.0, -2.0])
    A = np.zeros((8, 8))
    for k, v in enumerate(a):
        A[2 * k, 2 * k + 1], A[2 * k + 1, 2 * k] = v, -v
    s, la = pfaffian.slogpf(A)
    assert s * np.exp(la) == pytest.approx(np.prod(a))
    P = np.eye(8)[[1, 0, 2, 3, 4, 5, 6, 7]]  # one transposition flips the sign
    s2, la2 = pfaffian.slogpf(P @ A @ P.T)
    assert s2 == -s and la2 == pytest.approx(la)


def test_singular_and_odd():
    A = np.zeros((4, 4))
    s, la = pfaffian.slogpf(A)
    assert s == 0 and la == -np.inf
    s, la = pfaffian.slogpf(rand_skew(np.random.default_rng(0), 5))
    assert s == 0 and la == -np.inf


def test_batched_matches_single():
    rng = np.random.default_rng(5)
    A = rand_skew(rng, 24, batch=7)
    s, la = pfaffian.slogpf(A)
    for b in range(7):
        sb, lb = pfaffian.slogpf(A[b])
        assert s[b] == sb and la[b] == pytest.approx(lb, abs=1e-12)


@pytest.mark.parametrize("n,nb", [(6, 8), (56, 8), (100, 6), (224, 6), (224, 4)])
def test_panel_restatement_fp64(n, nb):
    """The CUDA kernel's blocked algorithm agrees with Parlett-Reid in FP64."""
    rng = np.random.default_rng(n * 7 + nb)
    A = rand_skew(rng, n)
    s0, l0 = pfaffian.slogpf(A)
    s1, l1 = pfaffian.slogpf_panel(A, nb)
    assert s1 == s0
    assert l1 == pytest.approx(l0, abs=1e-9)


def test_panel_restatement_fp32():
    rng = np.random.default_rng(9)
    A = rand_skew(rng, 56)
    s0, l0 = pfaffian.slogpf(A)
    s1, l1 = pfaffian.slogpf_panel(A.astype(np.float32), 8, np.float32)
    assert s1 == s0 and abs(l1 - l0) < 1e-3
