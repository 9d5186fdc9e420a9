"""Batched FP64 log-Pfaffian (oracle).

``slogpf`` is the Parlett-Reid skew-symmetric LTL^T reduction with partial pivoting, the
published algorithm of M. Wimmer, "Efficient numerical computation of the Pfaffian for dense
and banded skew-symmetric matrices", ACM TOMS 38, 30 (2012).  It stands in for
``fermix.slogpf`` (called at ``code/backflow/models.py:210``; fermix 0.1.0 is a third-party
package that is not part of the reference tree), which returns (sign, log|pf|).

``slogpf_panel`` restates, step for step, the blocked algorithm of the CUDA kernel (lazy
panel columns, row pivoting by index relabelling, compaction plus rank-2k trailing update at
the end of each panel) so that its arithmetic can be checked in FP64 and FP32 on the CPU.
"""

from __future__ import annotations

import itertools

import numpy as np


def slogpf(A: np.ndarray):
    """(sign, logabs) of pf(A) for antisymmetric A of shape (..., n, n), in FP64.

    Step k (even) pivots the largest |A[i, k]|, i > k, into row/column k + 1 (a sign flip
    when it moves), multiplies the Pfaffian by A[k, k+1] and applies the rank-2 Gauss
    update A[k+2:, k+2:] += tau a^T - a tau^T with tau = A[k, k+2:] / A[k, k+1] and
    a = A[k+2:, k+1].  A zero pivot gives sign 0 and logabs -inf.
    """
    A = np.array(A, dtype=np.float64, copy=True)
    batch_shape = A.shape[:-2]
    n = A.shape[-1]
    A = A.reshape(-1, n, n)
    B = A.shape[0]
    sign = np.ones(B)
    logabs = np.zeros(B)
    if n % 2:
        return np.zeros(batch_shape), np.full(batch_shape, -np.inf)
    ar = np.arange(B)
    for k in range(0, n - 1, 2):
        kp = k + 1 + np.argmax(np.abs(A[:, k + 1 :, k]), axis=1)
        moved = kp != k + 1
        if moved.any():
            r1 = A[ar, k + 1, :].copy()
            A[ar, k + 1, :] = A[ar, kp, :]
            A[ar, kp, :] = r1
            c1 = A[ar, :, k + 1].copy()
            A[ar, :, k + 1] = A[ar, :, kp]
            A[ar, :, kp] = c1
            sign[moved] *= -1.0
        piv = A[:, k, k + 1].copy()
        zero = piv == 0.0
        sign *= np.sign(piv)
        with np.errstate(divide="ignore"):
            logabs += np.log(np.abs(piv))
        if k + 2 < n:
            piv[zero] = 1.0
            tau = A[:, k, k + 2 :] / piv[:, None]
            a = A[:, k + 2 :, k + 1]
            A[:, k + 2 :, k + 2 :] += tau[:, :, None] * a[:, None, :] - a[:, :, None] * tau[:, None, :]
    logabs[sign == 0] = -np.inf
    return sign.reshape(batch_shape), logabs.reshape(batch_shape)


def pf_bruteforce(A: np.ndarray) -> float:
    """Pfaffian by expansion along the first row (tiny n only; known-answer tests)."""
    n = A.shape[0]
    if n == 0:
        return 1.0
    if n % 2:
        return 0.0
    total = 0.0
    for j in range(1, n):
        rest = [i for i in range(1, n) if i != j]
        total += (-1) ** (j + 1) * A[0, j] * pf_bruteforce(A[np.ix_(rest, rest)])
    return total


def pf_permutation_sum(A: np.ndarray) -> float:
    """Pfaffian from its definition as a sum over perfect matchings (n <= 8)."""
    n = A.shape[0]
    total = 0.0
    for perm in itertools.permutations(range(n)):
        ok = all(perm[2 * i] < perm[2 * i + 1] for i in range(n // 2)) and all(
            perm[2 * i] < perm[2 * i + 2] for i in range(n // 2 - 1)
        )
        if not ok:
            continue
        inv = sum(1 for i in range(n) for j in range(i + 1, n) if perm[i] > perm[j])
        term = float((-1) ** inv)
        for i in range(n // 2):
            term *= A[perm[2 * i], perm[2 * i + 1]]
        total += term
    return total


def _col(L: np.ndarray, c: int) -> np.ndarray:
    """Column c of the antisymmetric matrix whose strict lower triangle is L."""
    n = L.shape[0]
    out = np.zeros(n, dtype=L.dtype)
    out[c + 1 :] = L[c + 1 :, c]
    out[:c] = -L[c, :c]
    return out


def slogpf_panel(A: np.ndarray, nb: int = 8, dtype=np.float64):
    """The CUDA kernel's blocked Parlett-Reid, restated for one matrix.

    The strict lower triangle is stored; within a panel of ``nb`` steps a pivot only
    relabels indices (``log_of`` / ``phys_of``), panel columns are formed lazily from
    the stored column plus the panel's rank-2 terms, and at the end of the panel the
    trailing triangle is relabelled (compacted) and updated with U V^T - V U^T.
    The pivot product is accumulated in FP64 mantissa/exponent form.
    """
    A = np.asarray(A)
    n = A.shape[0]
    if n % 2:
        return 0.0, -np.inf
    L = np.tril(A, -1).astype(dtype)
    sign = 1.0
    mant, expo = 1.0, 0
    k0 = 0
    while k0 < n - 1:
        steps = min(nb, (n - k0) // 2)
        log_of = np.arange(n)
        phys_of = np.arange(n)
        U = np.zeros((n, steps), dtype=dtype)
        V = np.zeros((n, steps), dtype=dtype)
        for j in range(steps):
            k = k0 + 2 * j
            ck = phys_of[k]
            col = _col(L, ck) + U[:, :j] @ V[ck, :j] - V[:, :j] @ U[ck, :j]
            cand = np.where(log_of > k, np.abs(col), -1.0)
            r = int(np.argmax(cand))
            lr, p1 = int(log_of[r]), int(phys_of[k + 1])
            if lr != k + 1:
                sign = -sign
            log_of[r], log_of[p1] = k + 1, lr
            phys_of[k + 1], phys_of[lr] = r, p1
            piv = -col[r]
            if piv == 0:
                return 0.0, -np.inf
            sign *= np.sign(piv)
            mant, e = np.frexp(mant * abs(float(piv)))
            expo += int(e)
            d = _col(L, r) + U[:, :j] @ V[r, :j] - V[:, :j] @ U[r, :j]
            live = log_of > k + 1
            U[:, j] = np.where(live, d, 0)
            V[:, j] = np.where(live, col / piv, 0)
        k_end = k0 + 2 * steps
        m = n - k_end
        if m > 1:
            idx = phys_of[k_end:]
            full = np.zeros((n, n), dtype=dtype)
            full += L
            full -= L.T
            T = full[np.ix_(idx, idx)]
            Ui, Vi = U[idx], V[idx]
            T = T + Ui @ Vi.T - Vi @ Ui.T
            L[k_end:, k_end:] = np.tril(T, -1)
        k0 = k_end
    return sign, float(np.log(mant) + expo * np.log(2.0))
