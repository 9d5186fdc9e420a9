"""Pfaffian backflow amplitude, FP64 oracle.

psi(s) = pf(F(s)) * fermion_inverse_sign(s) with the occupied pairing block
F[p, q] = sum_a Y[p, a] Wt[2 s_p + s_q, r(p, q), a] Y[q, a]
(``code/backflow/pf_kernel.py:1-11,156-166``; ``code/backflow/models.py:198-211``).

The backflow CNN is the one the graded configurations specify: 4 periodic 3x3 convolution
layers 2 -> C -> C -> C -> C (C = 32), tanh-approximated GELU after every layer but the last
(no final activation, as in ``models.py:325``), on the 2-channel +-1 occupation image
(channel 0 = up, channel 1 = down).  Output channels [0, d) are y_up and [d, 2d) are y_down,
d = C / 2 (``models.py:163-167``).
"""

from __future__ import annotations

import numpy as np

from . import lattice, pfaffian

GELU_C = np.sqrt(2.0 / np.pi)


def gelu_tanh(x):
    """tanh-approximated GELU (Hendrycks & Gimpel 2016), the default of jax.nn.gelu."""
    return 0.5 * x * (1.0 + np.tanh(GELU_C * (x + 0.044715 * x**3)))


def softplus(x):
    return np.log1p(np.exp(-abs(x))) + max(x, 0.0)


def build_wtilde(W: np.ndarray, theta: float, Lx: int, Ly: int, dtype=np.float64):
    """(3, N, d) raw parameters -> (4, N, d) table ``[uu, ud, du, dd]``
    (``code/backflow/pf_kernel.py:107-124``).

    uu/dd are antisymmetrised in r, du(r) = -ud(-r), times the envelope
    exp(-lam D_r) / (N sum_r exp(-lam D_r)) with lam = softplus(theta).  The blocks are
    formed in the dtype of W and the envelope in FP64 rounded once to ``dtype``, so the
    table satisfies Wt[2 sq + sp, -r] = -Wt[2 sp + sq, r] exactly.
    """
    _, neg, dist = lattice.displacement_tables(Lx, Ly)
    N = Lx * Ly
    W = np.asarray(W)
    w_ud = W[0]
    w_uu = (W[1] - W[1][neg]) / W.dtype.type(2)
    w_dd = (W[2] - W[2][neg]) / W.dtype.type(2)
    w_du = -w_ud[neg]
    lam = softplus(float(theta))
    pref = np.exp(-lam * dist)
    pref = (pref / (N * pref.sum())).astype(dtype)
    blocks = np.stack([w_uu, w_ud, w_du, w_dd]).astype(dtype)
    return blocks * pref[None, :, None]


def conv3x3_periodic(x: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    """x (B, Ci, Lx, Ly), w (Co, Ci, 3, 3), b (Co,) -> (B, Co, Lx, Ly); cross-correlation
    out[o, x, y] = b[o] + sum w[o, i, u, v] in[i, x + u - 1, y + v - 1] (periodic)."""
    out = np.broadcast_to(b[None, :, None, None], (x.shape[0], w.shape[0]) + x.shape[2:]).copy()
    for u in range(3):
        for v in range(3):
            xs = np.roll(x, shift=(1 - u, 1 - v), axis=(2, 3))
            out += np.einsum("oi,bixy->boxy", w[:, :, u, v], xs, optimize=True)
    return out


def input_image(s: np.ndarray, Lx: int, Ly: int) -> np.ndarray:
    """(B, 2N) int8 -> (B, 2, Lx, Ly) float +-1 image, channel 0 up, 1 down."""
    s = np.asarray(s)
    return s.reshape(s.shape[0], 2, Lx, Ly).astype(np.float64)


def cnn_forward(s: np.ndarray, conv_w, conv_b, Lx: int, Ly: int) -> np.ndarray:
    """Backflow features y (B, 2, N, d) of configurations s (B, 2N)."""
    x = input_image(s, Lx, Ly)
    nl = len(conv_w)
    for l in range(nl):
        x = conv3x3_periodic(x, np.asarray(conv_w[l], np.float64), np.asarray(conv_b[l], np.float64))
        if l < nl - 1:
            x = gelu_tanh(x)
    B, C = x.shape[:2]
    d = C // 2
    return np.swapaxes(x.reshape(B, 2, d, Lx * Ly), 2, 3)


def fermion_idx(s: np.ndarray) -> np.ndarray:
    """(B, 2N) -> (B, n) ascending occupied mode indices (all rows must have the same n)."""
    s = np.asarray(s)
    occ = s > 0
    n = int(occ[0].sum())
    idx = np.nonzero(occ)[1].reshape(s.shape[0], n)
    return idx


def fermion_inverse_sign(s: np.ndarray) -> np.ndarray:
    """(-1)^(k(k-1)/2) with k occupied modes: the reordering sign between ascending and
    descending products of creation operators.  (quantax 0.4.0's function of this name
    is not executable here; for every configured filling k(k-1)/2 is even.)"""
    k = (np.asarray(s) > 0).sum(-1)
    return np.where((k * (k - 1) // 2) % 2 == 0, 1.0, -1.0)


def pairing_occ(Y: np.ndarray, idx: np.ndarray, Wt: np.ndarray, Lx: int, Ly: int) -> np.ndarray:
    """F (B, n, n) = sum_a Y[p, a] Wt[2 s_p + s_q, r(p, q), a] Y[q, a]  (FP64), the
    formula of ``pairing_occ_reference`` (``pf_kernel.py:371-382``)."""
    disp, _, _ = lattice.displacement_tables(Lx, Ly)
    N = Lx * Ly
    sp, site = np.divmod(idx, N)
    B, n, d = Y.shape
    F = np.empty((B, n, n))
    for b in range(B):
        r = disp[site[b][:, None], site[b][None, :]]
        blk = 2 * sp[b][:, None] + sp[b][None, :]
        Wg = Wt[blk, r]  # (n, n, d)
        F[b] = np.einsum("pa,pqa,qa->pq", Y[b], Wg, Y[b], optimize=True)
    return F


def pairing_matrix_einsum(y: np.ndarray, W: np.ndarray, theta: float, Lx: int, Ly: int) -> np.ndarray:
    """The einsum twin: full antisymmetric (2N, 2N) pairing matrix of one configuration
    (``code/backflow/models.py:169-196``), FP64."""
    disp, neg, dist_r = lattice.displacement_tables(Lx, Ly)
    W = np.asarray(W, np.float64)
    w_ud = W[0]
    w_uu = (W[1] - W[1][neg]) / 2
    w_dd = (W[2] - W[2][neg]) / 2
    f_ud = np.einsum("ia,ija,ja->ij", y[0], w_ud[disp], y[1])
    f_uu = np.einsum("ia,ija,ja->ij", y[0], w_uu[disp], y[0])
    f_dd = np.einsum("ia,ija,ja->ij", y[1], w_dd[disp], y[1])
    lam = softplus(float(theta))
    pref = np.exp(-lam * dist_r[disp])
    pref = pref / pref.sum()
    f = np.block([[f_uu, f_ud], [-f_ud.T, f_dd]]) * np.tile(pref, (2, 2))
    return (f - f.T) / 2


def occupied_features(y: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Y (B, n, d) = y.reshape(B, 2N, d)[idx] (``pf_kernel.py:395``)."""
    B = y.shape[0]
    yf = y.reshape(B, -1, y.shape[-1])
    return np.take_along_axis(yf, idx[:, :, None], axis=1)


def amplitude(s: np.ndarray, params: dict, chunk: int = 64):
    """Unprojected (sign, logabs) of psi(s) for s (B, 2N), FP64.

    ``params``: dict with conv_w, conv_b (lists), W (3, N, d), theta, Lx, Ly; with
    ``net="resconv"`` also ``embed`` (C, 4), and conv_w / conv_b hold the residual blocks'
    convolutions (``oracle.resconv``).
    """
    Lx, Ly = params["Lx"], params["Ly"]
    Wt = build_wtilde(params["W"], params["theta"], Lx, Ly, np.float64)
    s = np.asarray(s)
    signs, logs = [], []
    for c0 in range(0, s.shape[0], chunk):
        sc = s[c0 : c0 + chunk]
        if params.get("net", "cnn") == "resconv":
            from .resconv import resconv_forward

            y = resconv_forward(sc, params["embed"], params["conv_w"], params["conv_b"], Lx, Ly)
        else:
            y = cnn_forward(sc, params["conv_w"], params["conv_b"], Lx, Ly)
        idx = fermion_idx(sc)
        Y = occupied_features(y, idx)
        F = pairing_occ(Y, idx, Wt, Lx, Ly)
        F = 0.5 * (F - np.swapaxes(F, 1, 2))
        sg, la = pfaffian.slogpf(F)
        signs.append(sg * fermion_inverse_sign(sc))
        logs.append(la)
    return np.concatenate(signs), np.concatenate(logs)
