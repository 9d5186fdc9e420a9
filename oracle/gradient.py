"""Gradient of log|psi| with respect to the backflow parameters, FP64 oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): the checker of the library's
per-sample Jacobian kernels, never the thing that is measured.

The reference trains with SR/AdamSR (``code/train_pfaffian_16x16_tpm02.py:100-101``), which
needs the per-sample derivatives O_k(s) = d log psi(s) / d theta_k.  JAX produces them by
differentiating ``PfaffianBackflow.__call__`` (``code/backflow/models.py:198-211``); this
module restates every link of that chain by hand:

* the Pfaffian adjoint (``fermix.slogpf``'s derivative, ``models.py:210``):
  d log|pf F| = 1/2 tr(F^{-1} dF), so G[p, q] = d log|pf F| / dF[p, q] = 1/2 (F^{-1})[q, p];
* the custom VJP of the occupied gather (``code/backflow/pf_kernel.py:193-320,354-365``):
  dY[p, a] = sum_q (G - G^T)[p, q] Wt[blk(p, q), r(p, q), a] Y[q, a] and
  dWt[blk, r, a] = sum over the pairs (p, q) with that block and displacement of
  G[p, q] Y[p, a] Y[q, a];
* the backward of ``build_wtilde`` (``pf_kernel.py:107-124``): the block
  antisymmetrisation and the softplus distance envelope;
* the backward of the backflow CNN (periodic 3x3 cross-correlations with tanh-GELU between
  layers, the graded configuration's network) and of the feature gather
  ``y.reshape(2N, d)[idx]`` (``pf_kernel.py:395``);
* the symmetry projection: d log|psi_P| = sum_g w_g d log|psi(g s)| with
  w_g = eta_g psi(g s) / sum_h eta_h psi(h s).

Parameters are flattened in the order conv_w[0] (OIHW), conv_b[0], ..., conv_w[L-1],
conv_b[L-1], W (3, N, d), theta: the column order of the library's Jacobian.
"""

from __future__ import annotations

import numpy as np

from . import backflow, lattice, pfaffian, projection


def param_count(params: dict) -> int:
    n = sum(np.size(w) + np.size(b) for w, b in zip(params["conv_w"], params["conv_b"]))
    return int(n + np.size(params["W"]) + 1)


def flatten_params(params: dict) -> np.ndarray:
    parts = []
    for w, b in zip(params["conv_w"], params["conv_b"]):
        parts += [np.ravel(w), np.ravel(b)]
    parts += [np.ravel(params["W"]), np.atleast_1d(np.float64(params["theta"]))]
    return np.concatenate([np.asarray(p, np.float64) for p in parts])


def unflatten_params(vec: np.ndarray, like: dict) -> dict:
    out = dict(like)
    off = 0
    conv_w, conv_b = [], []
    for w, b in zip(like["conv_w"], like["conv_b"]):
        conv_w.append(vec[off : off + np.size(w)].reshape(np.shape(w)))
        off += np.size(w)
        conv_b.append(vec[off : off + np.size(b)].reshape(np.shape(b)))
        off += np.size(b)
    out["conv_w"], out["conv_b"] = conv_w, conv_b
    out["W"] = vec[off : off + np.size(like["W"])].reshape(np.shape(like["W"]))
    off += np.size(like["W"])
    out["theta"] = float(vec[off])
    return out


def slogpf_adjoint(F: np.ndarray) -> np.ndarray:
    """G = d log|pf F| / dF = 1/2 F^{-T} for antisymmetric F (..., n, n)."""
    return 0.5 * np.swapaxes(np.linalg.inv(np.asarray(F, np.float64)), -1, -2)


def pairing_occ_vjp(Y: np.ndarray, idx: np.ndarray, Wt: np.ndarray, G: np.ndarray, Lx: int,
                    Ly: int):
    """Cotangents (dY (B, n, d), dWt (B, 4, N, d)) of F = pairing_occ(Y, idx, Wt) for the
    output cotangent G (B, n, n): ``_pairing_occ_bwd`` (``pf_kernel.py:354-365``) per item."""
    disp, _, _ = lattice.displacement_tables(Lx, Ly)
    N = Lx * Ly
    B, n, d = Y.shape
    dY = np.empty((B, n, d))
    dWt = np.zeros((B, 4, N, d))
    for b in range(B):
        sp, site = np.divmod(idx[b], N)
        r = disp[site[:, None], site[None, :]]
        blk = 2 * sp[:, None] + sp[None, :]
        Wg = Wt[blk, r]  # (n, n, d)
        Gb = np.asarray(G[b], np.float64)
        dY[b] = np.einsum("pq,pqa,qa->pa", Gb - Gb.T, Wg, Y[b], optimize=True)
        contrib = Gb[:, :, None] * Y[b][:, None, :] * Y[b][None, :, :]
        np.add.at(dWt[b], (blk, r), contrib)
    return dY, dWt


def build_wtilde_vjp(W: np.ndarray, theta: float, dWt: np.ndarray, Lx: int, Ly: int):
    """Cotangents (dW (..., 3, N, d), dtheta (...)) of Wt = build_wtilde(W, theta) for dWt
    (..., 4, N, d)."""
    _, neg, dist = lattice.displacement_tables(Lx, Ly)
    N = Lx * Ly
    W = np.asarray(W, np.float64)
    lam = backflow.softplus(float(theta))
    e = np.exp(-lam * dist)
    pref = e / (N * e.sum())
    D = dWt * pref[:, None]  # cotangent of the blocks before the envelope
    dW = np.empty(dWt.shape[:-3] + (3, N, W.shape[-1]))
    dW[..., 0, :, :] = D[..., 1, :, :] - D[..., 2, neg, :]
    dW[..., 1, :, :] = 0.5 * (D[..., 0, :, :] - D[..., 0, neg, :])
    dW[..., 2, :, :] = 0.5 * (D[..., 3, :, :] - D[..., 3, neg, :])
    blocks = np.stack([(W[1] - W[1][neg]) / 2, W[0], -W[0][neg], (W[2] - W[2][neg]) / 2])
    dpref = np.einsum("...bra->...r", dWt * blocks)
    mean_d = float((dist * e).sum() / e.sum())
    dlam = np.sum(dpref * pref * (mean_d - dist), axis=-1)
    sig = 1.0 / (1.0 + np.exp(-float(theta)))
    return dW, dlam * sig


def gelu_tanh_grad(x):
    k = backflow.GELU_C
    t = np.tanh(k * (x + 0.044715 * x**3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * k * (1.0 + 3 * 0.044715 * x * x)


def cnn_vjp(s: np.ndarray, conv_w, conv_b, Lx: int, Ly: int, dy: np.ndarray):
    """Per-configuration cotangents (dconv_w list of (B, Co, Ci, 3, 3), dconv_b list of
    (B, Co)) of the backflow features y = cnn_forward(s) (B, 2, N, d) for dy."""
    x = backflow.input_image(s, Lx, Ly)
    nl = len(conv_w)
    ins, zs = [], []
    for l in range(nl):
        ins.append(x)
        z = backflow.conv3x3_periodic(x, np.asarray(conv_w[l], np.float64),
                                      np.asarray(conv_b[l], np.float64))
        zs.append(z)
        x = backflow.gelu_tanh(z) if l < nl - 1 else z
    B, C = x.shape[:2]
    d = C // 2
    delta = np.swapaxes(dy, 2, 3).reshape(B, C, Lx, Ly)
    dws, dbs = [None] * nl, [None] * nl
    for l in range(nl - 1, -1, -1):
        w = np.asarray(conv_w[l], np.float64)
        a = ins[l]
        dw = np.empty((B,) + w.shape)
        for u in range(3):
            for v in range(3):
                xs = np.roll(a, shift=(1 - u, 1 - v), axis=(2, 3))
                dw[:, :, :, u, v] = np.einsum("boxy,bixy->boi", delta, xs, optimize=True)
        dws[l] = dw
        dbs[l] = delta.sum((2, 3))
        if l > 0:
            dx = np.zeros_like(a)
            for u in range(3):
                for v in range(3):
                    t = np.einsum("oi,boxy->bixy", w[:, :, u, v], delta, optimize=True)
                    dx += np.roll(t, shift=(u - 1, v - 1), axis=(2, 3))
            delta = dx * gelu_tanh_grad(zs[l - 1])
    return dws, dbs


def image_log_grad(s: np.ndarray, params: dict):
    """Unprojected (sign, logabs, J (B, P)) with J = d log|psi(s)| / d theta, FP64."""
    Lx, Ly = params["Lx"], params["Ly"]
    N = Lx * Ly
    s = np.asarray(s)
    Wt = backflow.build_wtilde(params["W"], params["theta"], Lx, Ly, np.float64)
    y = backflow.cnn_forward(s, params["conv_w"], params["conv_b"], Lx, Ly)
    idx = backflow.fermion_idx(s)
    Y = backflow.occupied_features(y, idx)
    F = backflow.pairing_occ(Y, idx, Wt, Lx, Ly)
    F = 0.5 * (F - np.swapaxes(F, 1, 2))
    sg, la = pfaffian.slogpf(F)
    G = slogpf_adjoint(F)
    dY, dWt = pairing_occ_vjp(Y, idx, Wt, G, Lx, Ly)
    B, n, d = Y.shape
    dyf = np.zeros((B, 2 * N, d))
    np.put_along_axis(dyf, idx[:, :, None], dY, axis=1)
    dws, dbs = cnn_vjp(s, params["conv_w"], params["conv_b"], Lx, Ly, dyf.reshape(B, 2, N, d))
    dW, dth = build_wtilde_vjp(params["W"], params["theta"], dWt, Lx, Ly)
    parts = []
    for dw, db in zip(dws, dbs):
        parts += [dw.reshape(B, -1), db.reshape(B, -1)]
    parts += [dW.reshape(B, -1), np.asarray(dth).reshape(B, 1)]
    return sg * backflow.fermion_inverse_sign(s), la, np.concatenate(parts, axis=1)


def log_jacobian(s: np.ndarray, params: dict, symm: bool = True, chunk: int = 16):
    """(sign, logabs, J (B, P)) of psi_P(s) (psi(s) when ``symm`` is False), with
    J[b, k] = d log|psi_P(s_b)| / d theta_k in the flattened parameter order."""
    s = np.asarray(s)
    Lx, Ly = params["Lx"], params["Ly"]
    out_s, out_l, out_j = [], [], []
    for c0 in range(0, s.shape[0], chunk):
        sc = s[c0 : c0 + chunk]
        if not symm:
            sg, la, J = image_log_grad(sc, params)
        else:
            maps = lattice.symmetry_mode_maps(Lx, Ly)
            G = maps.shape[0]
            imgs = projection.image_configs(sc, maps).reshape(-1, sc.shape[1])
            eta = projection.image_signs(sc, maps)
            sgi, lai, Ji = image_log_grad(imgs, params)
            sgi = sgi.reshape(-1, G) * eta
            lai = lai.reshape(-1, G)
            sg, lt = projection.signed_logsumexp(sgi, lai, axis=1)
            w = sgi * np.exp(lai - lt[:, None]) * sg[:, None]  # eta_g psi_g / sum_h eta_h psi_h
            J = np.einsum("bg,bgk->bk", w, Ji.reshape(sc.shape[0], G, -1))
            la = lt - np.log(G)
        out_s.append(sg)
        out_l.append(la)
        out_j.append(J)
    return np.concatenate(out_s), np.concatenate(out_l), np.concatenate(out_j)
