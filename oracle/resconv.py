"""Residual backflow CNN of the released Pfaffian-backflow states, FP64 oracle (test
infrastructure only).

The reference builds it at ``code/backflow/models.py:319-329`` as quantax's ``ResConv``
(16 blocks, 64 channels, 3x3 kernels, RMSNorm, final bias, identity final activation, no
translation symmetrisation).  quantax 0.4.0 is not part of the reference tree and cannot run
here, so the network is restated from its published description
(``data/supplement/tableS1_network/network_settings.json:21-56``, the "normal" block):

    x_0[c, i] = E[c, occ(i)]            learned C-vector per site occupation
                                        (empty, up, down, double): occ = n_up + 2 n_dn
    x_{b+1}   = x_b + Conv2(GELU(Conv1(GELU(RMSNorm(x_b)))))      b = 0 .. blocks - 1
    y         = x_blocks / sqrt(blocks + 1)

Convolutions are 3x3 periodic cross-correlations with bias (``conv3x3_periodic``); RMSNorm
divides by the root mean square over all channels and sites, without affine parameters
(``RMS_EPS`` inside the root); GELU is the tanh form (the default of ``jax.nn.gelu``).
Features: channels [0, d) spin up, [d, 2d) spin down, d = C / 2 (``models.py:163-167``).
"""

from __future__ import annotations

import numpy as np

from .backflow import conv3x3_periodic, gelu_tanh

RMS_EPS = 1e-6


def occupation_index(s: np.ndarray, Lx: int, Ly: int) -> np.ndarray:
    """(B, 2N) +-1 -> (B, Lx, Ly) occupation index n_up + 2 n_dn in {0, 1, 2, 3}."""
    s = np.asarray(s)
    N = Lx * Ly
    up = (s[:, :N] > 0).astype(np.int64)
    dn = (s[:, N:] > 0).astype(np.int64)
    return (up + 2 * dn).reshape(-1, Lx, Ly)


def rms_norm(x: np.ndarray, eps: float = RMS_EPS) -> np.ndarray:
    """x (B, C, Lx, Ly) / sqrt(mean over (C, Lx, Ly) of x^2 + eps)."""
    ms = np.mean(x * x, axis=(1, 2, 3), keepdims=True)
    return x / np.sqrt(ms + eps)


def resconv_forward(s: np.ndarray, embed, conv_w, conv_b, Lx: int, Ly: int,
                    eps: float = RMS_EPS) -> np.ndarray:
    """Features y (B, 2, N, d) of configurations s (B, 2N).

    ``embed`` (C, 4); ``conv_w`` 2 * blocks arrays (C, C, 3, 3) in block order (first, second
    convolution of each block); ``conv_b`` the matching (C,) biases."""
    E = np.asarray(embed, np.float64)
    occ = occupation_index(s, Lx, Ly)
    x = np.moveaxis(E[:, occ], 0, 1)  # (B, C, Lx, Ly)
    blocks = len(conv_w) // 2
    for b in range(blocks):
        h = gelu_tanh(rms_norm(x, eps))
        h = gelu_tanh(conv3x3_periodic(h, np.asarray(conv_w[2 * b], np.float64),
                                       np.asarray(conv_b[2 * b], np.float64)))
        x = x + conv3x3_periodic(h, np.asarray(conv_w[2 * b + 1], np.float64),
                                 np.asarray(conv_b[2 * b + 1], np.float64))
    x = x / np.sqrt(blocks + 1.0)
    B, C = x.shape[:2]
    d = C // 2
    return np.swapaxes(x.reshape(B, 2, d, Lx * Ly), 2, 3)
