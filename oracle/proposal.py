"""Learned hop proposal, FP64 oracle (test infrastructure only).

The reference samples with quantax's uniform ParticleHop (``code/states.py:397-408``); the
learned proposal has no counterpart there.  This module restates the network, the masked
softmax over moves, the training loss with its hand-derived gradient, and the exact
Metropolis-Hastings acceptance, so that the CUDA kernels can be checked against it.

Network: periodic 3x3 CNN 2 -> 16 -> 16 -> 16 on the +-1 occupation image (channel 0 up,
1 down), tanh-GELU after layers 1 and 2, none after layer 3 (the same convolution convention
as ``backflow.conv3x3_periodic``).  Output channel c = sigma * 8 + d at site i is the logit of
moving the spin-sigma electron at site i one hop in direction d (``lattice.HOP_DIRS`` order).
Move index m = c * N + i.  A move is valid when that electron exists, d < n_dirs, and the target
site of the same spin is empty; q(m | s) is the softmax of the logits over the valid moves.

Parameters, one flat vector of PARAM_COUNT values: W1 (16, 2, 3, 3), b1 (16), W2 (16, 16, 3, 3),
b2 (16), W3 (16, 16, 3, 3), b3 (16).

Training records (s_b, m_b, w_b): a configuration from plain-sampler chains, a move drawn
uniformly among its valid moves and the weight w_b = min(1, |psi(s')/psi(s)|^2).  The loss
L = -(1/B) sum_b w_b log q(m_b | s_b) is minimised by q(m | s) proportional to
min(1, |psi(s_m)/psi(s)|^2), i.e. a proposal that offers moves in proportion to their
Metropolis acceptance.  Gradient: dL/dz = (w_b / B) (q - onehot(m_b)) on valid entries.

Acceptance with reverse probability: a move s -> s' is accepted when
log u < 2 (log|psi(s')| - log|psi(s)|) + log q(m' | s') - log q(m | s), m' the reverse hop
(same spin, from the target site back in the opposite direction).
"""

from __future__ import annotations

import numpy as np

from . import lattice
from .backflow import GELU_C, conv3x3_periodic, gelu_tanh, input_image

CH = 16
N_OUT = 16
SHAPES = [(CH, 2, 3, 3), (CH,), (CH, CH, 3, 3), (CH,), (N_OUT, CH, 3, 3), (N_OUT,)]
PARAM_COUNT = int(sum(np.prod(s) for s in SHAPES))
# Opposite hop direction of each direction in lattice.HOP_DIRS order.
OPPOSITE = np.array([1, 0, 3, 2, 7, 6, 5, 4])


def init_params(seed: int = 0, std: float = 0.05) -> np.ndarray:
    """Seeded N(0, std) weights and zero biases, FP32."""
    rng = np.random.default_rng(seed)
    parts = []
    for shp in SHAPES:
        parts.append(rng.normal(0.0, std, size=shp).ravel() if len(shp) > 1 else np.zeros(shp))
    return np.concatenate(parts).astype(np.float32)


def round_bf16(x: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 (round to nearest even) -> FP32, the weights the CUDA kernels evaluate."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def unpack(theta: np.ndarray):
    theta = np.asarray(theta, np.float64)
    out, o = [], 0
    for shp in SHAPES:
        k = int(np.prod(shp))
        out.append(theta[o : o + k].reshape(shp))
        o += k
    return out


def gelu_grad(x):
    t = np.tanh(GELU_C * (x + 0.044715 * x**3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C * (1.0 + 3 * 0.044715 * x * x)


def _forward(s, theta, Lx, Ly):
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    x0 = input_image(s, Lx, Ly)
    h1 = conv3x3_periodic(x0, W1, b1)
    a1 = gelu_tanh(h1)
    h2 = conv3x3_periodic(a1, W2, b2)
    a2 = gelu_tanh(h2)
    z = conv3x3_periodic(a2, W3, b3)
    return x0, h1, a1, h2, a2, z


def logits(s, theta, Lx: int, Ly: int) -> np.ndarray:
    """(B, 2N) int8 -> (B, 16, N) logits."""
    z = _forward(s, theta, Lx, Ly)[-1]
    return z.reshape(z.shape[0], N_OUT, Lx * Ly)


def valid_mask(s, Lx: int, Ly: int, n_dirs: int = 8) -> np.ndarray:
    """(B, 16, N) bool: electron present, direction in use, target of the same spin empty."""
    s = np.asarray(s)
    N = Lx * Ly
    nbr = lattice.neighbour_table(Lx, Ly)  # (N, 8)
    occ = s.reshape(-1, 2, N) > 0
    m = np.zeros((s.shape[0], 2, 8, N), bool)
    for d in range(n_dirs):
        m[:, :, d, :] = occ & ~occ[:, :, nbr[:, d]]
    return m.reshape(-1, N_OUT, N)


def log_q(s, theta, Lx: int, Ly: int, n_dirs: int = 8) -> np.ndarray:
    """(B, 16 N) log-probabilities of the moves (-inf where invalid), m = c N + i."""
    z = logits(s, theta, Lx, Ly).reshape(len(s), -1)
    v = valid_mask(s, Lx, Ly, n_dirs).reshape(len(s), -1)
    zm = np.where(v, z, -np.inf)
    mx = zm.max(1, keepdims=True)
    lse = mx + np.log(np.exp(zm - mx).sum(1, keepdims=True))
    return zm - lse


def apply_move(s, m, Lx: int, Ly: int):
    """Configurations after move m (B,): returns (s', from_mode, to_mode)."""
    s = np.array(s, copy=True)
    N = Lx * Ly
    nbr = lattice.neighbour_table(Lx, Ly)
    m = np.asarray(m, np.int64)
    c, i = m // N, m % N
    sigma, d = c // 8, c % 8
    fr = sigma * N + i
    to = sigma * N + nbr[i, d]
    rows = np.arange(len(s))
    s[rows, fr] = -1
    s[rows, to] = 1
    return s, fr, to


def reverse_move(m, Lx: int, Ly: int):
    N = Lx * Ly
    nbr = lattice.neighbour_table(Lx, Ly)
    m = np.asarray(m, np.int64)
    c, i = m // N, m % N
    sigma, d = c // 8, c % 8
    return (sigma * 8 + OPPOSITE[d]) * N + nbr[i, d]


def select_move(logq_row: np.ndarray, u: float) -> int:
    """Inverse-CDF selection in ascending move order: the first m with CDF(m) > u."""
    p = np.exp(logq_row)
    cdf = np.cumsum(p)
    return int(min(np.searchsorted(cdf, u * cdf[-1], side="right"), len(p) - 1))


def loss_and_grad(s, moves, weights, theta, Lx: int, Ly: int, n_dirs: int = 8):
    """L = -(1/B) sum_b w_b log q(m_b | s_b) and dL/dtheta (flat), FP64, by hand-derived
    backpropagation through the masked softmax and the three periodic convolutions."""
    s = np.asarray(s)
    B = s.shape[0]
    N = Lx * Ly
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    x0, h1, a1, h2, a2, z = _forward(s, theta, Lx, Ly)
    lq = log_q(s, theta, Lx, Ly, n_dirs)
    w = np.asarray(weights, np.float64)
    mv = np.asarray(moves, np.int64)
    picked = lq[np.arange(B), mv]
    loss = -(w * picked).sum() / B
    q = np.exp(lq)  # zero where invalid
    dz = q * (w / B)[:, None]
    dz[np.arange(B), mv] -= w / B
    dz = dz.reshape(B, N_OUT, Lx, Ly)

    def conv_back(dout, xin, Wt):
        dW = np.zeros_like(Wt)
        din = np.zeros_like(xin)
        for u in range(3):
            for v in range(3):
                xs = np.roll(xin, shift=(1 - u, 1 - v), axis=(2, 3))
                dW[:, :, u, v] = np.einsum("boxy,bixy->oi", dout, xs, optimize=True)
                ds = np.roll(dout, shift=(u - 1, v - 1), axis=(2, 3))
                din += np.einsum("oi,boxy->bixy", Wt[:, :, u, v], ds, optimize=True)
        return dW, dout.sum((0, 2, 3)), din

    dW3, db3, da2 = conv_back(dz, a2, W3)
    dh2 = da2 * gelu_grad(h2)
    dW2, db2, da1 = conv_back(dh2, a1, W2)
    dh1 = da1 * gelu_grad(h1)
    dW1, db1, _ = conv_back(dh1, x0, W1)
    grad = np.concatenate([g.ravel() for g in (dW1, db1, dW2, db2, dW3, db3)])
    return float(loss), grad


def adam_step(theta, m, v, grad, t: int, lr: float, b1: float = 0.9, b2: float = 0.999,
              eps: float = 1e-8):
    """One Adam update (Kingma & Ba 2015) with bias correction; returns (theta, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1**t)
    vh = v / (1 - b2**t)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v
