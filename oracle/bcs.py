"""BCS-backflow amplitude, FP64 oracle (TEST INFRASTRUCTURE ONLY, see ``oracle/__init__.py``).

``code/backflow/models.py:214-302`` (``BCSBackflow``) and ``code/backflow/bcs_kernel.py:1-70``:

    F[p, q] = sum_a Yu[p, a] Wt_ud[site_p - site_q, a] Yd[q, a] + delta_d fd[site_p, site_q]
    psi(s)  = det(F) (-1)^(n_up (n_up - 1) / 2) fermion_inverse_sign(s)

for the occupied up modes p and down modes q, with Wt_ud = W (N, d) times the distance envelope
exp(-lam D_r) / (N sum_r exp(-lam D_r)) (``bcs_kernel.py:61-69``) and fd the nearest-neighbour
d-wave form factor, -1 on x bonds and +1 on y bonds (``models.py:80-82``).  The features are the
two spin halves of the backflow network's output, as for the Pfaffian state.

The same amplitude is the Pfaffian of the antisymmetric 2n x 2n matrix [[0, F], [-F^T, 0]]
(pf = (-1)^(n (n - 1) / 2) det F), i.e. the Pfaffian state whose same-spin blocks vanish;
``as_pfaffian_params`` builds those parameters so that the two oracles check each other.
"""

from __future__ import annotations

import numpy as np

from . import backflow, lattice, projection


def dwave_factor(Lx: int, Ly: int) -> np.ndarray:
    """(N,) fd as a function of the displacement r: -1 for |dx| = 1, dy = 0; +1 for dx = 0,
    |dy| = 1 (minimum image), else 0."""
    x, y = lattice.site_xy(Lx, Ly)
    mx = np.minimum(x, Lx - x)
    my = np.minimum(y, Ly - y)
    fd = np.zeros(Lx * Ly)
    fd[(mx == 1) & (my == 0)] = -1.0
    fd[(mx == 0) & (my == 1)] = 1.0
    return fd


def wt_ud(W: np.ndarray, theta: float, Lx: int, Ly: int) -> np.ndarray:
    """(N, d) W times the distance envelope (``bcs_kernel.build_wt_ud``), FP64."""
    _, _, dist = lattice.displacement_tables(Lx, Ly)
    lam = backflow.softplus(float(theta))
    pref = np.exp(-lam * dist)
    pref = pref / (Lx * Ly * pref.sum())
    return np.asarray(W, np.float64) * pref[:, None]


def occupied_block(Yu, iu, Yd, idn, Wud, delta_d, Lx, Ly):
    """F (B, n_up, n_dn) of ``BCSBackflow.occupied_block``; iu, idn are site indices."""
    disp, _, _ = lattice.displacement_tables(Lx, Ly)
    fd = dwave_factor(Lx, Ly)
    B = Yu.shape[0]
    F = np.empty((B, iu.shape[1], idn.shape[1]))
    for b in range(B):
        r = disp[iu[b][:, None], idn[b][None, :]]
        F[b] = np.einsum("pa,pqa,qa->pq", Yu[b], Wud[r], Yd[b], optimize=True) + delta_d * fd[r]
    return F


def amplitude(s: np.ndarray, params: dict, chunk: int = 64):
    """Unprojected (sign, logabs) of the BCS-backflow state, FP64.  ``params`` as for
    ``backflow.amplitude`` with W of shape (N, d) and ``delta_d``."""
    Lx, Ly = params["Lx"], params["Ly"]
    N = Lx * Ly
    Wud = wt_ud(params["W"], params["theta"], Lx, Ly)
    s = np.asarray(s)
    signs, logs = [], []
    for c0 in range(0, s.shape[0], chunk):
        sc = s[c0 : c0 + chunk]
        if params.get("net", "cnn") == "resconv":
            from .resconv import resconv_forward

            y = resconv_forward(sc, params["embed"], params["conv_w"], params["conv_b"], Lx, Ly)
        else:
            y = backflow.cnn_forward(sc, params["conv_w"], params["conv_b"], Lx, Ly)
        occ = sc > 0
        n_up = int(occ[0, :N].sum())
        iu = np.nonzero(occ[:, :N])[1].reshape(sc.shape[0], n_up)
        idn = np.nonzero(occ[:, N:])[1].reshape(sc.shape[0], -1)
        Yu = np.take_along_axis(y[:, 0], iu[:, :, None], axis=1)
        Yd = np.take_along_axis(y[:, 1], idn[:, :, None], axis=1)
        F = occupied_block(Yu, iu, Yd, idn, Wud, float(params["delta_d"]), Lx, Ly)
        sg, la = np.linalg.slogdet(F)
        sg = sg * (-1.0) ** (n_up * (n_up - 1) // 2) * backflow.fermion_inverse_sign(sc)
        signs.append(sg)
        logs.append(la)
    return np.concatenate(signs), np.concatenate(logs)


def projected_amplitude(s: np.ndarray, params: dict, symm: bool = True):
    """(sign, logabs) of the projected BCS state (of psi(s) when ``symm`` is False), with the
    images and signs of ``projection.projected_amplitude``."""
    s = np.asarray(s)
    if not symm:
        return amplitude(s, params)
    Lx, Ly = params["Lx"], params["Ly"]
    maps = lattice.symmetry_mode_maps(Lx, Ly)
    G = maps.shape[0]
    imgs = projection.image_configs(s, maps)
    eta = projection.image_signs(s, maps)
    sg, la = amplitude(imgs.reshape(-1, s.shape[1]), params)
    sgn, lab = projection.signed_logsumexp(sg.reshape(-1, G) * eta, la.reshape(-1, G), axis=1)
    return sgn, lab - np.log(G)


def as_pfaffian_params(params: dict) -> dict:
    """Pfaffian-state parameters with the same amplitude when delta_d = 0: W (3, N, d) =
    [W_ud, 0, 0] (vanishing same-spin blocks)."""
    W = np.asarray(params["W"], np.float64)
    out = dict(params)
    out["W"] = np.stack([W, np.zeros_like(W), np.zeros_like(W)])
    out.pop("delta_d", None)
    return out
