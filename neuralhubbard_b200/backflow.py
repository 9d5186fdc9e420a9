"""Pfaffian backflow model and its operators on the GPU (host side of the C ABI).

Mirrors the reference's operator surface:

* ``PairGeometry``        <- ``code/backflow/pf_kernel.py:58-77``
* ``build_wtilde``        <- ``code/backflow/pf_kernel.py:107-124``
* ``pairing_occ``         <- ``code/backflow/pf_kernel.py:335-351`` (forward only)
* ``slogpf``              <- ``fermix.slogpf`` as called at ``code/backflow/models.py:210``
* ``slogpf_adjoint``      <- the derivative of ``fermix.slogpf`` (d log|pf F| / dF)
* ``pairing_occ_vjp``     <- the custom VJP of ``pairing_occ`` (``pf_kernel.py:193-320,354-365``)
* ``PfaffianBackflow``    <- ``code/backflow/models.py:121-211`` with the backflow CNN of the
                             graded configurations (4 periodic 3x3 layers, 32 channels,
                             tanh-GELU between layers, 2-channel +-1 input).

Every computation runs in libnh_b200.so; tensors are torch CUDA tensors used for device memory
and streams only.
"""

from __future__ import annotations

import ctypes
from typing import NamedTuple, Optional

import numpy as np
import torch

from . import _lib


class PairGeometry(NamedTuple):
    """Static description of the pairing problem (``pf_kernel.py:58-77``)."""

    LX: int
    LY: int
    d: int
    n_up: int
    n_dn: int

    @property
    def N(self) -> int:
        return self.LX * self.LY

    @property
    def n_occ(self) -> int:
        return self.n_up + self.n_dn


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _require_cuda(t: torch.Tensor, dtype: torch.dtype, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    return t.contiguous()


_WS: dict = {}


def workspace(nbytes: int, device: torch.device, tag: str = "default") -> torch.Tensor:
    """A cached byte buffer of at least ``nbytes`` on ``device`` (grown on demand)."""
    key = (str(device), tag)
    buf = _WS.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _WS[key] = buf
    return buf


def init_params(Lx: int, Ly: int, channels: int = 32, layers: int = 4, std: float = 0.02,
                seed: int = 0) -> dict:
    """Seeded random parameters (numpy FP32): conv weights and biases N(0, std), the pairing
    parameters W (3, N, d) N(0, 1) / sqrt(d) and theta = 0.55 (``models.py:146-149``)."""
    rng = np.random.default_rng(seed)
    conv_w, conv_b = [], []
    cin = 2
    for _ in range(layers):
        conv_w.append(rng.normal(0.0, std, (channels, cin, 3, 3)).astype(np.float32))
        conv_b.append(rng.normal(0.0, std, (channels,)).astype(np.float32))
        cin = channels
    d = channels // 2
    W = (rng.normal(0.0, 1.0, (3, Lx * Ly, d)) / np.sqrt(d)).astype(np.float32)
    return dict(conv_w=conv_w, conv_b=conv_b, W=W, theta=np.float32(0.55), Lx=Lx, Ly=Ly)


def build_wtilde(W: torch.Tensor, theta: float, geom: PairGeometry, fp64: bool = False):
    """(3, N, d) -> (4, N, d) spin-block table with the distance envelope (FP32), and with
    ``fp64`` also the same table in FP64: returns ``(Wt, Wt64)`` then."""
    W = _require_cuda(W, torch.float32, "W")
    if tuple(W.shape) != (3, geom.N, geom.d):
        raise ValueError(f"W shape {tuple(W.shape)} != (3, {geom.N}, {geom.d})")
    Wt = torch.empty((4, geom.N, geom.d), dtype=torch.float32, device=W.device)
    Wt64 = torch.empty((4, geom.N, geom.d), dtype=torch.float64, device=W.device) if fp64 else None
    _lib.call("nh_build_wtilde", W.data_ptr(), float(theta), geom.LX, geom.LY, geom.d,
              Wt.data_ptr(), _ptr(Wt64), stream_ptr(W.device))
    return (Wt, Wt64) if fp64 else Wt


def pairing_occ(Y: torch.Tensor, idx: torch.Tensor, Wt: torch.Tensor, geom: PairGeometry) -> torch.Tensor:
    """F (..., n, n) = sum_a Y[p, a] Wt[2 s_p + s_q, site_p - site_q, a] Y[q, a], exactly
    antisymmetric; Y (..., n, d) FP32, idx (..., n) int32 ascending occupied modes."""
    Y = _require_cuda(Y, torch.float32, "Y")
    idx = _require_cuda(idx, torch.int32, "idx")
    Wt = _require_cuda(Wt, torch.float32, "Wt")
    n, d = Y.shape[-2], Y.shape[-1]
    if d != geom.d or idx.shape[-1] != n or tuple(Wt.shape) != (4, geom.N, d):
        raise ValueError("pairing_occ: inconsistent shapes")
    batch = int(np.prod(Y.shape[:-2])) if Y.dim() > 2 else 1
    F = torch.empty(Y.shape[:-2] + (n, n), dtype=torch.float32, device=Y.device)
    _lib.call("nh_pairing_occ", Y.data_ptr(), idx.data_ptr(), Wt.data_ptr(), geom.LX, geom.LY, d,
              n, batch, F.data_ptr(), stream_ptr(Y.device))
    return F


def pairing_occ_vjp(Y: torch.Tensor, idx: torch.Tensor, Wt: torch.Tensor, G: torch.Tensor,
                    geom: PairGeometry):
    """Cotangents (dY (..., n, d), dWt (..., 4, N, d)) of F = pairing_occ(Y, idx, Wt) for the
    output cotangent G (..., n, n): ``_pairing_occ_bwd`` (``pf_kernel.py:354-365``) per matrix,
    with dY formed from G - G^T and dWt from G; a batched caller sums dWt over the batch."""
    Y = _require_cuda(Y, torch.float32, "Y")
    idx = _require_cuda(idx, torch.int32, "idx")
    Wt = _require_cuda(Wt, torch.float32, "Wt")
    G = _require_cuda(G, torch.float32, "G")
    n, d = Y.shape[-2], Y.shape[-1]
    if (d != geom.d or idx.shape[-1] != n or tuple(Wt.shape) != (4, geom.N, d)
            or tuple(G.shape[-2:]) != (n, n) or G.shape[:-2] != Y.shape[:-2]):
        raise ValueError("pairing_occ_vjp: inconsistent shapes")
    batch = int(np.prod(Y.shape[:-2])) if Y.dim() > 2 else 1
    dY = torch.empty_like(Y)
    dWt = torch.empty(Y.shape[:-2] + (4, geom.N, d), dtype=torch.float32, device=Y.device)
    _lib.call("nh_pairing_occ_vjp", Y.data_ptr(), idx.data_ptr(), Wt.data_ptr(), G.data_ptr(),
              geom.LX, geom.LY, d, n, batch, dY.data_ptr(), dWt.data_ptr(), stream_ptr(Y.device))
    return dY, dWt


def slogpf_adjoint(F: torch.Tensor):
    """(G, flags): G = d log|pf F| / dF = 1/2 F^{-T} for antisymmetric F (..., n, n), FP32,
    n even and at most 224; flags mark singular (FLAG_ZERO_PIVOT) or non-finite matrices, whose
    G is zero."""
    F = _require_cuda(F, torch.float32, "F")
    n = F.shape[-1]
    if F.shape[-2] != n:
        raise ValueError("slogpf_adjoint: matrices must be square")
    batch = int(np.prod(F.shape[:-2])) if F.dim() > 2 else 1
    G = torch.empty_like(F)
    flags = torch.empty(F.shape[:-2], dtype=torch.int32, device=F.device)
    _lib.call("nh_pfaffian_adjoint", F.data_ptr(), n, batch, G.data_ptr(), flags.data_ptr(),
              stream_ptr(F.device))
    return G, flags


# FP64 features (and an FP64 refinement of the log-Pfaffian against the FP64 pairing block) for
# every image whose estimated error |w_g| x pivot ratio exceeds this; w_g is the image's signed
# share of the projected amplitude (1 without projection).  5 keeps log|psi| within 1e-4 of FP64
# on every configuration of the 16x16 benchmark set for both CNN forms.
DEFAULT_COND_TAU = 5.0
# Projected amplitudes whose 8 images cancel by more than this factor are recomputed in FP64:
# the cancellation amplifies the FP32 error of the images by the same factor.
DEFAULT_CANCEL_TAU = 8.0
# Images whose FP32 pivot ratio exceeds this are refined in FP64 with their FP32 pivot order
# against their own FP32 pairing block (a blocked static-pivot elimination, no pivot search):
# it removes the FP32 factorisation error.  Off by default: the images whose error matters
# already get FP64 features and the same refinement through cond_tau.
DEFAULT_REFINE_TAU = 0.0


def slogpf(F: torch.Tensor, cond_tau: float = DEFAULT_COND_TAU):
    """(sign FP32, logabs FP64, flags int32) of the Pfaffians of antisymmetric F (..., n, n)
    in FP32, n even and at most 1024; only the strict lower triangle is read.  Matrices whose
    pivot ratio exceeds ``cond_tau`` are factorised again in FP64 (flags NH_FLAG_GROWTH |
    NH_FLAG_REFINED): for n <= 224 with the pivot order of the FP32 factorisation held fixed,
    beyond with FP64 partial pivoting; ``cond_tau=0`` keeps the plain FP32 result."""
    F = _require_cuda(F, torch.float32, "F")
    n = F.shape[-1]
    if F.shape[-2] != n:
        raise ValueError("slogpf: matrices must be square")
    batch_shape = F.shape[:-2]
    batch = int(np.prod(batch_shape)) if len(batch_shape) else 1
    sign = torch.empty(batch, dtype=torch.float32, device=F.device)
    logabs = torch.empty(batch, dtype=torch.float64, device=F.device)
    flags = torch.empty(batch, dtype=torch.int32, device=F.device)
    nbytes = _lib.load().nh_slogpf_workspace_bytes(n, batch)
    ws = workspace(nbytes, F.device, "slogpf")
    _lib.call("nh_slogpf", F.data_ptr(), n, batch, float(cond_tau), sign.data_ptr(),
              logabs.data_ptr(), flags.data_ptr(), ws.data_ptr(), ws.numel(),
              stream_ptr(F.device))
    return sign.reshape(batch_shape), logabs.reshape(batch_shape), flags.reshape(batch_shape)


class PfaffianBackflow:
    """psi(s) = pf[n * f(n) * n] * fermion_inverse_sign(s) (``models.py:121-211``) with the
    backflow CNN of the graded configurations, or, for parameters with ``net="resconv"`` (a
    released state, ``checkpoint.load_pfaffian_backflow``), the residual CNN of
    ``models.py:319-329``; parameters live on the GPU in FP32."""

    def __init__(self, Lx: int, Ly: int, n_up: int, n_dn: int, params: Optional[dict] = None,
                 channels: int = 32, layers: int = 4, seed: int = 0, device="cuda",
                 cond_tau: float = DEFAULT_COND_TAU, cnn_mode: int = 0,
                 pf_mode: int = 0, cancel_tau: float = DEFAULT_CANCEL_TAU,
                 refine_tau: float = DEFAULT_REFINE_TAU):
        """``cond_tau``: items whose pivot ratio exceeds it are recomputed end to end in FP64
        (``0`` keeps every item on the FP32 path).  ``cnn_mode``: 0 FP32 CUDA cores, 1 tcgen05
        BF16, 2 tcgen05 BF16 x3 (near-FP32); modes 1 and 2 need 16x16, 32 channels, 4 layers.
        ``pf_mode``: 0 Pfaffian on CUDA cores, 1 matrix in tensor memory with tcgen05 updates.
        ``cancel_tau`` (projected amplitudes): configurations whose images cancel by more than
        this factor are recomputed in FP64 (0 = off; default 8).  ``refine_tau``: images whose
        FP32 pivot ratio exceeds it get their log-Pfaffian refined in FP64 with the FP32 pivot
        order (0 = off, 1 = every image; n <= 224)."""
        self.device = torch.device(device)
        self.cond_tau = float(cond_tau)
        self.refine_tau = float(refine_tau)
        self.cnn_mode = int(cnn_mode)
        self.pf_mode = int(pf_mode)
        self.cancel_tau = float(cancel_tau)
        if params is None:
            params = init_params(Lx, Ly, channels, layers, seed=seed)
        self.net = _lib.NET_RESCONV if params.get("net", "cnn") == "resconv" else _lib.NET_CNN
        self.channels = int(params["conv_w"][0].shape[0])
        # residual network: ``layers`` counts blocks of two convolutions
        self.layers = len(params["conv_w"]) // (2 if self.net == _lib.NET_RESCONV else 1)
        self.geom = PairGeometry(Lx, Ly, self.channels // 2, n_up, n_dn)
        self.host_params = params
        self.set_params(params)

    def set_params(self, params: dict) -> None:
        dev = self.device
        head = [np.asarray(params["embed"], np.float32).ravel()] if self.net else []
        self.conv_w = torch.from_numpy(np.concatenate(
            head + [np.asarray(w, np.float32).ravel() for w in params["conv_w"]])).to(dev)
        self.conv_b = torch.from_numpy(np.concatenate(
            [np.asarray(b, np.float32).ravel() for b in params["conv_b"]])).to(dev)
        if self.net == _lib.NET_RESCONV:
            nf = _lib.load().nh_pack_resconv_weights_floats(self.channels, self.layers)
            self.conv_w_packed = torch.empty(nf, dtype=torch.float32, device=dev)
            _lib.call("nh_pack_resconv_weights", self.conv_w.data_ptr(), self.channels,
                      self.layers, self.conv_w_packed.data_ptr(), stream_ptr(dev))
        else:
            self.conv_w_packed = torch.empty_like(self.conv_w)
            _lib.call("nh_pack_cnn_weights", self.conv_w.data_ptr(), self.channels,
                      self.layers, self.conv_w_packed.data_ptr(), stream_ptr(dev))
        self.conv_w_tc = None
        if self.net == _lib.NET_RESCONV and self.geom.LX == 16 and self.geom.LY == 16:
            nbytes = _lib.load().nh_pack_resconv_weights_tc_bytes(self.layers)
            self.conv_w_tc = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            _lib.call("nh_pack_resconv_weights_tc", self.conv_w.data_ptr(), self.channels,
                      self.layers, self.conv_w_tc.data_ptr(), stream_ptr(dev))
        if self.net == _lib.NET_CNN and self.channels == 32 and self.layers == 4:
            nbytes = _lib.load().nh_pack_cnn_weights_tc_bytes()
            self.conv_w_tc = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            _lib.call("nh_pack_cnn_weights_tc", self.conv_w.data_ptr(), self.channels,
                      self.layers, self.conv_w_tc.data_ptr(), stream_ptr(dev))
        self.W = torch.from_numpy(np.asarray(params["W"], np.float32)).to(dev).contiguous()
        self.theta = float(params["theta"])
        self.Wt, self.Wt64 = build_wtilde(self.W, self.theta, self.geom, fp64=True)
        self.host_params = params

    ansatz = _lib.ANSATZ_PFAFFIAN
    delta_d = 0.0

    def c_params(self) -> _lib.BackflowParams:
        g = self.geom
        return _lib.BackflowParams(self.conv_w.data_ptr(), self.conv_b.data_ptr(),
                                   self.conv_w_packed.data_ptr(), _ptr(self.conv_w_tc),
                                   self.Wt.data_ptr(), self.Wt64.data_ptr(), g.LX, g.LY, g.n_up,
                                   g.n_dn, self.channels, self.layers, self.cnn_mode, self.pf_mode,
                                   self.net, self.ansatz, self.cond_tau, self.cancel_tau,
                                   self.refine_tau, float(self.delta_d))

    @property
    def param_count(self) -> int:
        """Parameters of the backflow CNN state (the Jacobian's columns): conv weights and
        biases per layer, W (3, N, d) and theta."""
        return int(_lib.load().nh_param_count(ctypes.byref(self.c_params())))

    def features(self, spins: torch.Tensor) -> torch.Tensor:
        """(B, 2, N, d) backflow features of int8 configurations (B, 2N)."""
        spins = _require_cuda(spins, torch.int8, "spins")
        B = spins.shape[0]
        out = torch.empty((B, 2, self.geom.N, self.geom.d), dtype=torch.float32,
                          device=spins.device)
        p = self.c_params()
        _lib.call("nh_cnn_forward", spins.data_ptr(), B, ctypes.byref(p), out.data_ptr(),
                  stream_ptr(spins.device))
        return out


class BCSBackflow(PfaffianBackflow):
    """The BCS-backflow state of ``code/backflow/models.py:214-302``:
    psi(s) = det F (-1)^(n_up (n_up - 1) / 2) fermion_inverse_sign(s) with the occupied up x down
    block F[p, q] = sum_a y_up[p, a] Wt_ud[site_p - site_q, a] y_dn[q, a] + delta_d fd(p, q)
    (``bcs_kernel.py:1-70``; fd the nearest-neighbour d-wave form factor).  The features are the
    two spin halves of the backflow network's output (d = 16: 32 channels); parameters are those
    of ``PfaffianBackflow`` with W of shape (N, d) and ``delta_d`` (default 0.1, as
    ``models.py:246``).  n_up == n_dn <= 224; FP64 recompute of flagged images up to 128.  The
    reference's own BCS network (a learned (2, d, C) head on its ResConv trunk, d = 64,
    ``models.py:261-270,330-331``) is not supported: the determinant's gather takes d = 16."""

    ansatz = _lib.ANSATZ_BCS

    def __init__(self, Lx: int, Ly: int, n_up: int, n_dn: int, params: Optional[dict] = None,
                 seed: int = 0, **kw):
        if params is None:
            params = init_params(Lx, Ly, kw.get("channels", 32), kw.get("layers", 4), seed=seed)
            params["W"] = params["W"][0]
            params["delta_d"] = 0.1
        super().__init__(Lx, Ly, n_up, n_dn, params=params, seed=seed, **kw)

    def set_params(self, params: dict) -> None:
        W = np.asarray(params["W"], np.float32)
        if W.ndim != 2:
            raise ValueError(f"BCS W must be (N, d), got {W.shape}")
        self.delta_d = float(params.get("delta_d", 0.1))
        full = dict(params)
        full["W"] = np.stack([W, np.zeros_like(W), np.zeros_like(W)])
        super().set_params(full)
        self.host_params = params
