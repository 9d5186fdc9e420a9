"""quantax-shaped variational state: ``state(spins) -> LogArray`` (the call of
``code/quick_start.py:27`` on the ``Variational`` built at ``code/states.py:318-320``).

The amplitude of a batch runs in one C-ABI call (``nh_amplitude``): symmetry images, backflow
CNN, occupied pairing gather, log-Pfaffian and the signed log-sum over the 8 images of
Flip(0) @ Flip(1) @ SpinInverse() (``code/states.py:274-279``).  ``Variational.jacobian`` gives
the per-sample derivatives of log|psi| that SR / AdamSR consume
(``code/train_pfaffian_16x16_tpm02.py:100-101``) in one call (``nh_log_jacobian``).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _lib
from .backflow import PfaffianBackflow, stream_ptr, workspace


@dataclass
class LogArray:
    """sign * exp(logabs); logabs is FP64 because |log psi| is far outside FP32's resolution
    (``README.md:90-91`` of the reference)."""

    sign: torch.Tensor
    logabs: torch.Tensor
    flags: Optional[torch.Tensor] = None

    def __len__(self) -> int:
        return self.sign.shape[0]

    def __getitem__(self, i):
        return LogArray(self.sign[i], self.logabs[i], None if self.flags is None else self.flags[i])

    def numpy(self):
        return self.sign.cpu().numpy(), self.logabs.cpu().numpy()


@dataclass
class Samples:
    """Configurations and their amplitudes (``quantax.sampler.Samples``)."""

    spins: torch.Tensor
    psi: Optional[LogArray] = None


def as_spins(spins, device) -> torch.Tensor:
    if isinstance(spins, np.ndarray):
        spins = torch.from_numpy(np.ascontiguousarray(spins.astype(np.int8)))
    if not isinstance(spins, torch.Tensor):
        raise TypeError("spins must be a numpy array or a torch tensor")
    if spins.dtype != torch.int8:
        spins = spins.to(torch.int8)
    return spins.to(device, non_blocking=True).contiguous()


class Variational:
    """Symmetry-projected (``symm=True``) or bare amplitudes of a ``PfaffianBackflow``.

    ``max_parallel`` bounds the configurations per C-ABI call (the forward chunk of
    ``code/states.py:80,316-320``); the workspace for one chunk is allocated once and cached.
    """

    def __init__(self, model: PfaffianBackflow, symm: bool = True, max_parallel: int = 8192,
                 check_timeout: bool = True):
        """``check_timeout`` (tensor-core forms only): read the output flags back after each call
        and raise ``DeviceTimeoutError`` if a tensor-core kernel's bounded wait expired (one
        small device-to-host copy; pass False to keep the call free of host synchronisation and
        test ``LogArray.flags`` for ``FLAG_TIMEOUT`` yourself)."""
        self.model = model
        self.n_symm = 8 if symm else 1
        self.max_parallel = int(max_parallel)
        self.check_timeout = bool(check_timeout) and (model.cnn_mode in (1, 2)
                                                      or model.pf_mode == 1)

    @property
    def device(self):
        return self.model.device

    @property
    def N(self) -> int:
        return self.model.geom.N

    def __call__(self, spins) -> LogArray:
        spins = as_spins(spins, self.device)
        B = spins.shape[0]
        if spins.dim() != 2 or spins.shape[1] != 2 * self.N:
            raise ValueError(f"spins shape {tuple(spins.shape)} != (B, {2 * self.N})")
        sign = torch.empty(B, dtype=torch.float32, device=self.device)
        logabs = torch.empty(B, dtype=torch.float64, device=self.device)
        flags = torch.empty(B, dtype=torch.int32, device=self.device)
        p = self.model.c_params()
        lib = _lib.load()
        chunk = min(B, self.max_parallel) if B else 1
        nbytes = lib.nh_amplitude_workspace_bytes(chunk, self.n_symm, ctypes.byref(p))
        ws = workspace(nbytes, self.device, "amplitude")
        st = stream_ptr(self.device)
        for c0 in range(0, B, chunk):
            c1 = min(B, c0 + chunk)
            _lib.call("nh_amplitude", spins[c0:c1].data_ptr(), c1 - c0, self.n_symm,
                      ctypes.byref(p), sign[c0:].data_ptr(), logabs[c0:].data_ptr(),
                      flags[c0:].data_ptr(), ws.data_ptr(), ws.numel(), st)
        if self.check_timeout:
            _lib.check_flags(flags, "nh_amplitude")
        return LogArray(sign, logabs, flags)

    def jacobian(self, spins, max_parallel: Optional[int] = None):
        """(LogArray, O): O (B, P) FP32 with O[b, k] = d log|psi_P(s_b)| / d theta_k (or of
        log|psi(s_b)| without projection), columns in the order conv_w[0], conv_b[0], ...,
        conv_w[L-1], conv_b[L-1], W (3, N, d), theta (``PfaffianBackflow.param_count``).
        FP32 CUDA-core forward and backward; the backflow CNN with n <= 224."""
        spins = as_spins(spins, self.device)
        B = spins.shape[0]
        if spins.dim() != 2 or spins.shape[1] != 2 * self.N:
            raise ValueError(f"spins shape {tuple(spins.shape)} != (B, {2 * self.N})")
        m = self.model
        P = m.param_count
        if P <= 0:
            raise ValueError("jacobian: the backflow CNN state only")
        sign = torch.empty(B, dtype=torch.float32, device=self.device)
        logabs = torch.empty(B, dtype=torch.float64, device=self.device)
        flags = torch.empty(B, dtype=torch.int32, device=self.device)
        jac = torch.empty((B, P), dtype=torch.float32, device=self.device)
        p = m.c_params()
        lib = _lib.load()
        chunk = min(B, max_parallel or self.max_parallel) if B else 1
        nbytes = lib.nh_log_jacobian_workspace_bytes(chunk, self.n_symm, ctypes.byref(p))
        ws = workspace(nbytes, self.device, "jacobian")
        st = stream_ptr(self.device)
        for c0 in range(0, B, chunk):
            c1 = min(B, c0 + chunk)
            _lib.call("nh_log_jacobian", spins[c0:c1].data_ptr(), c1 - c0, self.n_symm,
                      ctypes.byref(p), m.W.data_ptr(), float(m.theta), jac[c0:].data_ptr(),
                      sign[c0:].data_ptr(), logabs[c0:].data_ptr(), flags[c0:].data_ptr(),
                      ws.data_ptr(), ws.numel(), st)
        return LogArray(sign, logabs, flags), jac
