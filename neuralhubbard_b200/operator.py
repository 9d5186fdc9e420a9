"""Hubbard Hamiltonian with the local-energy entry point ``Oloc`` (the ``H.Oloc(state,
Samples(spins, psi))`` call of ``code/quick_start.py:33``; H built as
``Hubbard(U=8, t=[1.0, t'], n_neighbor=[1, 2])`` at ``code/states.py:244-247``)."""

from __future__ import annotations

import ctypes
import threading
from typing import Dict, Optional, Sequence, Tuple, Union

import torch

from . import _lib
from .backflow import stream_ptr, workspace
from .state import Samples, Variational, as_spins


_CHUNK_LOCK = threading.Lock()
_CHUNK_CACHE: Dict[Tuple, int] = {}


def _tune_key(state: Variational, H: "Hubbard") -> Tuple:
    g = state.model.geom
    m = state.model
    return (str(state.device), g.LX, g.LY, g.n_up, g.n_dn, state.n_symm, H.n_dirs,
            getattr(m, "cnn_mode", 0), getattr(m, "pf_mode", 0))


class Hubbard:
    """H = -sum_{<ij> sigma} t_ij (c+_i c_j + h.c.) + U sum_i n_i,up n_i,down on the periodic
    lattice of the state; ``t`` and ``n_neighbor`` follow quantax: a scalar t with
    n_neighbor=1, or t=[t, t'] with n_neighbor=[1, 2]."""

    def __init__(self, U: float = 8.0, t: Union[float, Sequence[float]] = 1.0,
                 n_neighbor: Union[int, Sequence[int]] = 1):
        ts = [float(t)] if isinstance(t, (int, float)) else [float(x) for x in t]
        nn = [int(n_neighbor)] if isinstance(n_neighbor, int) else [int(x) for x in n_neighbor]
        if len(ts) != len(nn) or nn not in ([1], [1, 2]):
            raise ValueError("supported: n_neighbor=1 or [1, 2] with one t per neighbour order")
        self.U = float(U)
        self.t = ts[0]
        self.tp = ts[1] if len(ts) > 1 else 0.0
        self.n_dirs = 8 if len(ts) > 1 else 4
        self.last_n_conn: Optional[int] = 0

    def c_params(self) -> _lib.HubbardParams:
        return _lib.HubbardParams(self.t, self.tp, self.U, self.n_dirs)

    def Oloc(self, state: Variational, samples: Samples, chunk_configs: Optional[int] = None,
             count_connections: bool = True) -> torch.Tensor:
        """(B,) FP64 local energies E_loc(s) = sum_s' <s|H|s'> psi(s') / psi(s).

        ``chunk_configs``: 0 evaluates every connected configuration in one persistent pass (a
        fused kernel taking (configuration, image, connection) items off a device work counter;
        the backflow CNN with n <= 224, else the library's chunks); > 0 evaluates chunks of that
        many configurations; None takes what ``autotune`` picked for this lattice and form (the
        persistent pass if nothing was tuned).  With ``count_connections`` the call waits once
        for the number of connections (kept in ``last_n_conn``); without it, it never waits for
        the GPU and can be captured in a CUDA graph."""
        spins = as_spins(samples.spins, state.device)
        psi = samples.psi if samples.psi is not None else state(spins)
        B = spins.shape[0]
        if chunk_configs is None:
            chunk_configs = _CHUNK_CACHE.get(_tune_key(state, self), 0)
        chunk_configs = max(0, int(chunk_configs))
        eloc = torch.empty(B, dtype=torch.float64, device=state.device)
        p = state.model.c_params()
        h = self.c_params()
        lib = _lib.load()
        nbytes = lib.nh_local_energy_workspace_bytes(B, state.n_symm, chunk_configs, ctypes.byref(p))
        ws = workspace(nbytes, state.device, "local_energy")
        nconn = ctypes.c_int64(0)
        _lib.call("nh_local_energy", spins.data_ptr(), psi.sign.contiguous().data_ptr(),
                  psi.logabs.contiguous().data_ptr(), B, state.n_symm, ctypes.byref(p),
                  ctypes.byref(h), chunk_configs, eloc.data_ptr(),
                  ctypes.byref(nconn) if count_connections else None,
                  ws.data_ptr(), ws.numel(), stream_ptr(state.device))
        self.last_n_conn = int(nconn.value) if count_connections else None
        return eloc

    def autotune(self, state: Variational, samples: Samples,
                 candidates: Sequence[int] = (0, 2048, 8192, 32768), repeats: int = 2) -> int:
        """Time ``Oloc`` on ``samples`` for each evaluation shape (0: the persistent fused pass;
        else chunks of that many configurations), CUDA events after one warm-up call each;
        remember the fastest for this lattice, neighbour range, symmetry and precision form,
        and return it.  Later ``Oloc`` calls without ``chunk_configs`` use it."""
        best, best_ms = 0, float("inf")
        st = torch.cuda.current_stream(state.device)
        for c in candidates:
            self.Oloc(state, samples, chunk_configs=int(c))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(repeats):
                self.Oloc(state, samples, chunk_configs=int(c), count_connections=False)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / repeats
            if ms < best_ms:
                best, best_ms = int(c), ms
        with _CHUNK_LOCK:
            _CHUNK_CACHE[_tune_key(state, self)] = best
        return best

    def hop_list(self, spins: torch.Tensor, Lx: int, Ly: int):
        """Connection bookkeeping: (counts (B,), offsets (B+1,), rec (C, 2), hval (C,))."""
        spins = as_spins(spins, spins.device if isinstance(spins, torch.Tensor) else "cuda")
        B, M = spins.shape
        n_max = int((spins > 0).sum(1).max().item()) if B else 0
        cap = max(1, B * n_max * self.n_dirs)
        counts = torch.empty(B, dtype=torch.int32, device=spins.device)
        offsets = torch.empty(B + 1, dtype=torch.int64, device=spins.device)
        rec = torch.empty((cap, 2), dtype=torch.int32, device=spins.device)
        hval = torch.empty(cap, dtype=torch.float64, device=spins.device)
        h = self.c_params()
        _lib.call("nh_hop_list", spins.data_ptr(), B, Lx, Ly, ctypes.byref(h), counts.data_ptr(),
                  offsets.data_ptr(), rec.data_ptr(), hval.data_ptr(), stream_ptr(spins.device))
        total = int(offsets[-1].item())
        return counts, offsets, rec[:total], hval[:total]
