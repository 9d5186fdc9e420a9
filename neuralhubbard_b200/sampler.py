"""Metropolis hop sampler (``ParticleHop`` of ``code/states.py:397-408``; sweeps as in
``code/measure_orderparams.py:128``).

The plain uniform-hop proposal: a uniformly chosen electron hops along a uniformly chosen
direction (4 nearest or 8 nearest + next-nearest); a move onto an occupied site is a null
move.  The proposal is symmetric and accepted with min(1, |psi(s')/psi(s)|^2).  All steps run
in ``nh_metropolis_steps``; random numbers are Philox4x32-10 counters keyed by ``seed``, so a
run is reproducible and independent of how the steps are split into calls.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Union

import numpy as np
import torch

from . import _lib
from .backflow import stream_ptr, workspace
from .state import LogArray, Samples, Variational, as_spins


def random_spins(rng: np.random.Generator, batch: int, N: int, n_up: int, n_dn: int) -> np.ndarray:
    """(batch, 2N) int8 +-1 with exactly n_up / n_dn occupied sites (uniform per half)."""
    s = -np.ones((batch, 2 * N), dtype=np.int8)
    up = np.argsort(rng.random((batch, N)), axis=1)[:, :n_up]
    dn = np.argsort(rng.random((batch, N)), axis=1)[:, :n_dn]
    np.put_along_axis(s, up, 1, axis=1)
    np.put_along_axis(s, N + dn, 1, axis=1)
    return s


class ParticleHop:
    """``nsamples`` Metropolis chains with the plain uniform-hop proposal."""

    def __init__(self, state: Variational, nsamples: int, thermal_steps: int = 0,
                 sweep_steps: Optional[int] = None,
                 n_neighbor: Union[int, Sequence[int]] = 1, initial_spins=None, seed: int = 0):
        self.state = state
        self.nsamples = int(nsamples)
        g = state.model.geom
        nn = [n_neighbor] if isinstance(n_neighbor, int) else list(n_neighbor)
        self.n_dirs = 8 if 2 in nn else 4
        self.sweep_steps = int(sweep_steps) if sweep_steps is not None else g.N
        self.seed = int(seed)
        self.step = 0
        if initial_spins is None:
            initial_spins = random_spins(np.random.default_rng(seed), self.nsamples, g.N,
                                         g.n_up, g.n_dn)
        spins = as_spins(initial_spins, state.device)
        if spins.shape[0] != self.nsamples:
            spins = spins.repeat((self.nsamples + spins.shape[0] - 1) // spins.shape[0], 1)
            spins = spins[: self.nsamples].contiguous()
        self.spins = spins
        self.psi = state(self.spins)
        self.accepted = torch.zeros(self.nsamples, dtype=torch.int32, device=state.device)
        self.proposed_steps = 0
        if thermal_steps:
            self.run(thermal_steps)

    def run(self, nsteps: int) -> None:
        """Advance every chain by ``nsteps`` Metropolis steps."""
        if nsteps <= 0:
            return
        st = self.state
        p = st.model.c_params()
        lib = _lib.load()
        nbytes = lib.nh_metropolis_workspace_bytes(self.nsamples, st.n_symm, ctypes.byref(p))
        ws = workspace(nbytes, st.device, "metropolis")
        sign = self.psi.sign.contiguous()
        logabs = self.psi.logabs.contiguous()
        _lib.call("nh_metropolis_steps", self.spins.data_ptr(), sign.data_ptr(), logabs.data_ptr(),
                  self.nsamples, st.n_symm, ctypes.byref(p), self.n_dirs, self.seed, self.step,
                  int(nsteps), self.accepted.data_ptr(), ws.data_ptr(), ws.numel(),
                  stream_ptr(st.device))
        self.psi = LogArray(sign, logabs)
        self.step += int(nsteps)
        self.proposed_steps += int(nsteps)

    def sweep(self, nsteps: Optional[int] = None) -> Samples:
        self.run(self.sweep_steps if nsteps is None else nsteps)
        return Samples(self.spins.clone(), LogArray(self.psi.sign.clone(), self.psi.logabs.clone()))

    @property
    def acceptance(self) -> float:
        if self.proposed_steps == 0:
            return 0.0
        return float(self.accepted.sum().item()) / (self.nsamples * self.proposed_steps)
