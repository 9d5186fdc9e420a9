"""Metropolis samplers (``ParticleHop``, ``SiteExchange`` and ``MixSampler`` of
``code/states.py:397-408``; sweeps as in ``code/measure_orderparams.py:128``).

ParticleHop: a uniformly chosen electron hops along a uniformly chosen direction (4 nearest or
8 nearest + next-nearest); a move onto an occupied site is a null move.  SiteExchange: a
uniformly chosen site swaps its occupation (both spin species) with one of its neighbours; equal
occupations are a null move.  Both proposals are symmetric and accepted with
min(1, |psi(s')/psi(s)|^2).  MixSampler runs a ParticleHop and a SiteExchange chain set as one
(the reference samples with ``MixSampler([ParticleHop(state, B/2), SiteExchange(state, B/2)])``).
All steps run in ``nh_metropolis_steps_mixed``; random numbers are Philox4x32-10 counters keyed
by ``seed``, so a run is reproducible and independent of how the steps are split into calls.
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


def _n_dirs(n_neighbor) -> int:
    nn = [n_neighbor] if isinstance(n_neighbor, int) else list(n_neighbor)
    return 8 if 2 in nn else 4


class _Chains:
    """``nsamples`` Metropolis chains: chains [0, first_exchange) make hop steps, the others
    site-exchange steps."""

    def __init__(self, state: Variational, nsamples: int, first_exchange: int, n_dirs: int,
                 thermal_steps: int, sweep_steps: Optional[int], initial_spins, seed: int):
        self.state = state
        self.nsamples = int(nsamples)
        self.first_exchange = int(first_exchange)
        g = state.model.geom
        self.n_dirs = int(n_dirs)
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
        self._psi: Optional[LogArray] = None  # evaluated on first use (components of a
        # MixSampler never evaluate theirs)
        self.accepted = torch.zeros(self.nsamples, dtype=torch.int32, device=state.device)
        self.proposed_steps = 0
        if thermal_steps:
            self.run(thermal_steps)

    @property
    def psi(self) -> LogArray:
        if self._psi is None:
            self._psi = self.state(self.spins)
        return self._psi

    @psi.setter
    def psi(self, value: LogArray) -> None:
        self._psi = value

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
        _lib.call("nh_metropolis_steps_mixed", self.spins.data_ptr(), sign.data_ptr(),
                  logabs.data_ptr(), self.nsamples, st.n_symm, ctypes.byref(p), self.n_dirs,
                  self.first_exchange, self.seed, self.step, int(nsteps),
                  self.accepted.data_ptr(), ws.data_ptr(), ws.numel(), stream_ptr(st.device))
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


class ParticleHop(_Chains):
    """``nsamples`` Metropolis chains with the plain uniform-hop proposal."""

    def __init__(self, state: Variational, nsamples: int, thermal_steps: int = 0,
                 sweep_steps: Optional[int] = None,
                 n_neighbor: Union[int, Sequence[int]] = 1, initial_spins=None, seed: int = 0):
        super().__init__(state, nsamples, nsamples, _n_dirs(n_neighbor), thermal_steps,
                         sweep_steps, initial_spins, seed)


class SiteExchange(_Chains):
    """``nsamples`` Metropolis chains with the site-exchange proposal: a uniform site and one of
    its neighbours (nearest, or nearest and next-nearest) swap their occupations."""

    def __init__(self, state: Variational, nsamples: int, thermal_steps: int = 0,
                 sweep_steps: Optional[int] = None,
                 n_neighbor: Union[int, Sequence[int]] = 1, initial_spins=None, seed: int = 0):
        super().__init__(state, nsamples, 0, _n_dirs(n_neighbor), thermal_steps, sweep_steps,
                         initial_spins, seed)


class MixSampler(_Chains):
    """One chain set made of the chains of a ParticleHop and a SiteExchange sampler
    (``qtx.sampler.MixSampler`` as built at ``code/states.py:397-408``): the hop chains come
    first (indices [0, n_hop)), the exchange chains after them.  The component samplers give the
    chain counts and the neighbour range; their own chains are not used."""

    def __init__(self, samplers: Sequence[_Chains], thermal_steps: int = 0,
                 sweep_steps: Optional[int] = None, initial_spins=None, seed: int = 0):
        if not samplers:
            raise ValueError("MixSampler needs at least one sampler")
        state = samplers[0].state
        if any(smp.state is not state for smp in samplers):
            raise ValueError("MixSampler: the samplers must share one state")
        if len({smp.n_dirs for smp in samplers}) != 1:
            raise ValueError("MixSampler: the samplers must use the same neighbour range")
        n_hop = sum(smp.nsamples for smp in samplers if isinstance(smp, ParticleHop))
        n_exc = sum(smp.nsamples for smp in samplers if isinstance(smp, SiteExchange))
        if n_hop + n_exc != sum(smp.nsamples for smp in samplers):
            raise TypeError("MixSampler combines ParticleHop and SiteExchange samplers")
        super().__init__(state, n_hop + n_exc, n_hop, samplers[0].n_dirs, thermal_steps,
                         sweep_steps, initial_spins, seed)
