"""Learned hop proposal: parameters, GPU training and the Metropolis sampler that uses it.

The reference samples with quantax's uniform ``ParticleHop`` (``code/states.py:397-408``); this
module adds a proposal network that chooses which electron hops where.  The network (a periodic
3x3 CNN 2 -> 16 -> 16 -> 16, see ``include/nh_b200.h``) is trained on the GPU by the library's
own forward/backward/Adam kernels, and it is used under an exact Metropolis-Hastings correction,
so the sampled distribution stays |psi|^2 whatever the network has learned.

Training data: configurations taken from plain-sampler chains; for each, one move drawn
uniformly among its valid moves and a weight w(|psi(s')/psi(s)|^2) (``target_weight``: the
Metropolis acceptance min(1, r) by default, or a locally balanced sqrt(r) or r / (1 + r)).  The
loss -(1/B) sum w log q(m | s) is minimised by a proposal that offers moves in proportion to w.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from .backflow import stream_ptr, workspace
from .sampler import ParticleHop
from .state import LogArray, Variational, as_spins

N_OUT = 16
PARAM_COUNT = _lib.PROPOSAL_PARAMS
SHAPES = [(16, 2, 3, 3), (16,), (16, 16, 3, 3), (16,), (16, 16, 3, 3), (16,)]
HOP_DIRS = np.array([(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (1, -1), (-1, 1), (-1, -1)])


def init_proposal_params(seed: int = 0, std: float = 0.05) -> np.ndarray:
    """Seeded N(0, std) weights and zero biases (flat FP32, ``PARAM_COUNT`` values)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, std, size=s).ravel() if len(s) > 1 else np.zeros(s) for s in SHAPES]
    return np.concatenate(parts).astype(np.float32)


def neighbour_table(Lx: int, Ly: int) -> np.ndarray:
    """(N, 8) target site of each site along each hop direction."""
    x, y = np.divmod(np.arange(Lx * Ly), Ly)
    nx = (x[:, None] + HOP_DIRS[None, :, 0]) % Lx
    ny = (y[:, None] + HOP_DIRS[None, :, 1]) % Ly
    return nx * Ly + ny


class HopProposal:
    """Parameters (FP32 master, Adam moments, BF16 image) of the proposal network on the GPU."""

    def __init__(self, Lx: int, Ly: int, n_dirs: int = 8, params: Optional[np.ndarray] = None,
                 seed: int = 0, std: float = 0.05, device="cuda"):
        self.Lx, self.Ly, self.N = int(Lx), int(Ly), int(Lx) * int(Ly)
        self.n_dirs = int(n_dirs)
        self.device = torch.device(device)
        if params is None:
            params = init_proposal_params(seed, std)
        self.master = torch.from_numpy(np.asarray(params, np.float32).copy()).to(self.device)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.weights = torch.empty(PARAM_COUNT, dtype=torch.bfloat16, device=self.device)
        self.t = 0
        self.refresh()

    def refresh(self) -> None:
        """Re-round the BF16 image after the master changed outside ``adam_step``."""
        _lib.call("nh_proposal_pack", self.master.data_ptr(), PARAM_COUNT,
                  self.weights.data_ptr(), stream_ptr(self.device))

    def c_params(self) -> _lib.ProposalParams:
        return _lib.ProposalParams(self.weights.data_ptr(), self.Lx, self.Ly, self.n_dirs, 0)

    def logits(self, spins) -> torch.Tensor:
        """(B, 16, N) raw logits of int8 configurations (B, 2N)."""
        spins = as_spins(spins, self.device)
        out = torch.empty((spins.shape[0], N_OUT, self.N), dtype=torch.float32,
                          device=self.device)
        q = self.c_params()
        _lib.call("nh_proposal_forward", spins.data_ptr(), spins.shape[0], ctypes.byref(q),
                  out.data_ptr(), stream_ptr(self.device))
        return out

    def sample(self, spins, seed: int, step: int):
        """One proposal per configuration: (from_mode, to_mode, valid, log q ratio)."""
        spins = as_spins(spins, self.device)
        B = spins.shape[0]
        i32 = dict(dtype=torch.int32, device=self.device)
        fr, to, ok = (torch.empty(B, **i32) for _ in range(3))
        lqr = torch.empty(B, dtype=torch.float32, device=self.device)
        q = self.c_params()
        _lib.call("nh_proposal_sample", spins.data_ptr(), B, ctypes.byref(q), int(seed),
                  int(step), fr.data_ptr(), to.data_ptr(), ok.data_ptr(), lqr.data_ptr(),
                  stream_ptr(self.device))
        return fr, to, ok, lqr

    def loss_grad(self, spins, moves, weights):
        """Loss -(1/B) sum w log q(m | s) and its gradient (FP32 tensors on the device)."""
        spins = as_spins(spins, self.device)
        moves = moves.to(self.device, torch.int32).contiguous()
        weights = weights.to(self.device, torch.float32).contiguous()
        B = spins.shape[0]
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        grad = torch.empty(PARAM_COUNT, dtype=torch.float32, device=self.device)
        q = self.c_params()
        nbytes = _lib.load().nh_proposal_backward_workspace_bytes(B, ctypes.byref(q))
        ws = workspace(nbytes, self.device, "proposal_backward")
        _lib.call("nh_proposal_backward", spins.data_ptr(), moves.data_ptr(), weights.data_ptr(),
                  B, ctypes.byref(q), loss.data_ptr(), grad.data_ptr(), ws.data_ptr(), ws.numel(),
                  stream_ptr(self.device))
        return loss, grad

    def adam_step(self, grad: torch.Tensor, lr: float, beta1: float = 0.9,
                  beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.t += 1
        _lib.call("nh_proposal_adam_step", self.master.data_ptr(), self.m.data_ptr(),
                  self.v.data_ptr(), grad.data_ptr(), PARAM_COUNT, self.t, float(lr),
                  float(beta1), float(beta2), float(eps), self.weights.data_ptr(),
                  stream_ptr(self.device))

    def train(self, records, steps: int, batch: int = 512, lr: float = 3e-3, seed: int = 0):
        """Adam on minibatches drawn (seeded, with replacement across epochs) from ``records``
        = (spins, moves, weights).  Returns the per-step losses (host floats)."""
        spins, moves, weights = records
        n = spins.shape[0]
        gen = torch.Generator(device="cpu")
        gen.manual_seed(int(seed))
        losses = []
        perm = torch.randperm(n, generator=gen)
        pos = 0
        for it in range(int(steps)):
            if pos + batch > n:
                perm = torch.randperm(n, generator=gen)
                pos = 0
            idx = perm[pos : pos + batch].to(self.device)
            pos += batch
            loss, grad = self.loss_grad(spins[idx], moves[idx], weights[idx])
            self.adam_step(grad, lr)
            losses.append(loss)
        return [float(x.item()) for x in losses]

    def numpy(self) -> np.ndarray:
        return self.master.detach().cpu().numpy()


def valid_moves(spins: torch.Tensor, Lx: int, Ly: int, n_dirs: int = 8) -> torch.Tensor:
    """(B, 16 N) bool: move m = (sigma * 8 + d) * N + i is valid."""
    N = Lx * Ly
    B = spins.shape[0]
    nbr = torch.from_numpy(neighbour_table(Lx, Ly)).to(spins.device)
    occ = spins.view(B, 2, N) > 0
    tgt = occ[:, :, nbr]  # (B, 2, N, 8)
    ok = occ[:, :, :, None] & ~tgt
    if n_dirs < 8:
        ok[:, :, :, n_dirs:] = False
    return ok.permute(0, 1, 3, 2).reshape(B, 16 * N)


def apply_moves(spins: torch.Tensor, moves: torch.Tensor, Lx: int, Ly: int) -> torch.Tensor:
    N = Lx * Ly
    nbr = torch.from_numpy(neighbour_table(Lx, Ly)).to(spins.device)
    c, i = moves // N, moves % N
    sg, d = c // 8, c % 8
    fr = sg * N + i
    to = sg * N + nbr[i, d]
    out = spins.clone()
    rows = torch.arange(spins.shape[0], device=spins.device)
    out[rows, fr] = -1
    out[rows, to] = 1
    return out


WEIGHTS = ("acceptance", "sqrt", "barker")


def target_weight(lr2: torch.Tensor, kind: str, clip: float = 20.0) -> torch.Tensor:
    """Training weight of a move with log |psi(s')/psi(s)|^2 = lr2.  The loss is minimised by
    q(m | s) proportional to the weight: "acceptance" min(1, r), or the locally balanced
    proposals of G. Zanella, JASA 115 (2020) 852, "sqrt" sqrt(r) (clipped) and "barker"
    r / (1 + r)."""
    if kind == "acceptance":
        return torch.exp(torch.clamp(lr2, max=0.0))
    if kind == "sqrt":
        return torch.exp(torch.clamp(0.5 * lr2, max=float(np.log(clip))))
    if kind == "barker":
        return torch.sigmoid(lr2)
    raise ValueError(f"weight {kind!r} not in {WEIGHTS}")


def training_records(state: Variational, spins, psi: Optional[LogArray] = None, seed: int = 0,
                     n_dirs: int = 8, chunk: int = 65536, weight: str = "acceptance"):
    """(spins, moves, weights) records: one uniformly drawn valid move per configuration and its
    ``target_weight`` (default min(1, |psi(s')/psi(s)|^2)), with the amplitudes from ``state``
    (one evaluation per record)."""
    g = state.model.geom
    spins = as_spins(spins, state.device)
    B = spins.shape[0]
    if psi is None:
        psi = state(spins)
    gen = torch.Generator(device=state.device)
    gen.manual_seed(int(seed))
    moves = torch.empty(B, dtype=torch.int64, device=state.device)
    weights = torch.empty(B, dtype=torch.float32, device=state.device)
    for a in range(0, B, chunk):
        s = spins[a : a + chunk]
        ok = valid_moves(s, g.LX, g.LY, n_dirs)
        score = torch.rand(ok.shape, generator=gen, device=state.device).masked_fill_(~ok, -1.0)
        m = score.argmax(1)
        sp = apply_moves(s, m, g.LX, g.LY)
        phi = state(sp)
        lr2 = 2.0 * (phi.logabs - psi.logabs[a : a + chunk])
        w = target_weight(lr2, weight).to(torch.float32)
        w = torch.where((phi.sign != 0) & ok.any(1), w, torch.zeros_like(w))
        moves[a : a + chunk] = m
        weights[a : a + chunk] = w
    return spins, moves.to(torch.int32), weights


class LearnedHop(ParticleHop):
    """Metropolis chains with the learned proposal and the exact Hastings correction."""

    def __init__(self, state: Variational, nsamples: int, proposal: HopProposal,
                 thermal_steps: int = 0, sweep_steps: Optional[int] = None, initial_spins=None,
                 seed: int = 0):
        self.proposal = proposal
        n_neighbor = (1, 2) if proposal.n_dirs == 8 else 1
        super().__init__(state, nsamples, 0, sweep_steps, n_neighbor, initial_spins, seed)
        if thermal_steps:
            self.run(thermal_steps)

    def run(self, nsteps: int) -> None:
        if nsteps <= 0:
            return
        st = self.state
        p = st.model.c_params()
        q = self.proposal.c_params()
        lib = _lib.load()
        nbytes = lib.nh_metropolis_learned_workspace_bytes(self.nsamples, st.n_symm,
                                                           ctypes.byref(p))
        ws = workspace(nbytes, st.device, "metropolis")
        sign = self.psi.sign.contiguous()
        logabs = self.psi.logabs.contiguous()
        _lib.call("nh_metropolis_steps_learned", self.spins.data_ptr(), sign.data_ptr(),
                  logabs.data_ptr(), self.nsamples, st.n_symm, ctypes.byref(p), ctypes.byref(q),
                  self.seed, self.step, int(nsteps), self.accepted.data_ptr(), ws.data_ptr(),
                  ws.numel(), stream_ptr(st.device))
        self.psi = LogArray(sign, logabs)
        self.step += int(nsteps)
        self.proposed_steps += int(nsteps)
