"""Fixed small workloads for profiling single kernels of the library (e.g. under Nsight Compute).

    python -m neuralhubbard_b200.profile_cases <case> [--repeat R]

Each case builds its inputs once and runs the operation ``repeat`` times (default 2, so that a
profiler can skip the first, cold launch).  Inputs exceed the 126 MB L2 where the kernel's DRAM
rate is the figure of interest.

cases:
  pairing            nh_pairing_occ, 16x16, 2048 matrices (F = 411 MB written)
  hops               nh_hop_list count/scan/emit, 16x16, 16384 configurations (16.6M connections)
  eloc               local energy, 8x8 unprojected, 32768 configurations (8.4M connections)
  proposal_sample    learned-proposal draw, 16x16, 4096 chains
  proposal_backward  learned-proposal loss and gradient, 16x16, 4096 records
  resconv_tc         residual network (16 blocks x 64 channels) on tcgen05, 16x16, 64 x 8 images
  resconv            the same network on CUDA cores (FP32)
"""

from __future__ import annotations

import argparse

import numpy as np
import torch

from . import (HopProposal, Hubbard, PfaffianBackflow, Samples, Variational, init_params,
               pairing_occ, random_spins)
from .proposal import valid_moves


def _model(L, cnn_mode=0):
    ne = 7 * L * L // 16
    return PfaffianBackflow(L, L, ne, ne, params=init_params(L, L, 32, 4, std=0.02, seed=0),
                            cnn_mode=cnn_mode), ne


def case_pairing(repeat):
    model, ne = _model(16)
    g = model.geom
    B = 2048
    rng = np.random.default_rng(0)
    Y = torch.from_numpy(rng.normal(size=(B, 2 * ne, g.d)).astype(np.float32)).cuda()
    idx = np.sort(np.stack([rng.choice(2 * g.N, 2 * ne, replace=False) for _ in range(B)]), 1)
    idx = torch.from_numpy(idx.astype(np.int32)).cuda()
    for _ in range(repeat):
        pairing_occ(Y, idx, model.Wt, g)


def case_hops(repeat):
    L = 16
    ne = 7 * L * L // 16
    s = torch.from_numpy(random_spins(np.random.default_rng(1), 16384, L * L, ne, ne)).cuda()
    H = Hubbard(8.0, [1.0, -0.2], [1, 2])
    for _ in range(repeat):
        H.hop_list(s, L, L)


def case_eloc(repeat):
    model, ne = _model(8)
    state = Variational(model, symm=False, max_parallel=65536)
    s = torch.from_numpy(random_spins(np.random.default_rng(2), 32768, 64, ne, ne)).cuda()
    psi = state(s)
    H = Hubbard(8.0, [1.0, -0.2], [1, 2])
    for _ in range(repeat):
        H.Oloc(state, Samples(s, psi), chunk_configs=65536, count_connections=False)


def case_proposal_sample(repeat):
    L = 16
    ne = 7 * L * L // 16
    q = HopProposal(L, L, 8, seed=3, std=0.1)
    s = torch.from_numpy(random_spins(np.random.default_rng(3), 4096, L * L, ne, ne)).cuda()
    for r in range(repeat):
        q.sample(s, 11, r)


def case_proposal_backward(repeat):
    L = 16
    ne = 7 * L * L // 16
    q = HopProposal(L, L, 8, seed=4, std=0.1)
    s = torch.from_numpy(random_spins(np.random.default_rng(4), 4096, L * L, ne, ne)).cuda()
    ok = valid_moves(s, L, L)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    m = torch.rand(ok.shape, generator=gen, device="cuda").masked_fill_(~ok, -1.0).argmax(1)
    w = torch.rand(4096, generator=gen, device="cuda")
    for _ in range(repeat):
        q.loss_grad(s, m.to(torch.int32), w)


def _resconv(repeat, cnn_mode):
    rng = np.random.default_rng(6)
    L, C = 16, 64
    params = dict(net="resconv", embed=rng.normal(size=(C, 4)).astype(np.float32),
                  conv_w=[(rng.normal(size=(C, C, 3, 3)) * 0.04).astype(np.float32)
                          for _ in range(32)],
                  conv_b=[(rng.normal(size=C) * 0.1).astype(np.float32) for _ in range(32)],
                  W=(rng.normal(size=(3, L * L, 32)) / np.sqrt(32)).astype(np.float32),
                  theta=0.55)
    ne = 7 * L * L // 16
    model = PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=cnn_mode, cond_tau=0.0,
                             cancel_tau=0.0)
    state = Variational(model, symm=True)
    s = torch.from_numpy(random_spins(np.random.default_rng(7), 64, L * L, ne, ne)).cuda()
    for _ in range(repeat):
        state(s)


def case_resconv_tc(repeat):
    _resconv(repeat, 2)


def case_resconv(repeat):
    _resconv(repeat, 0)


CASES = {"pairing": case_pairing, "hops": case_hops, "eloc": case_eloc,
         "proposal_sample": case_proposal_sample, "proposal_backward": case_proposal_backward,
         "resconv_tc": case_resconv_tc, "resconv": case_resconv}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--repeat", type=int, default=2)
    args = ap.parse_args(argv)
    CASES[args.case](args.repeat)
    torch.cuda.synchronize()
    print(f"{args.case}: ok")


if __name__ == "__main__":
    main()
