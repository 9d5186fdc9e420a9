"""Data parallelism over Monte Carlo chains (the only parallelism of the reference: the sample
axis is sharded over devices, ``code/README.md:53-56``; processes join through
``jax.distributed``, ``code/distributed.py:39-40``).

Each rank owns an independent block of chains and runs the whole hot path on its own GPU; the
only exchange is one all-reduce of FP64 (sum E, sum E^2, count) per sweep for the energy
estimate.  With NCCL this is a 24-byte all-reduce over NVLink; with gloo it runs on CPU.
"""

from __future__ import annotations

import os
from typing import Optional, Tuple

import torch
import torch.distributed as dist


def world() -> Tuple[int, int]:
    """(rank, world_size); (0, 1) when no process group is initialised."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard_chains(nsamples: int, rank: int, world_size: int) -> Tuple[int, int]:
    """(first chain, number of chains) of ``rank``: contiguous, sizes differ by at most one."""
    base, extra = divmod(int(nsamples), int(world_size))
    count = base + (1 if rank < extra else 0)
    start = rank * base + min(rank, extra)
    return start, count


def chain_seed(seed: int, rank: int) -> int:
    """Distinct Philox key per rank (the counter already carries the chain index)."""
    return (int(seed) + 0x9E3779B97F4A7C15 * (rank + 1)) & 0xFFFFFFFFFFFFFFFF


def energy_stats(eloc: torch.Tensor, N: int, group=None) -> dict:
    """Global E/N and sigma^2/N over all ranks' local energies with one FP64 all-reduce."""
    e = eloc.to(torch.float64)
    t = torch.stack([e.sum(), (e * e).sum(), torch.tensor(float(e.numel()), dtype=torch.float64,
                                                            device=e.device)])
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    s, s2, n = (float(x) for x in t.cpu())
    mean = s / n
    var = s2 / n - mean * mean
    return dict(E_per_site=mean / N, var_per_site=var / N, count=int(n))


def init_from_env(backend: Optional[str] = None, timeout_s: int = 120) -> bool:
    """Initialise the default process group from torchrun's environment (RANK, WORLD_SIZE,
    MASTER_ADDR, MASTER_PORT); returns False for a single process."""
    if int(os.environ.get("WORLD_SIZE", "1")) <= 1:
        return False
    if not dist.is_initialized():
        import datetime

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s))
    return True
