"""B200-native (sm_100a) Pfaffian-backflow VMC hot path: amplitudes, local energies and
Metropolis sampling of the periodic 2D Hubbard model through libnh_b200.so.

Drop-in surface (after ChenAo-Phys/NeuralHubbard's quantax usage):

    model = PfaffianBackflow(L, L, n_up, n_dn)           # code/backflow/models.py
    state = Variational(model, symm=True)                 # code/states.py:318-320
    psi = state(spins)                                    # psi.sign, psi.logabs
    H = Hubbard(U=8.0, t=[1.0, -0.2], n_neighbor=[1, 2])  # code/states.py:244-247
    eloc = H.Oloc(state, Samples(spins, psi))             # code/quick_start.py:33
    sampler = MixSampler([ParticleHop(state, 4096, n_neighbor=(1, 2)),  # code/states.py:397-408
                          SiteExchange(state, 4096, n_neighbor=(1, 2))])
    samples = sampler.sweep()

Learned proposal (new): HopProposal (network, GPU training), training_records (data from plain
chains) and LearnedHop (Metropolis with the exact Hastings correction).
"""

from ._lib import NativeLibraryError
from .backflow import (BCSBackflow, PairGeometry, PfaffianBackflow, build_wtilde, init_params,
                       pairing_occ, pairing_occ_vjp, slogpf, slogpf_adjoint)
from .operator import Hubbard
from .proposal import HopProposal, LearnedHop, training_records
from .sampler import MixSampler, ParticleHop, SiteExchange, random_spins
from .state import LogArray, Samples, Variational

__all__ = [
    "NativeLibraryError",
    "PairGeometry",
    "PfaffianBackflow",
    "BCSBackflow",
    "build_wtilde",
    "init_params",
    "pairing_occ",
    "pairing_occ_vjp",
    "slogpf_adjoint",
    "slogpf",
    "Hubbard",
    "HopProposal",
    "LearnedHop",
    "training_records",
    "ParticleHop",
    "SiteExchange",
    "MixSampler",
    "random_spins",
    "LogArray",
    "Samples",
    "Variational",
]
