"""Generate the committed golden fixtures of this directory.

    python tests/golden/make_golden.py

The reference (JAX + quantax + fermix) cannot run in this image, so the fixtures come from
sources that do not depend on the oracle's own algorithms:

* ``philox_kat.json``   the published Philox4x32-10 known-answer vectors of Random123
                        (Salmon et al., SC'11), written out by hand below;
* ``pfaffian_kat.npz``  small antisymmetric matrices with Pfaffians from the definition
                        (sum over perfect matchings), independent of Parlett-Reid;
* ``hubbard_4x4.npz``   <s|H|s'> rows of a 4x4 periodic lattice (t = 1, t' = -0.2, U = 8,
                        2 + 2 electrons) from explicit fermion operators on the Fock basis,
                        independent of the hop enumeration;
* ``oracle_amplitude_L4.npz``  regression pins of the oracle's own amplitudes (4x4 lattice,
                        seeded parameters), so that a change of the oracle is visible.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import backflow, hubbard, lattice, pfaffian, projection  # noqa: E402

PHILOX_KAT = [
    {"counter": [0, 0, 0, 0], "key": [0, 0],
     "out": [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]},
    {"counter": [0xFFFFFFFF] * 4, "key": [0xFFFFFFFF] * 2,
     "out": [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]},
    {"counter": [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], "key": [0xA4093822, 0x299F31D0],
     "out": [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]},
]


def seeded_params(L: int, channels: int, seed: int, std: float) -> dict:
    rng = np.random.default_rng(seed)
    conv_w, conv_b = [], []
    cin = 2
    for _ in range(4):
        conv_w.append(rng.normal(0.0, std, (channels, cin, 3, 3)))
        conv_b.append(rng.normal(0.0, std, (channels,)))
        cin = channels
    d = channels // 2
    W = rng.normal(0.0, 1.0, (3, L * L, d)) / np.sqrt(d)
    return dict(conv_w=conv_w, conv_b=conv_b, W=W, theta=0.55, Lx=L, Ly=L)


def main():
    with open(os.path.join(HERE, "philox_kat.json"), "w") as f:
        json.dump(PHILOX_KAT, f, indent=1)

    rng = np.random.default_rng(2024)
    mats, pfs = [], []
    for n in (2, 4, 6, 8):
        for _ in range(3):
            A = rng.normal(size=(n, n))
            A = A - A.T
            A8 = np.zeros((8, 8))
            A8[:n, :n] = A
            mats.append(A8)
            pfs.append(pfaffian.pf_permutation_sum(A))
    sizes = np.repeat([2, 4, 6, 8], 3)
    np.savez(os.path.join(HERE, "pfaffian_kat.npz"), A=np.array(mats), n=sizes, pf=np.array(pfs))

    basis = hubbard.fock_basis(16, 2, 2)
    H = hubbard.hamiltonian_matrix(basis, 4, 4, 1.0, -0.2, 8.0)
    pick = rng.choice(len(basis), 64, replace=False)
    rows = []
    for a in pick:
        nz = np.flatnonzero(H[a])
        rows.append([(int(j), float(H[a, j])) for j in nz])
    flat_j = np.concatenate([[j for j, _ in r] for r in rows])
    flat_v = np.concatenate([[v for _, v in r] for r in rows])
    counts = np.array([len(r) for r in rows])
    np.savez_compressed(os.path.join(HERE, "hubbard_4x4.npz"), spins=basis[pick], counts=counts,
                        conn=basis[flat_j.astype(np.int64)], vals=flat_v)

    params = seeded_params(4, 16, 7, 0.3)
    s = lattice.random_configs(np.random.default_rng(11), 6, 16, 7, 7)
    sg, la = backflow.amplitude(s, params)
    sgp, lap = projection.projected_amplitude(s, params)
    np.savez(os.path.join(HERE, "oracle_amplitude_L4.npz"), spins=s, sign=sg, logabs=la,
             sign_p=sgp, logabs_p=lap)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
