"""Projected energy per site of a released state on its stored equilibrated chains, through the
library's public API (the check that pins the reference's conventions end to end: the published
E/N of ``code/states.py:103-126`` / ``weights/README.md``).

    python tests/golden/released_energy.py [--name tpm02_L16_pfaffian] [--chains N]
                                           [--cnn-mode 2] [--save eloc.npy]

The released files must have been copied with ``tests/golden/fetch_released.py``.  Prints one
JSON line per batch of chains (running mean, its standard error, sigma^2/N, seconds) and a last
line with the published values and the distance in standard errors.  All 8192 chains of
``tpm02_L16_pfaffian`` take about 17 minutes on one B200 with the tensor-core form.
"""

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402
import torch  # noqa: E402

import neuralhubbard_b200 as nh  # noqa: E402
from neuralhubbard_b200 import checkpoint  # noqa: E402


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--name", default="tpm02_L16_pfaffian")
    ap.add_argument("--chains", type=int, default=0, help="0: all stored chains")
    ap.add_argument("--batch", type=int, default=0,
                    help="chains per call; 0: 1024 at 16x16, 64 on larger lattices")
    ap.add_argument("--cnn-mode", type=int, default=None, choices=[0, 2],
                    help="2 (tcgen05 residual network, 16x16 only) or 0; default 2 at 16x16")
    ap.add_argument("--released-dir", default=os.path.join(HERE, "released"))
    ap.add_argument("--save", default=None, help="write the per-chain E_loc / N here (.npy)")
    args = ap.parse_args()

    info = checkpoint.RELEASED[args.name]
    L = info.L
    N = L * L
    ne = 7 * N // 16
    base = os.path.join(args.released_dir, args.name)
    params = checkpoint.load_pfaffian_backflow(base + ".eqx", L, expect_md5=info.md5)
    spins = checkpoint.load_spins(base + "_spins.npz", N, ne, ne)
    if args.chains:
        spins = spins[:args.chains]
    cnn_mode = args.cnn_mode if args.cnn_mode is not None else (2 if L == 16 else 0)
    batch = args.batch or (1024 if L == 16 else 64)
    oloc_kw = {} if L == 16 else {"chunk_configs": 2048}
    state = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=cnn_mode))
    H = nh.Hubbard(8.0, [1.0, info.tprime], [1, 2])
    out = []
    t0 = time.time()
    for c0 in range(0, spins.shape[0], batch):
        s = torch.from_numpy(spins[c0:c0 + batch]).cuda()
        out.append(H.Oloc(state, nh.Samples(s, state(s)), **oloc_kw).cpu().numpy() / N)
        a = np.concatenate(out)
        print(json.dumps(dict(chains=len(a), mean=float(a.mean()),
                              err=float(a.std(ddof=1) / np.sqrt(len(a))),
                              var_per_site=float(a.var(ddof=1) * N),
                              seconds=time.time() - t0)), flush=True)
    a = np.concatenate(out)
    err = float(a.std(ddof=1) / np.sqrt(len(a)))
    print(json.dumps(dict(name=args.name, chains=len(a), mean=float(a.mean()), err=err,
                          published=info.energy, published_var_per_site=info.variance,
                          sigmas=float((a.mean() - info.energy) / err))))
    if args.save:
        np.save(args.save, a)


if __name__ == "__main__":
    main()
