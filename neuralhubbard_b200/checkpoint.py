"""Released Pfaffian-backflow states: parameter files (``weights/<name>.eqx``) and their
equilibrated chains (``weights/<name>_spins.npz``).

An ``.eqx`` file is equinox's ``tree_serialise_leaves`` output: the model's leaves in tree
order, each written as one ``.npy`` record (arrays and Python scalars alike), so it reads
with numpy alone.  For ``PfaffianBackflow(ResConv(...))`` (``code/backflow/models.py:120-151,
319-329``) the leaves are: the embedding's channel count, the embedding (C, 4, 1, 1), then
per residual block two (conv (C, C, 3, 3), bias (C, 1, 1)) pairs, the ResConv's static
fields (a flag, blocks, channels, kernel size), W (3, N, d), theta () and the zero pad.
The reference checks the file's md5 (``code/states.py:103-126,301-303``); ``RELEASED`` holds
those of the Pfaffian-backflow states with their published E/N and sigma^2/N
(``weights/README.md``).

Spin files hold ``bits = np.packbits(spins > 0, axis=-1)`` and ``shape`` (nchains, 2N)
(``code/states.py:328-352``).
"""

from __future__ import annotations

import hashlib
import io
from typing import NamedTuple, Optional

import numpy as np


class ReleasedState(NamedTuple):
    L: int
    tprime: float
    md5: str
    energy: float  # E/N of the projected state
    energy_err: float
    variance: float  # sigma^2 / N
    variance_err: float


RELEASED = {
    "tp0_L16_pfaffian": ReleasedState(16, 0.0, "17b770fe57367b09b27ad37538842ba0",
                                      -0.75813, 1e-5, 0.0259, 0.0002),
    "tpm02_L16_pfaffian": ReleasedState(16, -0.2, "aef48e8b7c10cfa183f8c0e8dcf84d06",
                                        -0.74533, 1e-5, 0.0272, 0.0005),
    "tpm02_L24_pfaffian": ReleasedState(24, -0.2, "17653481d380416e6df7033ba7902aee",
                                        -0.74585, 1e-5, 0.0257, 0.0003),
    "tpm02_L32_pfaffian": ReleasedState(32, -0.2, "83a4eb0c591b893e29b451c7b95cb0b1",
                                        -0.74569, 1e-5, 0.0294, 0.0005),
}


class CheckpointError(ValueError):
    """The file does not have the layout of a Pfaffian-backflow ResConv checkpoint."""


def read_leaves(path: str) -> list:
    """All ``.npy`` records of an equinox leaf file, in order."""
    raw = open(path, "rb").read()
    f = io.BytesIO(raw)
    leaves = []
    while f.tell() < len(raw):
        leaves.append(np.lib.format.read_array(f, allow_pickle=False))
    return leaves


def file_md5(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.md5(f.read()).hexdigest()


def load_pfaffian_backflow(path: str, L: Optional[int] = None,
                           expect_md5: Optional[str] = None) -> dict:
    """Parameters of a released Pfaffian-backflow state as the dict ``PfaffianBackflow``
    takes: ``net="resconv"``, ``embed`` (C, 4), ``conv_w`` / ``conv_b`` (2 * blocks arrays,
    block order), ``W`` (3, N, d), ``theta``.  ``L`` checks the lattice size; ``expect_md5``
    (e.g. ``RELEASED[name].md5``) checks the file's checksum first, as the reference does
    before loading (``code/states.py:308-311``), and raises ``CheckpointError`` on a mismatch."""
    if expect_md5 is not None:
        got = file_md5(path)
        if got != expect_md5:
            raise CheckpointError(f"{path}: md5 {got}, expected {expect_md5}")
    leaves = read_leaves(path)
    floats = [a for a in leaves if a.dtype == np.float32]
    if len(floats) < 5 or floats[0].ndim != 4 or floats[0].shape[1:] != (4, 1, 1):
        raise CheckpointError(f"{path}: no (C, 4, 1, 1) occupation embedding first")
    embed = floats[0][:, :, 0, 0]
    C = embed.shape[0]
    convs = floats[1:-3]
    if len(convs) % 2 or not convs:
        raise CheckpointError(f"{path}: odd number of convolution leaves")
    conv_w, conv_b = [], []
    for w, b in zip(convs[0::2], convs[1::2]):
        if w.shape != (C, C, 3, 3) or b.shape != (C, 1, 1):
            raise CheckpointError(f"{path}: convolution leaf shapes {w.shape}, {b.shape}")
        conv_w.append(np.ascontiguousarray(w))
        conv_b.append(np.ascontiguousarray(b[:, 0, 0]))
    W, theta, pad = floats[-3:]
    N = W.shape[1] if W.ndim == 3 else -1
    if W.ndim != 3 or W.shape[0] != 3 or W.shape[2] * 2 != C or theta.shape != () \
            or pad.ndim != 1 or np.any(pad != 0):
        raise CheckpointError(f"{path}: W {W.shape}, theta {theta.shape}, pad {pad.shape}")
    Lc = int(round(np.sqrt(N)))
    if Lc * Lc != N or (L is not None and L != Lc):
        raise CheckpointError(f"{path}: W holds {N} sites, not an L x L lattice with L = {L}")
    ints = [int(a) for a in leaves if a.dtype == np.int64]
    if len(conv_w) // 2 not in ints or C not in ints:
        raise CheckpointError(f"{path}: static fields {ints} do not name {len(conv_w) // 2} "
                              f"blocks of {C} channels")
    return dict(net="resconv", embed=np.ascontiguousarray(embed), conv_w=conv_w,
                conv_b=conv_b, W=np.ascontiguousarray(W), theta=float(theta))


def load_spins(path: str, N: Optional[int] = None, n_up: Optional[int] = None,
               n_dn: Optional[int] = None) -> np.ndarray:
    """Equilibrated chains as int8 +-1 (nchains, 2N), spin-up sites first.  With ``n_up`` /
    ``n_dn`` every chain's particle numbers are checked, as the reference does for its stored
    chains (``code/states.py:346-351``); a mismatch raises ``CheckpointError``."""
    with np.load(path) as f:
        bits, shape = f["bits"], tuple(int(x) for x in f["shape"])
    s = np.unpackbits(bits, axis=-1, count=shape[-1]).astype(np.int8)
    s = (2 * s - 1).reshape(shape)
    if N is not None and s.shape[1] != 2 * N:
        raise CheckpointError(f"{path}: configurations of length {s.shape[1]}, not {2 * N}")
    half = s.shape[1] // 2
    for want, part, name in ((n_up, s[:, :half], "up"), (n_dn, s[:, half:], "down")):
        if want is None:
            continue
        got = (part > 0).sum(1)
        bad = np.nonzero(got != want)[0]
        if bad.size:
            raise CheckpointError(f"{path}: chain {int(bad[0])} holds {int(got[bad[0]])} spin-"
                                  f"{name} electrons, not {want} ({bad.size} chains differ)")
    return s
