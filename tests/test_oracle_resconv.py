"""CPU checks of the released-state loader (equinox leaf files, packed spins) and of the residual
network oracle (translation equivariance, RMSNorm scale invariance of the blocks' input)."""

import os

import numpy as np
import pytest

from neuralhubbard_b200 import checkpoint
from oracle import lattice as olat
from oracle import resconv as orc

RELEASED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "released")


def write_leaves(path, leaves):
    with open(path, "wb") as f:
        for a in leaves:
            np.save(f, np.asarray(a))


def synthetic_leaves(rng, C=64, blocks=2, N=16, d=32):
    conv = []
    for _ in range(2 * blocks):
        conv += [rng.normal(size=(C, C, 3, 3)).astype(np.float32),
                 rng.normal(size=(C, 1, 1)).astype(np.float32)]
    return ([np.int64(C), rng.normal(size=(C, 4, 1, 1)).astype(np.float32)] + conv +
            [np.bool_(False), np.int64(blocks), np.int64(C), np.int64(3), np.int64(3),
             rng.normal(size=(3, N, d)).astype(np.float32), np.float32(-0.7),
             np.zeros(1791, np.float32)])


def test_checkpoint_reads_leaf_file(tmp_path):
    rng = np.random.default_rng(0)
    leaves = synthetic_leaves(rng)
    path = str(tmp_path / "state.eqx")
    write_leaves(path, leaves)
    p = checkpoint.load_pfaffian_backflow(path, 4)
    assert p["net"] == "resconv" and len(p["conv_w"]) == 4 and len(p["conv_b"]) == 4
    assert np.array_equal(p["embed"], leaves[1][:, :, 0, 0])
    assert np.array_equal(p["conv_w"][3], leaves[8]) and np.array_equal(p["conv_b"][3],
                                                                        leaves[9][:, 0, 0])
    assert p["W"].shape == (3, 16, 32) and p["theta"] == pytest.approx(-0.7)
    with pytest.raises(checkpoint.CheckpointError):
        checkpoint.load_pfaffian_backflow(path, 8)  # W holds a 4 x 4 lattice
    write_leaves(path, leaves[:-2] + [np.float32(0.1), np.ones(3, np.float32)])
    with pytest.raises(checkpoint.CheckpointError):  # non-zero pad
        checkpoint.load_pfaffian_backflow(path, 4)


def test_spins_round_trip(tmp_path):
    s = olat.random_configs(np.random.default_rng(1), 5, 16, 7, 7)
    path = str(tmp_path / "spins.npz")
    np.savez(path, bits=np.packbits(s > 0, axis=-1), shape=np.array(s.shape))
    assert np.array_equal(checkpoint.load_spins(path, 16), s)


def test_released_checkpoint():
    eqx = os.path.join(RELEASED, "tpm02_L16_pfaffian.eqx")
    if not os.path.exists(eqx):
        pytest.skip("released weights not fetched (tests/golden/fetch_released.py)")
    assert checkpoint.file_md5(eqx) == checkpoint.RELEASED["tpm02_L16_pfaffian"].md5
    p = checkpoint.load_pfaffian_backflow(eqx, 16)
    n = p["embed"].size + sum(w.size + b.size for w, b in zip(p["conv_w"], p["conv_b"]))
    assert n + p["W"].size + 1 + 1791 == 1208320  # code/states.py:_TABLE nparams
    s = checkpoint.load_spins(os.path.join(RELEASED, "tpm02_L16_pfaffian_spins.npz"), 256)
    assert s.shape == (8192, 512)
    assert np.all((s[:, :256] > 0).sum(1) == 112) and np.all((s[:, 256:] > 0).sum(1) == 112)


def test_resconv_translation_equivariance():
    """Shifting the configuration by a lattice translation shifts the features."""
    rng = np.random.default_rng(2)
    L, C = 6, 64
    embed = rng.normal(size=(C, 4))
    conv_w = [rng.normal(size=(C, C, 3, 3)) * 0.04 for _ in range(4)]
    conv_b = [rng.normal(size=C) * 0.1 for _ in range(4)]
    s = olat.random_configs(rng, 2, L * L, 10, 10)
    y = orc.resconv_forward(s, embed, conv_w, conv_b, L, L)
    img = s.reshape(2, 2, L, L)
    st = np.roll(img, shift=(2, 5), axis=(2, 3)).reshape(2, -1)
    yt = orc.resconv_forward(st, embed, conv_w, conv_b, L, L)
    yr = np.roll(y.reshape(2, 2, L, L, C // 2), shift=(2, 5), axis=(2, 3)).reshape(y.shape)
    assert np.allclose(yt, yr, atol=1e-12)


def test_occupation_index():
    s = np.array([[1, -1, 1, -1, -1, 1, 1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                   1, 1, -1, -1, -1, -1, 1, -1, -1, -1, -1, -1, -1, -1, -1, -1]], np.int8)
    occ = orc.occupation_index(s, 4, 4).ravel()
    assert list(occ[:8]) == [3, 2, 1, 0, 0, 1, 3, 0]
