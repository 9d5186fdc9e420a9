"""The allocation-free log-Pfaffian entry point (nh_slogpf_noalloc).

Some callers of this library cannot allocate device memory: they are handed only their input and
output buffers (for example by a host runtime that owns all device memory and gives a plugin no
workspace), or they must avoid cudaMalloc because it can synchronise the device.  For them
nh_slogpf_noalloc keeps its refinement scratch in a static device array instead of a caller
workspace.  This test calls it through the C ABI twice in a row and compares with nh_slogpf
(which takes a workspace).  It sits in its own file, collected last, so that a failure here
leaves every other test already run.
"""

import ctypes

import numpy as np
import pytest
import torch

from neuralhubbard_b200 import _lib

pytestmark = pytest.mark.gpu


def _batch(rng, n, B):
    A = rng.normal(size=(B, n, n)).astype(np.float32)
    A = A - np.swapaxes(A, 1, 2)
    # a few near-nodal matrices so that the FP64 refinement list is not empty
    Q = np.linalg.qr(rng.normal(size=(4, n, n)))[0]
    blocks = np.zeros((4, n, n))
    a = rng.uniform(0.5, 2.0, size=(4, n // 2))
    a[:, 3] *= 1e-6
    for k in range(n // 2):
        blocks[:, 2 * k, 2 * k + 1], blocks[:, 2 * k + 1, 2 * k] = a[:, k], -a[:, k]
    near = np.einsum("bji,bjk,bkl->bil", Q, blocks, Q).astype(np.float32)
    A[:4] = 0.5 * (near - np.swapaxes(near, 1, 2))
    return A


def _run(fn_name, F, n, B, tau, with_ws):
    lib = _lib.load()
    dev = F.device
    sign = torch.empty(B, dtype=torch.float32, device=dev)
    logabs = torch.empty(B, dtype=torch.float64, device=dev)
    flags = torch.empty(B, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    if with_ws:
        ws = torch.empty(lib.nh_slogpf_workspace_bytes(n, B), dtype=torch.uint8, device=dev)
        rc = lib.nh_slogpf(F.data_ptr(), n, B, tau, sign.data_ptr(), logabs.data_ptr(),
                           flags.data_ptr(), ws.data_ptr(), ws.numel(), st)
    else:
        rc = lib.nh_slogpf_noalloc(F.data_ptr(), n, B, tau, sign.data_ptr(), logabs.data_ptr(),
                                   flags.data_ptr(), st)
    _lib.check(rc, fn_name)
    torch.cuda.synchronize()
    return sign.cpu().numpy(), logabs.cpu().numpy(), flags.cpu().numpy()


@pytest.mark.parametrize("n,B", [(56, 300), (224, 40)])
def test_noalloc_matches_workspace_entry_point(n, B):
    rng = np.random.default_rng(n)
    F = torch.from_numpy(_batch(rng, n, B)).cuda()
    s0, l0, f0 = _run("nh_slogpf", F, n, B, 100.0, True)
    assert (f0 & _lib.FLAG_REFINED).any()
    for _ in range(2):  # two calls in a row share and overwrite the static scratch
        s1, l1, f1 = _run("nh_slogpf_noalloc", F, n, B, 100.0, False)
        assert np.array_equal(s1, s0)
        assert np.allclose(l1, l0, rtol=0, atol=1e-9)
        assert np.array_equal(f1, f0)


def test_noalloc_rejects_oversized_batch():
    lib = _lib.load()
    B = 65536 + 1
    rc = lib.nh_slogpf_noalloc(ctypes.c_void_p(8), 4, B, 100.0, ctypes.c_void_p(8),
                               ctypes.c_void_p(8), ctypes.c_void_p(8), None)
    assert rc == -2
    assert b"exceeds the static scratch limit" in lib.nh_last_error()


def test_noalloc_rejects_large_n():
    """Triangles beyond shared memory need workspace: n > 256 is refused with a pointer to
    nh_slogpf."""
    lib = _lib.load()
    rc = lib.nh_slogpf_noalloc(ctypes.c_void_p(8), 300, 4, 100.0, ctypes.c_void_p(8),
                               ctypes.c_void_p(8), ctypes.c_void_p(8), None)
    assert rc == -2
    assert b"nh_slogpf with a workspace" in lib.nh_last_error()


def test_noalloc_beyond_fp64_shared_memory_keeps_fp32():
    """For 236 < n <= 256 an FP64 triangle no longer fits in shared memory and this entry point
    has no workspace for one: ill-conditioned matrices are flagged NH_FLAG_GROWTH but keep their
    FP32 result (no NH_FLAG_REFINED), bit for bit the result of nh_slogpf without refinement."""
    n, B = 240, 8
    rng = np.random.default_rng(n)
    F = torch.from_numpy(_batch(rng, n, B)).cuda()
    s0, l0, _ = _run("nh_slogpf", F, n, B, 0.0, True)
    for _ in range(2):
        s1, l1, f1 = _run("nh_slogpf_noalloc", F, n, B, 100.0, False)
        assert np.all(f1[:4] & _lib.FLAG_GROWTH)  # the four near-nodal matrices
        assert not np.any(f1 & _lib.FLAG_REFINED)
        assert np.array_equal(s1, s0)
        assert np.array_equal(l1, l0)
