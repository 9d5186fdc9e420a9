"""Host-side checks that need no GPU: the C-ABI library loads and exports every symbol of
include/nh_b200.h, the ctypes table matches the header, and the chain-parallel statistics work
across two gloo ranks."""

import ctypes
import os
import re
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nh_b200.h")
LIB = os.path.join(ROOT, "neuralhubbard_b200", "libnh_b200.so")


def header_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nh_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    if not os.path.exists(LIB):
        pytest.skip("libnh_b200.so not built")
    lib = ctypes.CDLL(LIB)  # loads without a GPU: no compute call is made
    syms = header_symbols()
    assert len(syms) >= 13
    for s in syms:
        assert hasattr(lib, s), s
    lib.nh_abi_version.restype = ctypes.c_int
    want = int(re.search(r"#define NH_ABI_VERSION (\d+)", open(HEADER).read()).group(1))
    assert lib.nh_abi_version() == want


def header_arg_counts():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for name, args in re.findall(r"\b(nh_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        args = " ".join(args.split())
        out[name] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_ctypes_table_matches_header():
    from neuralhubbard_b200 import _lib

    assert sorted(_lib.SIGNATURES) == header_symbols()
    counts = header_arg_counts()
    for name, (_, argtypes) in _lib.SIGNATURES.items():
        assert len(argtypes) == counts[name], name


def test_argument_checks_before_device_work():
    """Entry points refuse bad sizes, missing buffers and bad workspaces with the documented
    status and message before touching the device (fake, never-dereferenced pointers)."""
    if not os.path.exists(LIB):
        pytest.skip("libnh_b200.so not built")
    from neuralhubbard_b200 import _lib

    lib = _lib.load()
    p = ctypes.c_void_p(4096)

    def slogpf(n, flags=p, ws=p, nbytes=1 << 26, tau=100.0):
        return lib.nh_slogpf(p, n, 4, tau, p, p, flags, ws, nbytes, None)

    assert slogpf(7) == -2 and b"must be even" in lib.nh_last_error()
    assert slogpf(1026) == -2
    assert lib.nh_slogpf(None, 56, 4, 100.0, p, p, p, p, 1 << 26, None) == -1
    assert slogpf(56, flags=None) == -1 and b"needs flags" in lib.nh_last_error()
    assert slogpf(56, nbytes=16) == -4
    assert slogpf(56, ws=None) == -4
    assert slogpf(56, ws=ctypes.c_void_p(4096 + 16)) == -1
    assert b"256-byte aligned" in lib.nh_last_error()
    assert lib.nh_slogpf_noalloc(p, 300, 4, 100.0, p, p, p, None) == -2
    # 256-byte granularity: one and two matrices need the same workspace, more need more
    assert lib.nh_slogpf_workspace_bytes(56, 1) == lib.nh_slogpf_workspace_bytes(56, 2)
    assert lib.nh_slogpf_workspace_bytes(56, 65) > lib.nh_slogpf_workspace_bytes(56, 64)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from neuralhubbard_b200 import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(_lib.NativeLibraryError):
        _lib.load()


def test_shard_chains_cover():
    from neuralhubbard_b200.distributed import shard_chains

    for n, w in [(10, 3), (8192, 8), (5, 8)]:
        parts = [shard_chains(n, r, w) for r in range(w)]
        assert sum(c for _, c in parts) == n
        assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(w - 1))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from neuralhubbard_b200.distributed import energy_stats, shard_chains

    rng = np.random.default_rng(0)
    e_all = torch.from_numpy(rng.normal(-0.7, 0.1, 1000))
    s, c = shard_chains(1000, rank, world)
    st = energy_stats(e_all[s : s + c], N=1)
    out[rank] = (st["E_per_site"], st["var_per_site"], st["count"])
    dist.barrier()
    dist.destroy_process_group()


def test_energy_stats_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    e_all = np.random.default_rng(0).normal(-0.7, 0.1, 1000)
    for r in range(2):
        m, v, n = out[r]
        assert n == 1000
        assert m == pytest.approx(e_all.mean(), abs=1e-12)
        assert v == pytest.approx(e_all.var(), rel=1e-9)


def test_tau_int_matches_oracle_and_ar1():
    """The package's chain statistics against the oracle's and the AR(1) closed form
    tau = (1 + phi) / (2 (1 - phi))."""
    from neuralhubbard_b200 import stats
    from oracle import sampler as osam

    rng = np.random.default_rng(0)
    phi, T, B = 0.8, 4000, 64
    x = np.zeros((T, B))
    e = rng.normal(size=(T, B))
    for t in range(1, T):
        x[t] = phi * x[t - 1] + e[t]
    tau = stats.tau_int(x)
    assert abs(tau - osam.tau_int(x)) < 1e-12
    assert abs(tau - (1 + phi) / (2 * (1 - phi))) < 0.25
    m, err = stats.jackknife_mean(x[:, 0])
    m0, err0 = osam.jackknife_mean(x[:, 0])
    assert m == m0 and abs(err - err0) < 1e-12
    assert stats.effective_rate(64, 4000, 0.5, 2.0) == 64 * 4000 / 2.0


def test_tau_int_error_bars_cover_ar1():
    """The error bars of tau_int: across 12 seeds of an AR(1) ensemble the estimate lies within
    3 (group-spread) error bars of the closed form, with the window's small downward bias
    included, and the two error estimates agree within a factor of 4."""
    from neuralhubbard_b200 import stats

    phi, T, B = 0.8, 2000, 128
    exact = (1 + phi) / (2 * (1 - phi))
    for seed in range(12):
        rng = np.random.default_rng(100 + seed)
        x = np.zeros((T, B))
        e = rng.normal(size=(T, B))
        for t in range(1, T):
            x[t] = phi * x[t - 1] + e[t]
        te = stats.tau_int_error(x)
        assert te["tau"] == stats.tau_int(x)
        assert te["window"] >= 5 * te["tau"]
        assert abs(te["tau"] - exact) < 3 * te["err_groups"] + 0.15, (seed, te)
        assert 0.25 < te["err_groups"] / te["err_sokal"] < 4.0, te
    assert stats.tau_int_error(np.zeros((100, 4)))["err_groups"] is None


def test_residual_network_argument_checks():
    """Packing sizes and the parameter checks of the residual network (net = NH_NET_RESCONV),
    all decided before any device work."""
    if not os.path.exists(LIB):
        pytest.skip("libnh_b200.so not built")
    from neuralhubbard_b200 import _lib

    lib = _lib.load()
    p8 = ctypes.c_void_p(4096)
    assert lib.nh_pack_resconv_weights_floats(64, 16) == 4 * 64 + 32 * 9 * 64 * 64
    assert lib.nh_pack_resconv_weights_tc_bytes(16) == 32 * 9 * 2 * 64 * 64 * 2
    assert lib.nh_pack_resconv_weights(p8, 32, 16, p8, None) == -2
    assert lib.nh_pack_resconv_weights(None, 64, 16, p8, None) == -1
    assert lib.nh_pack_resconv_weights_tc(p8, 48, 16, p8, None) == -2

    def amplitude(**kw):
        f = dict(conv_w=4096, conv_b=4096, conv_w_packed=4096, conv_w_tc=4096, Wt=4096,
                 Wt64=4096, Lx=16, Ly=16, n_up=112, n_dn=112, channels=64, layers=16,
                 cnn_mode=0, pf_mode=0, net=_lib.NET_RESCONV, ansatz=0, cond_tau=100.0,
                 cancel_tau=8.0)
        f.update(kw)
        prm = _lib.BackflowParams(**f)
        return lib.nh_amplitude(p8, 4, 8, ctypes.byref(prm), p8, p8, p8, p8, 1 << 30, None)

    assert amplitude(channels=32) == -2 and b"64 channels" in lib.nh_last_error()
    assert amplitude(cnn_mode=1) == -2
    assert amplitude(cnn_mode=2, Lx=8, Ly=8, n_up=28, n_dn=28) == -2
    assert amplitude(net=7) == -1 and b"net 7" in lib.nh_last_error()
    assert amplitude(ansatz=5) == -1 and b"ansatz 5" in lib.nh_last_error()
    # BCS ansatz: equal spin numbers, d = 16, no tensor-memory Pfaffian
    assert amplitude(net=_lib.NET_CNN, channels=32, layers=4, ansatz=_lib.ANSATZ_BCS,
                     n_dn=110) == -2 and b"BCS" in lib.nh_last_error()
    assert amplitude(net=_lib.NET_CNN, channels=32, layers=4, ansatz=_lib.ANSATZ_BCS,
                     pf_mode=1) == -2


def test_timeout_flag_raises():
    """NH_FLAG_TIMEOUT (a tensor-core kernel's bounded wait expired; the combination folds the
    device error word into every output flag) must surface as an exception in the host layer,
    and flags without it must pass."""
    import numpy as np

    from neuralhubbard_b200 import _lib

    ok = np.array([0, _lib.FLAG_REFINED, _lib.FLAG_GROWTH | _lib.FLAG_CANCEL], np.int32)
    _lib.check_flags(ok, "test")
    assert not _lib.timeout_flagged(ok)
    bad = ok | _lib.FLAG_TIMEOUT
    assert _lib.timeout_flagged(bad)
    with pytest.raises(_lib.DeviceTimeoutError):
        _lib.check_flags(bad, "test")
    import torch

    with pytest.raises(_lib.DeviceTimeoutError):
        _lib.check_flags(torch.from_numpy(bad), "test")


def test_new_entry_points_validate_arguments_without_a_gpu():
    """The backward, BCS and observable entry points reject bad arguments before any device
    work (status codes and nh_last_error; no CUDA call is made)."""
    import ctypes

    from neuralhubbard_b200 import _lib

    lib = _lib.load()
    p8 = ctypes.c_void_p(4096)
    assert lib.nh_pfaffian_adjoint(p8, 7, 4, p8, None, None) == -2  # odd n
    assert lib.nh_pfaffian_adjoint(p8, 226, 4, p8, None, None) == -2  # beyond 224
    assert lib.nh_pfaffian_adjoint(None, 8, 4, p8, None, None) == -1
    assert lib.nh_pairing_occ_vjp(p8, p8, p8, p8, 24, 24, 16, 100, 2, p8, p8, None) == -2

    def prm(**kw):
        f = dict(conv_w=4096, conv_b=4096, conv_w_packed=4096, conv_w_tc=4096, Wt=4096,
                 Wt64=4096, Lx=8, Ly=8, n_up=28, n_dn=28, channels=32, layers=4, cnn_mode=0,
                 pf_mode=0, net=_lib.NET_CNN, ansatz=_lib.ANSATZ_PFAFFIAN, cond_tau=5.0,
                 cancel_tau=8.0, refine_tau=0.0, delta_d=0.0)
        f.update(kw)
        return _lib.BackflowParams(**f)

    p = prm()
    assert lib.nh_param_count(ctypes.byref(p)) == (32 * 2 * 9 + 32) + 3 * (32 * 32 * 9 + 32) \
        + 3 * 64 * 16 + 1
    assert lib.nh_param_count(ctypes.byref(prm(net=_lib.NET_RESCONV))) == 0
    bcs = prm(ansatz=_lib.ANSATZ_BCS)
    rc = lib.nh_log_jacobian(p8, 4, 8, ctypes.byref(bcs), p8, 0.55, p8, p8, p8, None, p8,
                             1 << 30, None)
    assert rc == -2 and b"log_jacobian" in lib.nh_last_error()
    rc = lib.nh_log_jacobian(p8, 4, 3, ctypes.byref(p), p8, 0.55, p8, p8, p8, None, p8, 1 << 30,
                             None)
    assert rc == -1  # n_symm must be 1 or 8

    def obs(kind, a0, a1, **kw):
        q = prm(**kw)
        return lib.nh_observable(p8, p8, p8, 4, 8, ctypes.byref(q), kind, a0, a1, p8, p8,
                                 1 << 30, None)

    assert obs(7, 0, 0) == -1 and b"kind 7" in lib.nh_last_error()
    assert obs(_lib.OBS_TRANSVERSE_SPIN, 64, 0) == -1  # site beyond the 8x8 lattice
    assert obs(_lib.OBS_PAIR, 3, -1) == -1
    assert obs(_lib.OBS_HOP, 3, 2) == -1  # spin must be 0 or 1
    assert lib.nh_observable_workspace_bytes(4, 8, 9, ctypes.byref(p)) == 0
    assert lib.nh_observable_workspace_bytes(4, 8, _lib.OBS_PAIR, ctypes.byref(p)) > 0
