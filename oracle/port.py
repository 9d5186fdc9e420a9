"""ctypes wrapper of the compiled CPU restatement (``oracle/c/nh_port.c``).

TEST INFRASTRUCTURE / CPU BASELINE ONLY, like the rest of ``oracle``: it computes the same
projected amplitudes as ``oracle.projection.projected_amplitude`` (checked against it in
``tests/test_oracle_port.py``), in C with OpenMP across configurations, so that the CPU baseline
of ``bench.py`` runs the algorithm at compiled speed on all host cores.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import backflow, lattice

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "c", "nh_port.c")
# Two builds: portable x86-64 (SSE4.2) and AVX2 + FMA; the loader takes the second only on hosts
# whose /proc/cpuinfo lists those instruction sets (the built files travel to other hosts).
LIBS = {"x86-64-v2": os.path.join(HERE, "libnh_port.so"),
        "x86-64-v3": os.path.join(HERE, "libnh_port_avx2.so")}
# The FP32 builds (-DNHP_FP32): the same algorithm in float, the arithmetic of the reference's own
# JAX path, for a like-for-like CPU baseline.
LIBS32 = {"x86-64-v2": os.path.join(HERE, "libnh_port_f32.so"),
          "x86-64-v3": os.path.join(HERE, "libnh_port_f32_avx2.so")}
CFLAGS = ["-O3", "-fopenmp", "-fPIC", "-shared"]

_lib = None
_lib32 = None


def build(force: bool = False) -> None:
    """Compile the C restatement with gcc into ``oracle/libnh_port*.so`` (FP64 and FP32)."""
    for libs, extra in ((LIBS, []), (LIBS32, ["-DNHP_FP32"])):
        for march, lib in libs.items():
            if force or not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(SRC):
                subprocess.check_call(["gcc", *CFLAGS, *extra, f"-march={march}", SRC, "-o", lib,
                                       "-lm"])


def _host_has_avx2_fma() -> bool:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return all(f" {f}" in flags for f in ("avx2", "fma", "bmi2", "movbe"))


def load(fp32: bool = False):
    """The compiled library (FP64, or the FP32 build) for this host's instruction set."""
    global _lib, _lib32
    if (_lib32 if fp32 else _lib) is None:
        build()
        march = "x86-64-v3" if _host_has_avx2_fma() else "x86-64-v2"
        lib = ctypes.CDLL((LIBS32 if fp32 else LIBS)[march])
        fn = lib.nhp_amplitudes_f32 if fp32 else lib.nhp_amplitudes
        p = ctypes.c_void_p
        fn.restype = ctypes.c_int
        fn.argtypes = [p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                       p, p, p, ctypes.c_int, p, ctypes.c_int, p, p, ctypes.c_int]
        if fp32:
            _lib32 = lib
        else:
            _lib = lib
    return _lib32 if fp32 else _lib


def projected_amplitude(s: np.ndarray, params: dict, symm: bool = True, threads: int = 0,
                        fp32: bool = False):
    """(sign, logabs) of psi_P(s) (or psi(s) when ``symm`` is False) for s (B, 2N), FP64 (or
    the FP32 build's arithmetic with ``fp32``); the
    same ``params`` dict as the numpy oracle (conv_w, conv_b lists, W, theta, Lx, Ly)."""
    lib = load(fp32)
    fn = lib.nhp_amplitudes_f32 if fp32 else lib.nhp_amplitudes
    s = np.ascontiguousarray(s, dtype=np.int8)
    B, M = s.shape
    Lx, Ly = params["Lx"], params["Ly"]
    conv_w = np.ascontiguousarray(np.concatenate([np.asarray(w, np.float64).ravel()
                                                  for w in params["conv_w"]]))
    conv_b = np.ascontiguousarray(np.concatenate([np.asarray(b, np.float64).ravel()
                                                  for b in params["conv_b"]]))
    C = int(np.asarray(params["conv_w"][0]).shape[0])
    Wt = np.ascontiguousarray(backflow.build_wtilde(params["W"], params["theta"], Lx, Ly,
                                                    np.float64))
    maps = lattice.symmetry_mode_maps(Lx, Ly) if symm else np.arange(M)[None]
    maps = np.ascontiguousarray(maps, dtype=np.int64)
    n = int((s[0] > 0).sum()) if B else 2
    sign = np.empty(B)
    logabs = np.empty(B)
    rc = fn(s.ctypes.data, B, Lx, Ly, C, len(params["conv_w"]),
                            conv_w.ctypes.data, conv_b.ctypes.data, Wt.ctypes.data, n,
                            maps.ctypes.data, maps.shape[0], sign.ctypes.data,
                            logabs.ctypes.data, int(threads))
    if rc:
        raise RuntimeError(f"nhp_amplitudes failed ({rc})")
    return sign, logabs
