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
CFLAGS = ["-O3", "-fopenmp", "-fPIC", "-shared"]

_lib = None


def build(force: bool = False) -> None:
    """Compile the C restatement with gcc into ``oracle/libnh_port*.so``."""
    for march, lib in LIBS.items():
        if force or not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(SRC):
            subprocess.check_call(["gcc", *CFLAGS, f"-march={march}", SRC, "-o", lib, "-lm"])


def _host_has_avx2_fma() -> bool:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return all(f" {f}" in flags for f in ("avx2", "fma", "bmi2", "movbe"))


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIBS["x86-64-v3" if _host_has_avx2_fma() else "x86-64-v2"])
        p = ctypes.c_void_p
        lib.nhp_amplitudes.restype = ctypes.c_int
        lib.nhp_amplitudes.argtypes = [p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, p, p, p, ctypes.c_int, p, ctypes.c_int, p, p,
                                       ctypes.c_int]
        _lib = lib
    return _lib


def projected_amplitude(s: np.ndarray, params: dict, symm: bool = True, threads: int = 0):
    """(sign, logabs) of psi_P(s) (or psi(s) when ``symm`` is False) for s (B, 2N), FP64; the
    same ``params`` dict as the numpy oracle (conv_w, conv_b lists, W, theta, Lx, Ly)."""
    lib = load()
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
    rc = lib.nhp_amplitudes(s.ctypes.data, B, Lx, Ly, C, len(params["conv_w"]),
                            conv_w.ctypes.data, conv_b.ctypes.data, Wt.ctypes.data, n,
                            maps.ctypes.data, maps.shape[0], sign.ctypes.data,
                            logabs.ctypes.data, int(threads))
    if rc:
        raise RuntimeError(f"nhp_amplitudes failed ({rc})")
    return sign, logabs
