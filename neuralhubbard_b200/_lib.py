"""ctypes binding of libnh_b200.so (the C ABI declared in include/nh_b200.h).

The library is loaded from this package directory.  There is no fallback: if the shared
object is missing or fails to load, every operation raises ``NativeLibraryError``.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnh_b200.so")

NH_OK = 0
NET_CNN, NET_RESCONV = 0, 1
ANSATZ_PFAFFIAN, ANSATZ_BCS = 0, 1
OBS_TRANSVERSE_SPIN, OBS_PAIR, OBS_HOP = 0, 1, 2
FLAG_ZERO_PIVOT, FLAG_NONFINITE, FLAG_GROWTH, FLAG_REFINED, FLAG_CANCEL = 1, 2, 4, 8, 16
FLAG_TIMEOUT = 32
ABI_VERSION = 10

c_void_p, c_int, c_int64, c_uint64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64
c_float, c_double, c_size_t = ctypes.c_float, ctypes.c_double, ctypes.c_size_t


class NativeLibraryError(RuntimeError):
    """The CUDA library is missing, failed to load, or an entry point returned an error."""


class BackflowParams(ctypes.Structure):
    _fields_ = [
        ("conv_w", c_void_p),
        ("conv_b", c_void_p),
        ("conv_w_packed", c_void_p),
        ("conv_w_tc", c_void_p),
        ("Wt", c_void_p),
        ("Wt64", c_void_p),
        ("Lx", ctypes.c_int32),
        ("Ly", ctypes.c_int32),
        ("n_up", ctypes.c_int32),
        ("n_dn", ctypes.c_int32),
        ("channels", ctypes.c_int32),
        ("layers", ctypes.c_int32),
        ("cnn_mode", ctypes.c_int32),
        ("pf_mode", ctypes.c_int32),
        ("net", ctypes.c_int32),
        ("ansatz", ctypes.c_int32),
        ("cond_tau", c_double),
        ("cancel_tau", c_double),
        ("refine_tau", c_double),
        ("delta_d", c_double),
    ]


class HubbardParams(ctypes.Structure):
    _fields_ = [("t", c_double), ("tp", c_double), ("U", c_double), ("n_dirs", ctypes.c_int32)]


class ProposalParams(ctypes.Structure):
    _fields_ = [("weights", c_void_p), ("Lx", ctypes.c_int32), ("Ly", ctypes.c_int32),
                ("n_dirs", ctypes.c_int32), ("reserved", ctypes.c_int32)]


P_BF = ctypes.POINTER(BackflowParams)
P_H = ctypes.POINTER(HubbardParams)
P_Q = ctypes.POINTER(ProposalParams)
PROPOSAL_PARAMS = 4944

# name -> (restype, argtypes); every symbol declared in include/nh_b200.h.
SIGNATURES = {
    "nh_abi_version": (c_int, []),
    "nh_last_error": (ctypes.c_char_p, []),
    "nh_profile_enable": (c_int, [c_int]),
    "nh_profile_read": (c_int, [c_void_p, c_void_p, c_int]),
    "nh_build_wtilde": (c_int, [c_void_p, c_float, c_int, c_int, c_int, c_void_p, c_void_p,
                                c_void_p]),
    "nh_pack_cnn_weights": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "nh_pack_resconv_weights_floats": (c_size_t, [c_int, c_int]),
    "nh_pack_resconv_weights": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "nh_pack_resconv_weights_tc_bytes": (c_size_t, [c_int]),
    "nh_pack_resconv_weights_tc": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "nh_pack_cnn_weights_tc_bytes": (c_size_t, []),
    "nh_pack_cnn_weights_tc": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "nh_cnn_forward": (c_int, [c_void_p, c_int, P_BF, c_void_p, c_void_p]),
    "nh_pairing_occ": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int,
                               c_void_p, c_void_p]),
    "nh_slogpf_workspace_bytes": (c_size_t, [c_int, c_int]),
    "nh_slogpf": (c_int, [c_void_p, c_int, c_int, c_double, c_void_p, c_void_p, c_void_p,
                          c_void_p, c_size_t, c_void_p]),
    "nh_slogpf_noalloc": (c_int, [c_void_p, c_int, c_int, c_double, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
    "nh_amplitude_workspace_bytes": (c_size_t, [c_int, c_int, P_BF]),
    "nh_amplitude": (c_int, [c_void_p, c_int, c_int, P_BF, c_void_p, c_void_p, c_void_p,
                             c_void_p, c_size_t, c_void_p]),
    "nh_local_energy_workspace_bytes": (c_size_t, [c_int, c_int, c_int, P_BF]),
    "nh_local_energy": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, P_BF, P_H, c_int,
                                c_void_p, ctypes.POINTER(c_int64), c_void_p, c_size_t, c_void_p]),
    "nh_hop_list": (c_int, [c_void_p, c_int, c_int, c_int, P_H, c_void_p, c_void_p, c_void_p,
                            c_void_p, c_void_p]),
    "nh_metropolis_workspace_bytes": (c_size_t, [c_int, c_int, P_BF]),
    "nh_metropolis_steps": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, P_BF, c_int,
                                    c_uint64, c_int64, c_int, c_void_p, c_void_p, c_size_t,
                                    c_void_p]),
    "nh_metropolis_steps_mixed": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, P_BF,
                                          c_int, c_int, c_uint64, c_int64, c_int, c_void_p,
                                          c_void_p, c_size_t, c_void_p]),
    "nh_proposal_pack": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "nh_proposal_forward": (c_int, [c_void_p, c_int, P_Q, c_void_p, c_void_p]),
    "nh_proposal_sample": (c_int, [c_void_p, c_int, P_Q, c_uint64, c_int64, c_void_p, c_void_p,
                                   c_void_p, c_void_p, c_void_p]),
    "nh_proposal_backward_workspace_bytes": (c_size_t, [c_int, P_Q]),
    "nh_proposal_backward": (c_int, [c_void_p, c_void_p, c_void_p, c_int, P_Q, c_void_p,
                                     c_void_p, c_void_p, c_size_t, c_void_p]),
    "nh_proposal_adam_step": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int64,
                                      c_float, c_float, c_float, c_float, c_void_p, c_void_p]),
    "nh_pfaffian_adjoint": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "nh_pairing_occ_vjp": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                   c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "nh_param_count": (c_int64, [P_BF]),
    "nh_log_jacobian_workspace_bytes": (c_size_t, [c_int, c_int, P_BF]),
    "nh_log_jacobian": (c_int, [c_void_p, c_int, c_int, P_BF, c_void_p, c_float, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "nh_observable_workspace_bytes": (c_size_t, [c_int, c_int, c_int, P_BF]),
    "nh_observable": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, P_BF, c_int, c_int,
                              c_int, c_void_p, c_void_p, c_size_t, c_void_p]),
    "nh_metropolis_learned_workspace_bytes": (c_size_t, [c_int, c_int, P_BF]),
    "nh_metropolis_steps_learned": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, P_BF,
                                            P_Q, c_uint64, c_int64, c_int, c_void_p, c_void_p,
                                            c_size_t, c_void_p]),
}

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """Load (once) and return the library with its argument types set."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryError(
                f"{LIB_PATH} is missing; build it with `python -m neuralhubbard_b200.build`")
        try:
            lib = ctypes.CDLL(LIB_PATH)
        except OSError as e:
            raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.nh_abi_version() != ABI_VERSION:
            raise NativeLibraryError(f"{LIB_PATH} has ABI {lib.nh_abi_version()}, this package "
                                     f"expects {ABI_VERSION}; rebuild it")
        _lib = lib
        return lib


class DeviceTimeoutError(NativeLibraryError):
    """A bounded wait of a tensor-core kernel expired: the call's results are not valid."""


def timeout_flagged(flags) -> bool:
    """Whether any of the output flags (numpy array or torch tensor) carries FLAG_TIMEOUT."""
    if hasattr(flags, "cpu"):
        flags = flags.cpu().numpy()
    import numpy as np

    return bool((np.asarray(flags) & FLAG_TIMEOUT).any())


def check_flags(flags, what: str) -> None:
    """Raise DeviceTimeoutError when an output flag carries FLAG_TIMEOUT (the tensor-core
    kernels' device error word, folded into the flags by the image combination)."""
    if flags is not None and timeout_flagged(flags):
        raise DeviceTimeoutError(f"{what}: a tensor-core kernel's bounded wait expired "
                                 "(NH_FLAG_TIMEOUT); its amplitudes are NaN")


def check(rc: int, what: str) -> None:
    if rc != NH_OK:
        msg = load().nh_last_error()
        raise NativeLibraryError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


KERNEL_IDS = {
    "cnn": 0, "pfaffian": 1, "pairing": 2, "combine": 3, "hop_count": 4, "scan": 5,
    "hop_emit": 6, "eloc_reduce": 7, "mh_propose": 8, "compact": 9, "mh_accept": 10,
    "wtilde": 11, "pfaffian64": 12, "cnn64": 13, "flagged": 14, "pack": 15, "cnn_tc": 16,
    "pfaffian_tc": 17, "prop_sample": 18, "prop_forward": 19, "prop_backward": 20,
    "prop_adam": 21, "resconv": 22, "resconv64": 23, "resconv_tc": 24, "refine": 25,
    "fused": 26, "pf_adjoint": 27, "pairing_vjp": 28, "cnn_vjp": 29, "det": 30, "det64": 31,
    "observable": 32,
}
K_COUNT = 40


def profile_enable(on: bool) -> None:
    check(load().nh_profile_enable(1 if on else 0), "nh_profile_enable")


def profile_read() -> dict:
    """{kernel name: (milliseconds, launches)} accumulated since the last read."""
    ms = (ctypes.c_double * K_COUNT)()
    n = (ctypes.c_int64 * K_COUNT)()
    check(load().nh_profile_read(ctypes.addressof(ms), ctypes.addressof(n), K_COUNT),
          "nh_profile_read")
    return {k: (float(ms[i]), int(n[i])) for k, i in KERNEL_IDS.items() if n[i]}


def call(name: str, *args):
    """Call an int-returning entry point and raise on a non-zero status."""
    rc = getattr(load(), name)(*args)
    check(rc, name)
    return rc
