"""ctypes binding of libmtp_b200.so (the C ABI declared in include/mtp_b200.h).

The shared library is built in-tree (``make -C jax-mtp_b200/csrc``).  There is
no fallback: importing a compute entry point without the library raises.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmtp_b200.so")

MTP_OK = 0
STATUS = {0: "MTP_OK", 1: "MTP_E_INVALID", 2: "MTP_E_FORMAT", 3: "MTP_E_CAPACITY", 4: "MTP_E_SPECIES",
          5: "MTP_E_NONFINITE", 6: "MTP_E_CUDA", 7: "MTP_E_NODEVICE", 8: "MTP_E_OOM"}
PRECISION_FP64 = 0
PRECISION_MIXED = 1
EFLAG, VFLAG, EATOM, VATOM, REUSE_NEIGHBORS = 1, 2, 4, 8, 16
NOALLOC_MAX_ATOMS, NOALLOC_MAX_SLOTS = 16384, 262144

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "mtp_abi_version": (_I, []),
    "mtp_create": (_I, [ctypes.c_char_p, _I, _I, _D, _I, _I, ctypes.POINTER(_P)]),
    "mtp_destroy": (None, [_P]),
    "mtp_last_error": (ctypes.c_char_p, [_P]),
    "mtp_set_stream": (_I, [_P, _P]),
    "mtp_use_own_stream": (_I, [_P]),
    "mtp_get_info": (_I, [_P, _P]),
    "mtp_get_stats": (_I, [_P, _P]),
    "mtp_set_coeffs": (_I, [_P, _P, _P, _P]),
    "mtp_execute_potential": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _D, _P, _P, _P]),
    "mtp_compute": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P]),
    "mtp_compute_device": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P]),
    "mtp_compute_positions": (_I, [_P, _I, _I, _P, _P, _P, _I, _P, _P, _I, _P, _P, _P, _P, _P]),
    "mtp_compute_positions_device": (_I, [_P, _I, _I, _P, _P, _P, _I, _P, _P, _I, _P, _P, _P, _P, _P]),
    "mtp_sync_status": (_I, [_P]),
    "mtp_compute_batch_device": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "mtp_adjoint_batch_device": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "mtp_set_launch": (_I, [_P, _I, _I, _I]),
    "mtp_get_launch": (_I, [_P, _P]),
    "mtp_parse_info": (_I, [ctypes.c_char_p, _P, ctypes.c_char_p, _I]),
    "mtp_schedule_emulate": (_I, [ctypes.c_char_p, _I, _I, _P, _P, _P, _P]),
    "mtp_measure_fma_peak": (_I, [ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "mtp_neighbors_device": (_I, [_P, _I, _P, _P, _P, _D, _I, _P, _P, _P, _P]),
    "mtp_pack_rij_device": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _P]),
    "mtp_verlet_device": (_I, [_P, _I, _P, _P, _P, _P, _P, _I, _D, _I]),
    "mtp_profile": (_I, [_P, _I]),
    "mtp_profile_read": (_I, [_P, ctypes.POINTER(_D), ctypes.POINTER(_I)]),
    "mtp_compute_device_noalloc": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "mtp_host_alloc": (_I, [ctypes.c_size_t, ctypes.POINTER(_P)]),
    "mtp_host_free": (_I, [_P]),
}

_lib = None


class MTPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C jax-mtp_b200/csrc` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int, handle=None) -> None:
    if code != MTP_OK:
        msg = lib().mtp_last_error(handle)
        raise MTPError(code, msg.decode() if msg else "")
