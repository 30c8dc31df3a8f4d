"""ctypes binding of the C ABI in include/accusim_b200.h (libaccusim_b200.so, built in-tree).

There is no fallback: if the library is missing or no CUDA device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libaccusim_b200.so")

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
DBL = C.c_double
SZ = C.c_size_t


class AcsGrid(C.Structure):
    _fields_ = [("lo", DBL * 3), ("span", DBL * 3), ("box", DBL * 3), ("ncell", I32 * 3), ("periodic", I32),
                ("rc", DBL), ("rc2", DBL)]


# device status block: flags, need_nbr, rebuilds, fail_step, steps_done, pad[3]
STATUS_WORDS = 8
FLAG_OVERFLOW, FLAG_NONFINITE, FLAG_TIMEOUT = 1, 2, 4

ACS_OK, ACS_ERR_ARG, ACS_ERR_WORKSPACE, ACS_ERR_CUDA, ACS_ERR_LIST_OVERFLOW = 0, 1, 2, 3, 4
ACS_ERR_NONFINITE, ACS_ERR_TIMEOUT, ACS_ERR_UNSUPPORTED, ACS_ERR_NO_DEVICE = 5, 6, 7, 8

# name -> (restype, argtypes); the order matches include/accusim_b200.h
SIGNATURES = {
    "acs_abi_version": (C.c_int, []),
    "acs_status_string": (C.c_char_p, [C.c_int]),
    "acs_device_info": (C.c_int, [C.POINTER(C.c_int)] * 3),
    "acs_grid_setup": (C.c_int, [C.POINTER(AcsGrid), P, C.c_int, P, P, DBL]),
    "acs_nlist_work_bytes": (SZ, [I64, C.POINTER(AcsGrid)]),
    "acs_nlist_build": (C.c_int, [P, I64, C.POINTER(AcsGrid), I32, P, P, P, SZ, P, P]),
    "acs_nlist_pairs": (C.c_int, [P, P, I64, I32, P, P, I64, P, P]),
    "acs_nlist_displacement": (C.c_int, [P, P, I64, P, C.c_int, DBL, P, P]),
    "acs_force_work_bytes": (SZ, [I64]),
    "acs_lj_fp64": (C.c_int, [P, P, I64, P, C.c_int, P, P, I32, I32, P, P, DBL, P, P, P, SZ, P]),
    "acs_lj_fp64_noalloc": (C.c_int, [P, P, I64, P, C.c_int, P, P, I32, I32, P, P, DBL, P, P, P]),
    "acs_dsf_fp64": (C.c_int, [P, P, I64, P, C.c_int, P, P, I32, P, P, DBL, DBL, DBL, P, P, P, SZ, P]),
    "acs_vv_kick": (C.c_int, [P, P, I64, DBL, P]),
    "acs_langevin_ou": (C.c_int, [P, P, P, I64, DBL, P]),
    "acs_rdf_work_bytes": (SZ, [I64, P]),
    "acs_rdf_hist": (C.c_int, [P, P, I64, P, I32, I32, DBL, P, P, SZ, P]),
    "acs_vv_drift_wrap": (C.c_int, [P, P, I64, DBL, P, C.c_int, P]),
    "acs_vv_accel": (C.c_int, [P, P, P, P, I32, I64, P]),
    "acs_reduce_work_bytes": (SZ, [I64]),
    "acs_reduce_conserved": (C.c_int, [P, P, P, P, I32, I64, P, P, SZ, P]),
}


class AcsError(RuntimeError):
    """A status code other than ACS_OK returned through the C ABI."""

    def __init__(self, code, where=""):
        self.code = code
        super().__init__(f"{where}: {status_string(code)} (status {code})" if where else status_string(code))


class ListOverflow(AcsError):
    pass


_lib = None


def lib():
    """The loaded library; raises if it has not been built (python -m devinproj_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m devinproj_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(code: int) -> str:
    return lib().acs_status_string(int(code)).decode()


def check(code: int, where: str = ""):
    if code != ACS_OK:
        if code == ACS_ERR_LIST_OVERFLOW:
            raise ListOverflow(code, where)
        raise AcsError(code, where)


def ptr(t) -> int | None:
    """Device (or host) address of a torch tensor / numpy array, None for None."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def dbl3(x):
    """Host pointer to 3 doubles (kept alive by the returned array)."""
    if x is None:
        return None, None
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(3))
    return a, a.ctypes.data
