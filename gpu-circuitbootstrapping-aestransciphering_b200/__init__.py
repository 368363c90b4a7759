"""B200-native bootstrapping / AES-128 transciphering hot path: Python host glue.

The compute lives in ``libcbs_b200.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/cbs_b200.h``).  This module only locates and loads that library with ctypes
and declares argument types; there is no CPU fallback.  If the library is missing the
loader raises, so a missing build can never silently degrade to another path.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT_DIR = PKG_DIR.parent
LIB_PATH = PKG_DIR / "libcbs_b200.so"
HEADER_PATH = ROOT_DIR / "include" / "cbs_b200.h"

_lib: ctypes.CDLL | None = None

c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_vp = ctypes.c_void_p

CBS_STATUS = {
    0: "CBS_OK", 1: "CBS_ERR_INVALID_ARG", 2: "CBS_ERR_SHAPE_MISMATCH", 3: "CBS_ERR_OOM",
    4: "CBS_ERR_CUDA", 5: "CBS_ERR_DEVICE_TIMEOUT", 6: "CBS_ERR_UNSUPPORTED", 7: "CBS_ERR_NOT_READY",
}


class CbsError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {CBS_STATUS.get(status, status)}: {msg}")
        self.status = status


class DModulus(ctypes.Structure):
    _fields_ = [("value", ctypes.c_uint64), ("const_ratio", ctypes.c_uint64 * 2)]


def declared_symbols() -> list[str]:
    """Function names declared in include/cbs_b200.h (the C ABI)."""
    text = HEADER_PATH.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cbs_[a-z0-9_]+)\s*\(", text)))


def _declare(lib: ctypes.CDLL) -> None:
    st = ctypes.c_int
    sz = ctypes.c_size_t
    u32 = ctypes.c_uint32
    u64 = ctypes.c_uint64
    sigs = {
        "cbs_last_error": (ctypes.c_char_p, []),
        "cbs_abi_version": (ctypes.c_int, []),
        "cbs_fnwt_1d_opt_batched": (st, [c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_fnwt_1d_opt_outofplace_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_inwt_1d_opt_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_inwt_1d_opt_outofplace_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_inwt_1d_opt_permute_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_ntt_tables_host": (st, [u32, u64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_get_primes": (st, [u32, ctypes.c_int, u32, c_vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args


def load() -> ctypes.CDLL:
    """Load libcbs_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with build_lib.py (no CPU fallback exists)")
        _lib = ctypes.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def check(status: int, where: str) -> None:
    """Raise CbsError for a non-zero cbs_status."""
    if status != 0:
        lib = load()
        raise CbsError(status, where, lib.cbs_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    """Call a C-ABI entry point and raise on a non-OK status."""
    check(getattr(load(), name)(*args), name)
