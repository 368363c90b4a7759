"""Shared fixtures: the product library (C ABI), the CPU oracle and the reference pin."""
from __future__ import annotations

import ctypes
import importlib.util
import os
import tempfile
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

# the tests never read a tuning cache of the machine (a cached blind-rotation grouping would
# change what selecting the FFT64 backend does): every session gets an empty one of its own
os.environ["CBS_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="cbs_tune_"), "tune.json")
PKG_DIR = ROOT / "gpu-circuitbootstrapping-aestransciphering_b200"
ORACLE_DIR = ROOT / "oracle"
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_pkg():
    name = "cbs_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG_DIR / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _ensure_oracle() -> Path:
    so = ORACLE_DIR / "liboracle.so"
    src = ORACLE_DIR / "oracle.c"
    if not so.exists() or so.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(ORACLE_DIR), "liboracle.so"], check=True, capture_output=True)
    return so


_U64P = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_U32P = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_U16P = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")


def load_oracle() -> ctypes.CDLL:
    lib = ctypes.CDLL(str(_ensure_oracle()))
    u32, u64 = ctypes.c_uint32, ctypes.c_uint64
    lib.orc_get_primes.argtypes = [u32, ctypes.c_int, u32, _U64P]
    lib.orc_ntt_tables.argtypes = [u32, u64, _U64P, _U64P, _U64P, _U64P, _U64P]
    lib.orc_ntt_forward.argtypes = [_U64P, ctypes.c_size_t, u32, u64, _U64P]
    lib.orc_ntt_inverse.argtypes = [_U64P, ctypes.c_size_t, u32, u64, _U64P, u64]
    lib.orc_ntt_inverse_permute.argtypes = [_U64P, _U64P, _U32P, ctypes.c_size_t, u32, u64, _U64P, u64]
    lib.orc_negacyclic_mul.argtypes = [_U64P, _U64P, _U64P, u32, u64]
    lib.orc_auto_maps.argtypes = [_U32P, u32, u32]
    lib.orc_signed_decompose.argtypes = [u64, u64, u32, u32, _U64P]
    lib.orc_special_ms.argtypes = [u64, u32, u64, u32]
    lib.orc_special_ms.restype = u32
    lib.orc_mulmod.argtypes = [u64, u64, u64]
    lib.orc_mulmod.restype = u64
    lib.orc_aes128_encrypt.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]
    lib.orc_aes128_key_expand.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    lib.orc_aes_enc_tables.argtypes = [_U32P]
    lib.orc_extract_keyswitch.argtypes = [_U64P, _U32P, u32, u32, u64, _U16P, u32, u32, u32, u64, _U64P, _U64P, u32]
    lib.orc_num_threads.restype = ctypes.c_int
    return lib


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()


@pytest.fixture(scope="session")
def ref_host():
    so = ORACLE_DIR / "_ref" / "libref_host.so"
    if not so.exists():
        pytest.skip("reference host library (oracle/_ref) not built here")
    lib = ctypes.CDLL(str(so))
    u32, u64 = ctypes.c_uint32, ctypes.c_uint64
    lib.ref_get_primes.argtypes = [u32, ctypes.c_int, u32, _U64P]
    lib.ref_ntt_tables.argtypes = [u32, u64, _U64P, _U64P, _U64P, _U64P, _U64P]
    lib.ref_aes_enc_tables.argtypes = [_U32P]
    return lib


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def lib(pkg):
    return pkg.load()


def oracle_tables(oracle, n: int, q: int):
    rp, rps, irp, irps = (np.zeros(n, np.uint64) for _ in range(4))
    ninv = np.zeros(2, np.uint64)
    assert oracle.orc_ntt_tables(n.bit_length() - 1, q, rp, rps, irp, irps, ninv) == 0
    return rp, rps, irp, irps, ninv


def oracle_primes(oracle, n: int, bits: int, count: int) -> list[int]:
    out = np.zeros(count, np.uint64)
    assert oracle.orc_get_primes(n, bits, count, out) == 0
    return [int(x) for x in out]


def rand_mod(rng: np.random.Generator, q: int, shape) -> np.ndarray:
    return rng.integers(0, q, size=shape, dtype=np.uint64)
