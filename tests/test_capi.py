"""C-ABI checks that need no GPU: the library loads, exports every declared symbol,
validates arguments before touching the device, and its host helpers agree with the
pinned oracle."""
from __future__ import annotations

import ctypes
import json

import numpy as np
import pytest

from conftest import GOLDEN, oracle_primes, oracle_tables

REF = json.loads((GOLDEN / "reference_host.json").read_text())


def test_library_exports_every_declared_symbol(pkg, lib):
    names = pkg.declared_symbols()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(lib):
    assert lib.cbs_abi_version() >= 1


@pytest.mark.parametrize("case", REF["ntt_tables"], ids=lambda c: f"{c['n']}")
def test_host_tables_match_oracle(lib, oracle, case):
    n, q = case["n"], case["q"]
    mine = [np.zeros(n, np.uint64) for _ in range(4)]
    ninv = np.zeros(2, np.uint64)

    class DMod(ctypes.Structure):
        _fields_ = [("value", ctypes.c_uint64), ("const_ratio", ctypes.c_uint64 * 2)]

    dm = DMod()
    st = lib.cbs_ntt_tables_host(n, q, *(a.ctypes.data for a in mine), ninv.ctypes.data, ctypes.addressof(dm))
    assert st == 0
    want = oracle_tables(oracle, n, q)
    for a, b in zip(mine + [ninv], want):
        assert (a == b).all()
    assert dm.value == q
    assert [dm.const_ratio[0], dm.const_ratio[1]] == case["const_ratio"]


@pytest.mark.parametrize("case", REF["primes"], ids=lambda c: f"{c['ntt_size']}-{c['bits']}")
def test_host_primes_match_reference(lib, case):
    out = np.zeros(case["count"], np.uint64)
    assert lib.cbs_get_primes(case["ntt_size"], case["bits"], case["count"], out.ctypes.data) == 0
    assert [int(x) for x in out] == case["values"]


def test_argument_validation_without_device(lib):
    # invalid dim and null pointers are rejected before any CUDA call
    assert lib.cbs_fnwt_1d_opt_batched(None, None, None, None, 3000, 4, None) == 1
    assert b"dim" in lib.cbs_last_error()
    assert lib.cbs_fnwt_1d_opt_batched(None, None, None, None, 2048, 4, None) == 1
    assert b"null" in lib.cbs_last_error()
    assert lib.cbs_inwt_1d_opt_batched(None, None, None, None, None, None, 2048, 0, None) == 0  # empty batch
    buf = (ctypes.c_uint64 * 4)()
    p = ctypes.addressof(buf)
    assert lib.cbs_inwt_1d_opt_permute_batched(p, p, p, p, p, p, p, p, 2048, 1, None) == 1
    assert b"in-place" in lib.cbs_last_error()
    # AES ciphertext add: null context / pointers rejected, empty input accepted
    assert lib.cbs_aes128_ctr_add_ciphertext_device(None, p, 1, p, None) == 1
    assert lib.cbs_aes128_ctr_transcipher_ciphertext(None, p, p, 1, p, p) == 1
    # not enough NTT-friendly primes of 13 bits for N=2048
    assert lib.cbs_get_primes(2048, 13, 5, np.zeros(5, np.uint64).ctypes.data) == 1


def test_rns_context_validation_without_device(lib, oracle):
    """cbs_rns_context_create rejects bad chains before any device call."""
    n = 1 << 13
    good = np.array(oracle_primes(oracle, n, 50, 3), np.uint64)
    h = ctypes.c_void_p()

    def create(deg, q, p):
        q = np.ascontiguousarray(q, np.uint64)
        p = np.ascontiguousarray(p, np.uint64)
        return lib.cbs_rns_context_create(deg, q.ctypes.data, len(q), p.ctypes.data, len(p), ctypes.byref(h))

    assert create(n // 2 * 3, good[:2], good[2:]) == 1          # not a power of two
    assert create(1 << 9, good[:2], good[2:]) == 1              # below 2^10
    assert create(n, good[:2], np.array([], np.uint64)) == 1    # no special prime
    assert create(n, np.array([good[0], good[0]]), good[2:]) == 1  # duplicate
    assert create(n, np.array([good[0] + 2]), good[2:]) == 1   # not prime / not 1 mod 2N
    assert create(n, good[:1], np.array(oracle_primes(oracle, n, 50, 20)[3:20], np.uint64)) == 1  # alpha > 16
    assert h.value is None


def test_cpp_facade_compiles(tmp_path):
    """include/cbs_b200.hpp (the reference-shaped C++ surface) compiles against the C ABI."""
    import shutil
    import subprocess
    from conftest import ROOT
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "facade.cpp"
    src.write_text('#include "cbs_b200.hpp"\n'
                   'int main() {\n'
                   '  using namespace cbs_b200;\n'
                   '  void (*f)(uint64_t*, const uint64_t*, const uint64_t*, const cbs_dmodulus*, size_t, size_t,\n'
                   '            const cudaStream_t&) = fnwt_1d_opt_batched;\n'
                   '  (void)f;\n'
                   '  return sizeof(GPUCirBTSContext) > 0 && sizeof(RnsContext) > 0 ? 0 : 1;\n'
                   '}\n')
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-I", str(ROOT / "include"), "-I",
                        "/usr/local/cuda/include", str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("field,value", [("sigma_lwe", 1e3), ("sigma_rlwe", 5e4), ("sigma_lwe", -1.0),
                                         ("sigma_rlwe", float("nan"))])
def test_params_reject_sigma_out_of_range(pkg, lib, field, value):
    """The discrete-Gaussian samplers tabulate ~14 sigma entries: sigma is bounded to [0, 1000)
    by every parameter check (context creation and the host key generation alike)."""
    p = pkg.default_params()
    setattr(p, field, value)
    h = ctypes.c_void_p()
    assert lib.cbs_context_create(ctypes.byref(p), 8, ctypes.byref(h)) == 1
    assert b"sigma" in lib.cbs_last_error()
    assert h.value is None
    words = ctypes.c_size_t()
    assert lib.cbs_generate_mb_bsk_host(ctypes.byref(p), 1, 2, None, ctypes.byref(words)) == 1
    assert b"sigma" in lib.cbs_last_error()
