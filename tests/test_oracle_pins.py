"""Pin the CPU oracle: reference golden vectors, the FIPS-197 known answer, an
independent AES (OpenSSL via `cryptography`), and algebraic properties of the NTT."""
from __future__ import annotations

import ctypes
import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN, oracle_tables, rand_mod

REF = json.loads((GOLDEN / "reference_host.json").read_text())


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", REF["primes"], ids=lambda c: f"{c['ntt_size']}-{c['bits']}-{c['count']}")
def test_get_primes_matches_reference(oracle, case):
    out = np.zeros(case["count"], np.uint64)
    assert oracle.orc_get_primes(case["ntt_size"], case["bits"], case["count"], out) == 0
    assert [int(x) for x in out] == case["values"]


@pytest.mark.parametrize("case", REF["ntt_tables"], ids=lambda c: f"{c['n']}-{c['q']:x}")
def test_ntt_tables_match_reference(oracle, case):
    rp, rps, irp, irps, ninv = oracle_tables(oracle, case["n"], case["q"])
    for name, arr in zip(("rp", "rp_shoup", "irp", "irp_shoup"), (rp, rps, irp, irps)):
        assert [int(x) for x in arr[:8]] == case["head"][name]
        assert _sha(arr) == case["sha256"][name], name
    assert [int(ninv[0]), int(ninv[1])] == case["n_inv"]


def test_aes_fips197_known_answer(oracle):
    key = bytes(range(16))
    pt = bytes.fromhex("00112233445566778899aabbccddeeff")
    out = ctypes.create_string_buffer(16)
    oracle.orc_aes128_encrypt(key, pt, out)
    assert out.raw.hex() == "69c4e0d86a7b0430d8cdb78070b4c55a"


@pytest.mark.parametrize("i", range(len(REF["aes"]["cases"])))
def test_aes_matches_reference(oracle, i):
    c = REF["aes"]["cases"][i]
    key, pt = bytes.fromhex(c["key"]), bytes.fromhex(c["pt"])
    out = ctypes.create_string_buffer(16)
    oracle.orc_aes128_encrypt(key, pt, out)
    assert out.raw.hex() == c["ct"]
    rk = ctypes.create_string_buffer(176)
    oracle.orc_aes128_key_expand(key, rk)
    assert rk.raw.hex() == c["round_keys"]


def test_aes_matches_openssl(oracle):
    cryptography = pytest.importorskip("cryptography")
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    rng = np.random.default_rng(7)
    for _ in range(64):
        key, pt = rng.bytes(16), rng.bytes(16)
        enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
        want = enc.update(pt) + enc.finalize()
        out = ctypes.create_string_buffer(16)
        oracle.orc_aes128_encrypt(key, pt, out)
        assert out.raw == want


def test_aes_tables_match_reference(oracle):
    te = np.zeros(8 * 256, np.uint32)
    oracle.orc_aes_enc_tables(te)
    assert [int(x) for x in te] == REF["aes"]["enc_tables"]


def test_oracle_pins_agree_with_live_reference(oracle, ref_host):
    """When the reference's host code is built here, compare against it directly too."""
    rng = np.random.default_rng(3)
    for n, bits in [(2048, 54), (4096, 50), (8192, 60)]:
        a = np.zeros(2, np.uint64)
        b = np.zeros(2, np.uint64)
        assert oracle.orc_get_primes(n, bits, 2, a) == 0
        assert ref_host.ref_get_primes(n, bits, 2, b) == 0
        assert (a == b).all()
        mine = oracle_tables(oracle, n, int(a[1]))
        theirs = [np.zeros(n, np.uint64) for _ in range(4)] + [np.zeros(2, np.uint64)]
        assert ref_host.ref_ntt_tables(n.bit_length() - 1, int(a[1]), *theirs) == 0
        for x, y in zip(mine, theirs):
            assert (x == y).all()
    for _ in range(8):
        key, pt = rng.bytes(16), rng.bytes(16)
        o1, o2 = ctypes.create_string_buffer(16), ctypes.create_string_buffer(16)
        oracle.orc_aes128_encrypt(key, pt, o1)
        ref_host.ref_aes128_encrypt(key, pt, o2)
        assert o1.raw == o2.raw


@pytest.mark.parametrize("n", [16, 64, 256])
def test_ntt_convolution_theorem(oracle, n):
    """INTT(NTT(a) * NTT(b)) equals the schoolbook negacyclic product."""
    q = int(REF["primes"][1]["values"][0]) if n <= 1024 else None
    from conftest import oracle_primes
    q = oracle_primes(oracle, n, 54, 1)[0]
    rp, rps, irp, irps, ninv = oracle_tables(oracle, n, q)
    rng = np.random.default_rng(n)
    a, b = rand_mod(rng, q, n), rand_mod(rng, q, n)
    want = np.zeros(n, np.uint64)
    oracle.orc_negacyclic_mul(a, b, want, n, q)
    fa, fb = a.copy(), b.copy()
    oracle.orc_ntt_forward(fa, 1, n, q, rp)
    oracle.orc_ntt_forward(fb, 1, n, q, rp)
    prod = np.array([oracle.orc_mulmod(int(x), int(y), q) for x, y in zip(fa, fb)], np.uint64)
    oracle.orc_ntt_inverse(prod, 1, n, q, irp, int(ninv[0]))
    assert (prod == want).all()
    back = fa.copy()
    oracle.orc_ntt_inverse(back, 1, n, q, irp, int(ninv[0]))
    assert (back == a).all()


def test_ntt_evaluation_order(oracle):
    """Slot i of the forward NTT is the evaluation at psi^(2*bitrev(i)+1)."""
    from conftest import oracle_primes
    n = 32
    q = oracle_primes(oracle, n, 40, 1)[0]
    rp, *_ = oracle_tables(oracle, n, q)
    psi = int(rp[1 << 4 >> 4]) if False else None
    rng = np.random.default_rng(1)
    a = rand_mod(rng, q, n)
    f = a.copy()
    oracle.orc_ntt_forward(f, 1, n, q, rp)
    # psi = rp[bitrev(1)] = rp[n/2]
    psi = int(rp[n // 2])
    logn = n.bit_length() - 1
    for i in range(n):
        e = 2 * int(f"{i:0{logn}b}"[::-1], 2) + 1
        x = pow(psi, e, q)
        v = sum(int(c) * pow(x, j, q) for j, c in enumerate(a)) % q
        assert int(f[i]) == v


def test_decompose_reconstructs(oracle):
    """Signed digits recompose to the input up to the dropped low bits (plus a possible
    discarded top carry, which is a multiple of 2^logQ)."""
    from conftest import oracle_primes
    Q = oracle_primes(oracle, 2048, 54, 1)[0]
    rng = np.random.default_rng(11)
    for base, digits in [(1 << 12, 3), (1 << 6, 4), (1 << 9, 5), (1 << 7, 2)]:
        gb = base.bit_length() - 1
        ign = max(0, Q.bit_length() - digits * gb)
        out = np.zeros(digits, np.uint64)
        for x in list(rand_mod(rng, Q, 200)) + [0, 1, Q - 1, Q // 2, Q // 2 + 1]:
            oracle.orc_signed_decompose(int(x), Q, base, digits, out)
            ds = [int(d) - Q if int(d) > Q // 2 else int(d) for d in out]
            assert all(-base // 2 <= d < base // 2 + 1 for d in ds)
            rec = sum(d << (ign + gb * i) for i, d in enumerate(ds))
            xs = int(x) - Q if int(x) >= Q // 2 else int(x)
            err = (xs - rec) % (1 << Q.bit_length())
            err = min(err, (1 << Q.bit_length()) - err)
            assert err <= (1 << ign) // 2 + 1


def test_special_ms_rounding(oracle):
    """device_SpecialMS_IndexPos: round to a multiple of 2^bw in Z_2N (FP64 expression)."""
    two_n, q = 4096, 1 << 14
    for bw in (0, 1, 2):
        for v in range(0, q, 37):
            got = oracle.orc_special_ms(v, two_n, q, bw)
            want = (int(np.floor(v * (two_n / (q * (1 << bw))) + 0.5)) << bw) % two_n
            assert got == want
            assert got % (1 << bw) == 0
