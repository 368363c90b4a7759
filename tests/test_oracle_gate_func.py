"""CPU checks of the functional-bootstrapping restatement (the reference's BatchGPUEvalFunc /
Floor / Sign / Decomp, bitwise/src/binfhe-base-scheme-batch.cu:215-712, from
https://eprint.iacr.org/2021/1337) over the oracle's programmable bootstrap, with host-generated
gate keys at a short LWE dimension (exact integer products, seconds per bootstrap): every
evaluator decrypts to what it computes in the clear."""
from __future__ import annotations

import numpy as np
import pytest

from gate_harness import OracleGateFunc, declare_gate, lut_via_function, lwe_encrypt_mod, phase_mod

BETA = 128


@pytest.fixture(scope="module")
def fsetup(pkg, oracle):
    p = pkg.gate_default_params()
    p.n = 24
    keys = pkg.gate_generate_keys_host(p, 17)
    return p, keys, OracleGateFunc(declare_gate(oracle), p, keys)


def _centred(x, bits):
    x = np.asarray(x, np.int64) % (1 << bits)
    return np.where(x >= 1 << (bits - 1), x - (1 << bits), x)


def test_programmable_bootstrap_evaluates_the_table(fsetup):
    p, keys, fo = fsetup
    s = keys["s_lwe"]
    in_bits, f_bits = 10, 12  # q_in = 1024 (divides 2N = 2048), output mod 4096
    rng = np.random.default_rng(1)
    lut = rng.integers(0, 1 << f_bits, 512, dtype=np.uint64)
    ph = np.array([5, 200, 511, 600, 1000, 0], np.int64)
    a, b = lwe_encrypt_mod(rng, s, ph, in_bits, sigma_units=0)
    oa, ob = fo.bootstrap(a, b, in_bits, lut, f_bits)
    got = phase_mod(s, oa, ob, f_bits)
    want = [int(lut[x]) if x < 512 else (-int(lut[x - 512])) % (1 << f_bits) for x in ph]
    err = _centred(got - np.array(want, np.int64), f_bits)
    assert np.abs(err).max() < 64, err  # bootstrap + key-switch noise, about 2^-9 of the torus


@pytest.mark.parametrize("kind", ["negacyclic", "periodic", "arbitrary"])
def test_eval_func(fsetup, kind):
    p, keys, fo = fsetup
    s = keys["s_lwe"]
    P, q = 4, 1024  # plaintext modulus 4 on q = N (an arbitrary table needs q <= N)
    f = {"negacyclic": lambda m, p_: [1, 2, 3, 2][m], "periodic": lambda m, p_: m % 2,
         "arbitrary": lambda m, p_: (3 * m) % 4}[kind]
    lut = lut_via_function(f, P, q)
    ms = np.array([0, 1, 2, 3, 2, 1], np.int64)
    rng = np.random.default_rng(2)
    a, b = lwe_encrypt_mod(rng, s, ms * (q // P), 10, sigma_units=3)
    oa, ob = fo.eval_func(a, b, q, lut, BETA)
    got = phase_mod(s, oa, ob, 10)
    dec = ((got + q // (2 * P)) // (q // P)) % P
    assert list(dec) == [f(int(m), P) for m in ms], (kind, got)


def test_eval_floor(fsetup):
    p, keys, fo = fsetup
    s = keys["s_lwe"]
    mod_bits, q_bits = 13, 10
    rng = np.random.default_rng(3)
    x = np.array([100, 1500, 3000, 5000, 7000, 8000], np.int64)
    a, b = lwe_encrypt_mod(rng, s, x, mod_bits, sigma_units=2)
    oa, ob = fo.eval_floor(a, b, mod_bits, q_bits, BETA)
    got = phase_mod(s, oa, ob, mod_bits)
    q = 1 << q_bits
    want = (((x + BETA) // q) * q) % (1 << mod_bits)
    assert np.abs(_centred(got - want, mod_bits)).max() < BETA // 2, (got, want)


@pytest.mark.parametrize("scheme_switch", [False, True])
def test_eval_sign(fsetup, scheme_switch):
    p, keys, fo = fsetup
    s = keys["s_lwe"]
    mod_bits, q_bits = 14, 10
    rng = np.random.default_rng(4)
    x = np.array([300, 4000, 8000, 8500, 12000, 16000], np.int64)
    a, b = lwe_encrypt_mod(rng, s, x, mod_bits, sigma_units=2)
    oa, ob = fo.eval_sign(a, b, mod_bits, q_bits, BETA, scheme_switch)
    got = phase_mod(s, oa, ob, q_bits)
    q = 1 << q_bits
    msb = (x >= (1 << (mod_bits - 1))).astype(np.int64)
    want = np.where(msb == 1, q // 4, -q // 4) % q if scheme_switch else (msb * (q // 2)) % q
    assert np.abs(_centred(got - want, q_bits)).max() < q // 8, (got, want)


def test_eval_decomp(fsetup):
    p, keys, fo = fsetup
    s = keys["s_lwe"]
    mod_bits, q_bits = 14, 10
    rng = np.random.default_rng(5)
    x = np.array([300, 4000, 9000, 16000], np.int64)
    a, b = lwe_encrypt_mod(rng, s, x, mod_bits, sigma_units=2)
    digits = fo.eval_decomp(a, b, mod_bits, q_bits, BETA)
    # each floor removes log2(q / 2 beta) = 2 bits: 2^14 -> 2^12 -> 2^10, three digits mod 2^10
    assert [bits for _, bits in digits] == [10, 10, 10]
    # the same steps in the clear: digit = value mod q, value <- q floor((value + beta) / q) switched
    # down by 4
    q, val, mb = 1 << q_bits, x.copy(), mod_bits
    want = []
    while mb > q_bits:
        want.append(val % q)
        val = (((val + BETA) // q) * q) % (1 << mb)
        val = (val + 2) // 4 % (1 << (mb - 2))
        mb -= 2
    want.append(val % (1 << mb))
    for ((da, db), bits), w in zip(digits, want):
        got = phase_mod(s, da, db, bits)
        assert np.abs(_centred(got - w, bits)).max() < 32, (got, w)
