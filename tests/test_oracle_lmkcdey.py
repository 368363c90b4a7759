"""CPU checks of the LMKCDEY blind rotation (the reference's method = LMKCDEY,
bitwise/src/cirbts/cirbts-lmkcdey.cu; keys cirbts-init.cu:630-726) in the oracle: the keys
are what they claim (eval-key rows decrypt to g_j X^{s_i}, automorphism-key rows to
-g_j psi_k(s)), the automorphism maps are permutations that act as X -> X^k, and the LMKCDEY
accumulator decrypts to the same phase as the one-bit GINX accumulator on the same inputs,
within the key noise, when the switched masks are odd (LMKCDEY rounds every mask to odd) and
the test vector has one slot (num_lut = 1: the rotation is not quantized to multiples of
2^bitwidth, which odd masks could not respect)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_encrypt_bits, oracle_lmkcdey_keys

NUM_AUTO = 4


@pytest.fixture(scope="module")
def small(pkg, oracle):
    p = pkg.preset_params("2x18")
    p.N, p.n, p.num_lut = 1024, 13, 1
    q = np.zeros(1, np.uint64)
    oracle.orc_get_primes(1024, 54, 1, q)
    p.Q = int(q[0])
    keys = pkg.key_buffers(p)
    pkg.call("cbs_generate_keys_host", ctypes.byref(p), 41, *(keys[k].ctypes.data for k in pkg.KEY_FIELDS))
    oc = OracleCbs(oracle, p, keys)
    return p, keys, oc, oracle_lmkcdey_keys(oracle, p, keys, NUM_AUTO, 41)


def _poly_mul_monomial(e: int, N: int) -> list:
    """coefficients of X^e (e mod 2N) as signed ints"""
    v = [0] * N
    e %= 2 * N
    v[e % N] = 1 if e < N else -1
    return v


def test_auto_maps_are_the_automorphisms(pkg, oracle, small):
    p, keys, oc, lmk = small
    N, Q = p.N, p.Q
    pows = [2 * N - 5] + [pow(5, i, 2 * N) for i in range(1, NUM_AUTO + 1)]
    rng = np.random.default_rng(3)
    poly = rng.integers(0, Q, N, dtype=np.uint64)
    spec = poly.copy()
    oracle.orc_ntt_forward(spec, 1, N, Q, oc.rp)
    for k, pw in enumerate(pows):
        m = lmk["maps"][k]
        assert sorted(m.tolist()) == list(range(N))
        got = spec[m].copy()
        oracle.orc_ntt_inverse(got, 1, N, Q, oc.irp, int(oc.ninv[0]))
        want = [0] * N
        for i, c in enumerate(poly.tolist()):
            e = (i * pw) % (2 * N)
            if e < N:
                want[e] = (want[e] + c) % Q
            else:
                want[e - N] = (want[e - N] - c) % Q
        assert got.tolist() == want, pw


def test_keys_encrypt_their_messages(small):
    p, keys, oc, lmk = small
    N, Q, g = p.N, p.Q, p.base_g.bit_length() - 1
    s = keys["s_lwe"]
    for i in (0, p.n - 1):
        for j in range(p.digits_g):
            ph = oc.phase_coef(lmk["eval"][i, 2 * j + 1])
            want = [(1 << (g * (j + 1))) % Q * x for x in _poly_mul_monomial(int(s[i]), N)]
            err = [((int(a) - int(b) + Q // 2) % Q) - Q // 2 for a, b in zip(ph, want)]
            assert max(abs(x) for x in err) < 2 ** 20
    pows = [2 * N - 5] + [pow(5, i, 2 * N) for i in range(1, NUM_AUTO + 1)]
    sr = [int(x) for x in keys["s_rlwe"]]
    for k in (0, NUM_AUTO):
        ps = [0] * N
        for i, c in enumerate(sr):
            e = (i * pows[k]) % (2 * N)
            if e < N:
                ps[e] += c
            else:
                ps[e - N] -= c
        for j in range(p.digits_g):
            ph = oc.phase_coef(lmk["auto"][k, j])
            gj = 1 << (g * (j + 1))
            err = [((int(a) + gj * b + Q // 2) % Q) - Q // 2 for a, b in zip(ph, ps)]
            assert max(abs(x) for x in err) < 2 ** 20


@pytest.mark.parametrize("window", [0, 8])
def test_lmkcdey_rotation_matches_one_bit_phase(pkg, oracle, small, window):
    p, keys, oc, lmk = small
    if window:
        lmk = oracle_lmkcdey_keys(oracle, p, keys, NUM_AUTO, 41, window)
    N, Q = p.N, p.Q
    oracle.orc_special_ms.restype = ctypes.c_uint32
    bw = max(0, (p.num_lut - 1).bit_length())
    rng = np.random.default_rng(17)
    bits = [0, 1, 1, 0]
    a, b = lwe_encrypt_bits(rng, keys["s_lwe"], bits, p.q_lwe)
    # masks that switch exactly to odd values, where both rotations rotate by the same amount
    step = p.q_lwe // (2 * N)
    a = (2 * rng.integers(0, N, size=a.shape) + 1).astype(np.uint64) * np.uint64(step)
    dot = (a.astype(object) * keys["s_lwe"].astype(object)).sum(axis=1)
    b = np.array([(int(d) + m * (p.q_lwe // 2)) % p.q_lwe for d, m in zip(dot, bits)], dtype=np.uint64)
    assert all(oracle.orc_special_ms(int(x), 2 * N, p.q_lwe, bw) % 2 == 1 for x in a.reshape(-1)[:50])
    one = oc.br_acc(a, b)
    lk = oc.br_acc_lmkcdey(a, b, lmk)
    worst = 0
    for i in range(len(bits)):
        d = oc.phase_coef(lk[i]) - oc.phase_coef(one[i])
        e = [((int(x) * N + Q // 2) % Q) - Q // 2 for x in d]  # undo the N^-1 finalize scaling
        worst = max(worst, max(abs(x) for x in e))
    print(f"LMKCDEY vs one-bit GINX: max |phase difference| = 2^{np.log2(worst + 1):.1f}")
    assert worst < 2 ** 32


@pytest.mark.parametrize("preset,num_auto,window", [("2x18", 10, 0), ("2x18", 1, 0), ("2x18", 10, 32)])
def test_oracle_lmkcdey_keygen_matches_host(pkg, oracle, preset, num_auto, window):
    """The product's seeded host generation of the LMKCDEY keys and maps against the oracle's,
    word for word (the oracle's keys are the ones the GPU parity tests compare against); the
    windowed set (window 32 at N = 2048) holds 2N - 5, 5^1 .. 5^32 and 5^64 .. 5^992."""
    p = pkg.preset_params(preset)
    p.num_lut = 1
    keys = pkg.generate_keys_host(p, 7)
    want = oracle_lmkcdey_keys(oracle, p, keys, num_auto, 7, window)
    ev, au = pkg.generate_lmkcdey_keys_host(p, 7, num_auto, window)
    assert np.array_equal(ev, want["eval"])
    assert np.array_equal(au, want["auto"])
    assert np.array_equal(pkg.lmkcdey_auto_maps_host(p.N, num_auto, window), want["maps"])
    if window:
        assert au.shape[0] == 1 + window + (p.N // 2 - 1) // window - 1
