"""CPU checks of the multi-bit blind rotation (the reference's CIRBTS_PBS_MULTIBIT = 2 / 3 / 4
grouping; 4 is the staged 3 + 1 grouping with 8 keys per group): the host-generated grouped keys are RGSW encryptions of the subset products of
the secret bits, and the oracle's exact grouped blind rotation decrypts to the same
accumulator as the one-bit blind rotation on the same inputs, within the key noise (tail
groups included: n = 13 leaves one coefficient in the last group)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_encrypt_bits

SUBSETS = {2: [0b01, 0b10, 0b11], 3: [0b001, 0b010, 0b100, 0b011, 0b101, 0b110, 0b111],
           4: [0b0001, 0b0010, 0b0100, 0b1000, 0b0011, 0b0101, 0b0110, 0b0111]}


@pytest.fixture(scope="module")
def small(pkg, oracle):
    p = pkg.default_params()
    p.N, p.n = 1024, 13
    q = np.zeros(1, np.uint64)
    oracle.orc_get_primes(1024, 54, 1, q)
    p.Q = int(q[0])
    keys = pkg.key_buffers(p)
    pkg.call("cbs_generate_keys_host", ctypes.byref(p), 31, *(keys[k].ctypes.data for k in pkg.KEY_FIELDS))
    return p, keys, OracleCbs(oracle, p, keys)


@pytest.mark.parametrize("mb", [2, 3, 4])
def test_grouped_keys_encrypt_subset_products(pkg, small, mb):
    p, keys, oc = small
    mbk = pkg.generate_mb_bsk_host(p, 31, mb)
    K, l2, N = len(SUBSETS[mb]), 2 * p.digits_g, p.N
    groups = (p.n + mb - 1) // mb
    mbk = mbk.reshape(groups, K, l2, 2, N)
    s = keys["s_lwe"]
    gmax = (1 << (int(p.Q).bit_length() - p.digits_g * (p.base_g.bit_length() - 1)))
    for g in (0, groups - 1):
        for kk, mask in enumerate(SUBSETS[mb]):
            prod = 1
            for i in range(mb):
                if mask >> i & 1:
                    idx = g * mb + i
                    prod &= int(s[idx]) if idx < p.n else 0
            # row 1 (digit 0, body) has phase prod * g_0
            ph = oc.phase_coef(mbk[g, kk, 1])
            ph[0] -= prod * gmax
            assert max(abs(int(x)) for x in ph) < 2 ** 20


@pytest.mark.parametrize("mb", [2, 3, 4])
def test_grouped_blind_rotation_matches_one_bit(pkg, small, mb):
    p, keys, oc = small
    mbk = pkg.generate_mb_bsk_host(p, 31, mb)
    rng = np.random.default_rng(5 + mb)
    bits = [0, 1, 1]
    a, b = lwe_encrypt_bits(rng, keys["s_lwe"], bits, p.q_lwe)
    one = oc.br_acc(a, b)
    grp = oc.br_acc_mb(a, b, mbk, mb)
    Q, N = p.Q, p.N
    worst = 0
    for i in range(len(bits)):
        d = oc.phase_coef(grp[i]) - oc.phase_coef(one[i])
        e = [((int(x) * N + Q // 2) % Q) - Q // 2 for x in d]  # undo the N^-1 finalize scaling
        worst = max(worst, max(abs(x) for x in e))
    # both are exact; they differ by their key noise (~2^24 per accumulator at n = 13)
    print(f"mb={mb}: max |phase(grouped) - phase(one-bit)| = 2^{np.log2(worst + 1):.1f}")
    assert worst < 2 ** 28
