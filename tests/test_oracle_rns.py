"""CPU checks of the RNS oracle: transform identities and key-switching semantics.

The multi-prime NTT applies the per-prime tables pinned against the reference's host code
(tests/golden/reference_host.json), so its pin is the 1-D one.  Base conversion, modup,
moddown and the inner product follow src/rns_bconv.cu and src/eval_key_switch.cu; they are
checked here by what key switching must do: ct' = keyswitch(c2) decrypts under s to
c2 * s' up to a small error.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import oracle_tables
from rns_harness import (addmod, crt_centered, declare_rns, make_switch_key, mulmod, ntt, rns_primes, small_to_rns,
                         submod)


@pytest.fixture(scope="module")
def orns(oracle):
    return declare_rns(oracle)


def test_rns_ntt_matches_single_prime_ntt(orns):
    n = 1 << 13
    q, p = rns_primes(orns, n, 3, 1)
    mods = np.concatenate([q, p])
    rng = np.random.default_rng(5)
    x = np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in mods])
    y = ntt(orns, x, mods)
    for i, m in enumerate(mods):
        rp = oracle_tables(orns, n, int(m))[0]
        one = x[i].copy()
        orns.orc_ntt_forward(one, 1, n, int(m), rp)
        assert np.array_equal(one, y[i])
    assert np.array_equal(ntt(orns, y, mods, inverse=True), x)


@pytest.mark.parametrize("size_q,size_p,size_ql", [(4, 2, 4), (5, 2, 5), (5, 2, 3), (3, 1, 3), (6, 3, 4)])
def test_oracle_keyswitch_decrypts(orns, size_q, size_p, size_ql):
    n = 1 << 13
    logn = 13
    rng = np.random.default_rng(100 + size_q * 10 + size_p + size_ql)
    q, p = rns_primes(orns, n, size_q, size_p)
    chain = np.concatenate([q, p])
    s = rng.integers(-1, 2, n)
    sp = rng.integers(-1, 2, n)
    s_ntt = ntt(orns, small_to_rns(s, chain), chain)
    sp_ntt = ntt(orns, small_to_rns(sp, q), q)
    evk = make_switch_key(orns, rng, n, q, p, s_ntt, sp_ntt)
    ql = q[:size_ql]
    c2 = np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in ql])
    ct = np.zeros((2, size_ql, n), np.uint64)
    orns.orc_keyswitch(ct, np.ascontiguousarray(c2), np.ascontiguousarray(evk), logn, q, size_ql, size_q, p, size_p)
    colq = ql.reshape(-1, 1)
    dec = addmod(ct[0], mulmod(ct[1], s_ntt[:size_ql], colq), colq)
    err = submod(dec, mulmod(c2, sp_ntt[:size_ql], colq), colq)
    coef = ntt(orns, err, ql, inverse=True)
    e = crt_centered(coef, ql, 64)
    assert max(abs(v) for v in e) < 2 ** 30, max(abs(v) for v in e)
