"""The oracle's key generation (the CPU legs' keys, so the CPU baseline needs nothing from the
product library) against the product's seeded host key generation: the same seed gives the
same secrets, bootstrapping, HomTrace, SchemeSwitch and extraction keys, test vector, gadget
powers and automorphism maps word for word, and the same grouped (mb = 2, 4) keys."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import oracle_keys, oracle_keys_mb, oracle_params


@pytest.mark.parametrize("preset", ["3x12", "2x18"])
def test_oracle_keygen_matches_host_keygen(pkg, oracle, preset):
    p = pkg.preset_params(preset)
    want = pkg.generate_keys_host(p, 9)
    got = oracle_keys(oracle, p, 9)
    for f in ("s_lwe", "s_rlwe", "bsk", "ht", "ss", "ksk", "tv", "gpow", "maps"):
        assert np.array_equal(np.asarray(got[f]).reshape(-1), np.asarray(want[f]).reshape(-1).astype(got[f].dtype)), f


@pytest.mark.parametrize("mb", [2, 4])
def test_oracle_grouped_keygen_matches_host(pkg, oracle, mb):
    p = pkg.default_params()
    keys = pkg.generate_keys_host(p, 13)
    want = np.asarray(pkg.generate_mb_bsk_host(p, 13, mb)).reshape(-1)
    got = oracle_keys_mb(oracle, p, keys, mb, 13).reshape(-1)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("preset", ["3x12", "2x18"])
def test_oracle_params_match_presets(pkg, oracle, preset):
    assert vars(oracle_params(oracle, preset)) == pkg.preset_params(preset).as_dict()


def test_oracle_chacha_keygen_semantics(pkg, oracle):
    """The restatement of the device key generation makes valid keys: bootstrapping-key rows
    2j + 1 decrypt to s_i g_j (coefficient 0 of a constant polynomial), HomTrace rows to
    -sigma_r(s) g_j, the SchemeSwitch rows to s^2 g_j, and extraction-key rows to
    v s'_i base^j, all up to small noise."""
    from cbs_harness import RNG_KEY, oracle_chacha_keys
    from conftest import oracle_tables
    p = pkg.preset_params("2x18")
    p.n = 16
    k = oracle_chacha_keys(oracle, p, RNG_KEY)
    N, Q = p.N, p.Q
    rp, _, irp, _, ninv = oracle_tables(oracle, N, Q)
    s = (k["s_rlwe"].astype(np.int64) % Q).astype(np.uint64)
    s_ntt = s.copy()
    oracle.orc_ntt_forward(s_ntt, 1, N, Q, rp)

    def phase(ct):
        ph = ((ct[1].astype(object) - ct[0].astype(object) * s_ntt.astype(object)) % Q).astype(np.uint64)
        oracle.orc_ntt_inverse(ph, 1, N, Q, irp, int(ninv[0]))
        return np.array([int(x) - Q if int(x) > Q // 2 else int(x) for x in ph], dtype=object)

    ign = 54 - 2 * 18
    for i in range(p.n):
        for j in range(2):
            ph = phase(k["bsk"][i, 2 * j + 1])
            ph[0] -= int(k["s_lwe"][i]) * (1 << (ign + 18 * j))
            assert max(abs(int(x)) for x in ph) < 64
    ph = phase(k["ss"][0])
    s2 = np.zeros(N, dtype=object)  # s^2 in Z[X]/(X^N + 1)
    sr = k["s_rlwe"].astype(object)
    for a in np.nonzero(k["s_rlwe"])[0]:
        for b in np.nonzero(k["s_rlwe"])[0]:
            e = int(a) + int(b)
            v = sr[a] * sr[b]
            if e < N:
                s2[e] += v
            else:
                s2[e - N] -= v
    g0 = 1 << (54 - 5 * 9)
    diff = [((int(x) - int(y) * g0 + Q // 2) % Q) - Q // 2 for x, y in zip(ph, s2)]
    assert max(abs(d) for d in diff) < 64
    # extraction key rows: LWE_s(v s'_i base^j) mod qks
    qks, base = p.qks, p.base_ks
    ksk = k["ksk"].astype(np.int64)
    sl = k["s_lwe"].astype(np.int64)
    for (j, i, v) in [(0, 0, 1), (1, 5, 3), (0, N - 1, base - 1)]:
        row = ksk[j, i, v]
        dec = (int(row[p.n]) - int(row[: p.n] @ sl)) % qks
        m = (v * (int(k["s_rlwe"][i]) % qks) * (1 if j == 0 else base)) % qks
        assert min((dec - m) % qks, (m - dec) % qks) < 8
