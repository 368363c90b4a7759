"""CPU checks of the torus-32 gate-bootstrap oracle with host-generated keys: every gate's
truth table after blind rotation, sample extract and key switch (small LWE dimension so the
exact integer products finish in seconds)."""
from __future__ import annotations

import numpy as np
import pytest

from gate_harness import TRUTH, OracleGate, declare_gate, decrypt, encrypt, phase


@pytest.fixture(scope="module")
def setup(pkg, oracle):
    p = pkg.gate_default_params()
    p.n = 24  # the blind rotation is generic in n; a short one keeps the exact oracle fast
    keys = pkg.gate_generate_keys_host(p, 5)
    return p, keys, OracleGate(declare_gate(oracle), p, keys)


def test_keys_shapes_and_determinism(pkg, setup):
    p, keys, _ = setup
    again = pkg.gate_generate_keys_host(p, 5)
    for k in keys:
        assert np.array_equal(keys[k], again[k])
    assert set(np.unique(keys["s_lwe"])) <= {0, 1} and set(np.unique(keys["z_rlwe"])) <= {0, 1}


def test_ksk_rows_decrypt_to_scaled_key(setup):
    p, keys, _ = setup
    s = keys["s_lwe"]
    ksk = keys["ksk"]
    for (i, l, v) in [(0, 0, 0), (5, 3, 2), (p.N - 1, p.ks_levels - 1, 1)]:
        row = ksk[i, l, v]
        ph = phase(s, row[None, :p.n], row[None, p.n])[0]
        want = ((v + 1) * int(keys["z_rlwe"][i]) << (32 - (l + 1) * p.ks_base_bits)) % (1 << 32)
        want = want - (1 << 32) if want >= 1 << 31 else want
        assert abs(int(ph) - want) < 2 ** 22


@pytest.mark.parametrize("gate", range(6))
def test_oracle_gate_truth_tables(setup, gate):
    p, keys, og = setup
    rng = np.random.default_rng(10 + gate)
    x = np.array([0, 0, 1, 1], np.uint8)
    y = np.array([0, 1, 0, 1], np.uint8)
    a1, b1 = encrypt(rng, keys["s_lwe"], x, p.sigma_lwe)
    a2, b2 = encrypt(rng, keys["s_lwe"], y, p.sigma_lwe)
    a, b = og.combine(gate, a1, b1, a2, b2)
    ext = og.blind_rotate(a, b)
    oa, ob = og.keyswitch(ext)
    got = decrypt(keys["s_lwe"], oa, ob)
    assert list(got) == [TRUTH[gate](int(u), int(v)) for u, v in zip(x, y)]
    # the extracted LWE (under z) carries +-1/8 with small noise
    ph = phase(keys["z_rlwe"], ext[:, :p.N], ext[:, p.N])
    assert np.all(np.abs(np.abs(ph) - (1 << 29)) < 1 << 26)
