"""CPU checks of the torus circuit bootstrap with PFKS (oracle + host keys, small rings):
the level-2 blind rotation yields LWEs of m g_k, the private functional key switch turns
them into RGSW rows whose phases are m g_k (row 2k+1) and -m g_k z1 (row 2k)."""
from __future__ import annotations

import numpy as np
import pytest

from gate_harness import encrypt
from tcb_harness import OracleTcb, centered, declare_tcb, lwe64_phase_top, rgsw_row_errors


@pytest.fixture(scope="module")
def setup(pkg, oracle):
    p = pkg.tcb_default_params()
    p.n, p.N2, p.N1 = 12, 256, 64
    keys = pkg.tcb_generate_keys_host(p, 9)
    return p, keys, OracleTcb(declare_tcb(oracle), p, keys)


def test_host_keys_deterministic(pkg, setup):
    p, keys, _ = setup
    again = pkg.tcb_generate_keys_host(p, 9)
    for k in keys:
        assert np.array_equal(keys[k], again[k])


def test_pfks_key_rows_decrypt(setup):
    from tcb_harness import rlwe_phase
    p, keys, _ = setup
    z1, z2 = keys["z1"], keys["z2"]
    for (f, i, j, v) in [(1, 0, 0, 0), (1, 7, 3, 9), (0, 5, 1, 2), (0, p.N2, 7, 14)]:
        row = keys["pfks"][f, i, j, v]
        y = int(z2[i]) if i < p.N2 else 1
        m0 = ((v + 1) * y << (32 - (j + 1) * p.pfks_base_bits)) % (1 << 32)
        ph = rlwe_phase(row, z1)
        want = np.zeros(p.N1, np.int64)
        if f == 1:
            want[0] = m0
        else:
            want = -m0 * z1.astype(np.int64)
        assert np.max(np.abs(centered(ph - want))) < 2 ** 12


def test_circuit_bootstrap_rows(setup):
    p, keys, ot = setup
    rng = np.random.default_rng(3)
    bits = np.array([1, 0, 1], np.uint8)
    a, b = encrypt(rng, keys["s0"], bits, p.sigma_lwe)
    ext = ot.blind_rotate(a, b)
    # level-2 LWEs carry m g_k under z2 (64-bit torus; phases in units of 2^-32); the bound is
    # the gadget's rounding of the 37 dropped bits times the binary key: ~2^-28 sqrt(N2/2 n)
    for i, m in enumerate(int(x) for x in bits):
        for k in range(p.cb_levels):
            g = 2.0 ** (32 - (k + 1) * p.cb_bits)
            assert abs(lwe64_phase_top(ext[i, k], keys["z2"]) - m * g) < 2 ** 12
    rgsw = ot.pfks(ext)
    err = rgsw_row_errors(rgsw, bits, keys["z1"], p.cb_bits, p.cb_levels)
    assert np.max(np.abs(err)) < 2 ** 23
