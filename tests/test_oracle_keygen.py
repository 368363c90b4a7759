"""The oracle's key generation (the CPU legs' keys, so the CPU baseline needs nothing from the
product library) against the product's seeded host key generation: the same seed gives the
same secrets, bootstrapping, HomTrace, SchemeSwitch and extraction keys, test vector, gadget
powers and automorphism maps word for word, and the same grouped (mb = 2) keys."""
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


def test_oracle_grouped_keygen_matches_host(pkg, oracle):
    p = pkg.default_params()
    keys = pkg.generate_keys_host(p, 13)
    want = np.asarray(pkg.generate_mb_bsk_host(p, 13, 2)).reshape(-1)
    got = oracle_keys_mb(oracle, p, keys, 2, 13).reshape(-1)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("preset", ["3x12", "2x18"])
def test_oracle_params_match_presets(pkg, oracle, preset):
    assert vars(oracle_params(oracle, preset)) == pkg.preset_params(preset).as_dict()
