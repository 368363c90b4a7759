"""Limb sizing of the exact split-FFT blind rotation (cbs_split_fft_plan, host only).  The bound
is the largest rounded coefficient of one limb product: |limb| <= 2^(lb-1), |digit| <= 2^(g-1),
N * 2 digits terms and the factor 2 of X^a - 1, so bound_bits = lb + g - 1 + log2 N +
ceil(log2(2 digits)); it must stay <= 50 (the reference's margin, bitwise/src/cirbts/
cirbts-init.cu:1097-1120) and below Q/2."""
from __future__ import annotations

import math

import pytest


def _plan(pkg, p):
    return pkg.split_fft_plan(p)


@pytest.mark.parametrize("preset,want", [("3x12", (3, 18, 43)), ("2x18", (3, 18, 48))])
def test_split_plan_presets(pkg, preset, want):
    p = pkg.preset_params(preset)
    limbs, lb, bound = _plan(pkg, p)
    assert (limbs, lb, bound) == want
    g = int(p.base_g).bit_length() - 1
    logn = int(p.N).bit_length() - 1
    assert bound == lb + g - 1 + logn + math.ceil(math.log2(2 * p.digits_g))
    # balanced limbs cover the centred key coefficients: limbs * lb >= log2 Q
    assert limbs * lb >= int(p.Q).bit_length()
    # the reference's unsigned-limb sizing gives the same limb count on these presets
    ref_bits = 50 - (g + logn + math.ceil(math.log2(2 * p.digits_g)))
    assert math.ceil(int(p.Q).bit_length() / ref_bits) == limbs


@pytest.mark.parametrize("preset,want", [("3x12", (3, 18, 45)), ("2x18", (3, 18, 50))])
def test_split_plan_grouped(pkg, preset, want):
    """mb = 2: the monomial factor c0 + c1 + c0 c1 has L1 norm 8, two bits above X^a - 1."""
    assert pkg.split_fft_plan(pkg.preset_params(preset), 2) == want


def test_split_plan_wide_gadgets(pkg):
    p = pkg.preset_params("3x12")
    p.base_g, p.digits_g = 1 << 24, 2  # 24-bit digits: limbs of at most 14 bits, 4 of them
    assert _plan(pkg, p) == (4, 14, 50)
    p.N = 4096  # one more bit of N: 5 limbs of 13 bits, more than the kernel takes
    with pytest.raises(RuntimeError):
        _plan(pkg, p)
