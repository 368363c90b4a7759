"""CPU analysis of FP32 external products for each workload's parameters, with numpy's
single-precision FFT standing in for the FP32 transform (the folded negacyclic form of the
kernels: fold, twist, M-point complex FFT, product, inverse, untwist).

A limb split k = sum_j 2^(b j) k_j recombined in integers (the reference's split-FFT
backend, bitwise/src/cirbts/cirbts-init.cu:1084-1140, sizes its FP64 limbs by
limb_bits = 50 - (log2 Bg + log2 N + log2 digitsG2)) is exact only when every limb's
product sum rounds to the right integer; a limb whose product is not exact contributes its
FP32 error times the limb's weight.  Hence:

* torus-32 gate (N = 1024, digits of 2^7, 6 digit polynomials per column): an 8-bit top limb
  rounds exactly (distance to the integer far below 1/2), so the split k = lo + 2^24 hi
  leaves only the lo limb's FP32 error, about 2^11 rms of 2^32 per external product
  (whole-key FP32: about 2^19);
* the CBS blind rotation (54-bit Q, N = 2048, digits of 2^12): only limbs of at most 3 bits
  round exactly (18 or more limbs for 54 bits, each with its own inverse transform and key
  spectra, against one FP64 product), and the whole-key FP32 product misses by ~2^-7 of Q;
* the torus-64 level-2 rotation of the PFKS circuit bootstrap (N = 2048, digits of 2^9):
  limbs of at most 6 bits (11 or more for 64 bits).
Measured boundaries (max distance over 6 trials): 12-bit digits 0.14 / 0.31 / 0.63 / 1.25 at
2 / 3 / 4 / 5-bit limbs; 9-bit digits 0.14 / 0.31 / 0.63 / 1.25 at 5 / 6 / 7 / 8 bits; 7-bit
digits (N = 1024) 0.16 / 0.38 / 0.75 at 8 / 9 / 10 bits."""
from __future__ import annotations

import numpy as np
import pytest

sfft = pytest.importorskip("scipy.fft")


def _fold_fft(a, N, dt):
    M = N // 2
    j = np.arange(M)
    z = (a[..., :M] + 1j * a[..., M:]).astype(dt) * np.exp(1j * np.pi * j / N).astype(dt)
    return sfft.fft(z, axis=-1)


def _unfold_ifft(Z, N, dt):
    M = N // 2
    j = np.arange(M)
    z = sfft.ifft(Z, axis=-1) * np.exp(-1j * np.pi * j / N).astype(dt)
    return np.concatenate([z.real, z.imag], axis=-1).astype(np.float64)


def _limb_rounding(rng, N, digit_bits, limb_bits, rows=6, trials=4):
    """max |FP32 result - exact integer| of sum_r d_r * k_r with balanced digits and limbs."""
    worst = 0.0
    for _ in range(trials):
        d = rng.integers(-(1 << (digit_bits - 1)), 1 << (digit_bits - 1), (rows, N)).astype(np.float64)
        k = rng.integers(-(1 << (limb_bits - 1)), 1 << (limb_bits - 1), (rows, N)).astype(np.float64)
        y32 = _unfold_ifft((_fold_fft(d, N, np.complex64) * _fold_fft(k, N, np.complex64)).sum(0), N, np.complex64)
        y64 = _unfold_ifft((_fold_fft(d, N, np.complex128) * _fold_fft(k, N, np.complex128)).sum(0), N,
                           np.complex128)
        worst = max(worst, float(np.abs(y32 - np.rint(y64)).max()))
    return worst


def _whole_key_error(rng, N, digit_bits, key_bits, rows=6, trials=2):
    """rms error of the whole-key FP32 product relative to the modulus 2^key_bits."""
    errs = []
    for _ in range(trials):
        d = rng.integers(-(1 << (digit_bits - 1)), 1 << (digit_bits - 1), (rows, N)).astype(np.float64)
        k = rng.uniform(-0.5, 0.5, (rows, N))  # centred key / modulus
        y32 = _unfold_ifft((_fold_fft(d, N, np.complex64) * _fold_fft(k, N, np.complex64)).sum(0), N, np.complex64)
        y64 = _unfold_ifft((_fold_fft(d, N, np.complex128) * _fold_fft(k, N, np.complex128)).sum(0), N,
                           np.complex128)
        errs.append(y32 - y64)
    e = np.concatenate(errs)
    return float(np.sqrt(np.mean(e ** 2)))  # in units of the modulus


def test_gate_split_top_limb_is_exact():
    rng = np.random.default_rng(1)
    # the kernel's split: 8-bit top limb at N = 1024, 7-bit at N = 2048, 7-bit digits
    assert _limb_rounding(rng, 1024, 7, 8) < 0.35
    assert _limb_rounding(rng, 2048, 7, 7) < 0.35
    # whole 32-bit keys: the FP32 error is 2^-13 of the torus (2^19 of 2^32)
    rel = _whole_key_error(rng, 1024, 7, 32)
    assert 2.0 ** -15 < rel < 2.0 ** -11


def test_cbs_modulus_needs_many_exact_fp32_limbs():
    rng = np.random.default_rng(2)
    # 12-bit digits at N = 2048: 2-bit limbs round exactly, 5-bit limbs do not
    assert _limb_rounding(rng, 2048, 12, 2) < 0.35
    assert _limb_rounding(rng, 2048, 12, 5) > 0.5
    # whole 54-bit keys: the product is off by about 2^-7 of Q per external product
    rel = _whole_key_error(rng, 2048, 12, 54)
    assert rel > 2.0 ** -9


def test_torus64_level2_needs_narrow_limbs():
    rng = np.random.default_rng(3)
    # 9-bit digits at N = 2048: 5-bit limbs round exactly, 8-bit limbs do not
    assert _limb_rounding(rng, 2048, 9, 5) < 0.35
    assert _limb_rounding(rng, 2048, 9, 8) > 0.5
