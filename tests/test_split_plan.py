"""Limb sizing of the exact split-FFT blind rotation (cbs_split_fft_plan, host only).  The bound
is the largest rounded coefficient of one limb product: |limb| <= 2^(lb-1), |digit| <= 2^(g-1),
N * 2 digits terms and the factor 2 of X^a - 1, so bound_bits = lb + g - 1 + log2 N +
ceil(log2(2 digits)); it must stay <= 50 (the reference's margin, bitwise/src/cirbts/
cirbts-init.cu:1097-1120) and below Q/2."""
from __future__ import annotations

import math

import numpy as np
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


def test_split_plan_small_ring(pkg):
    """N = 1024 (the smoke case's ring): one bit less of N, the same 3 limbs, a bit more margin."""
    p = pkg.preset_params("3x12")
    p.N = 1024
    assert pkg.split_fft_plan(p, 1) == (3, 18, 42)
    assert pkg.split_fft_plan(p, 2) == (3, 18, 44)


def test_split_plan_wide_gadgets(pkg):
    p = pkg.preset_params("3x12")
    p.base_g, p.digits_g = 1 << 24, 2  # 24-bit digits: limbs of at most 14 bits, 4 of them
    assert _plan(pkg, p) == (4, 14, 50)
    p.N = 4096  # one more bit of N: 5 limbs of 13 bits, more than the kernel takes
    with pytest.raises(RuntimeError):
        _plan(pkg, p)


def _negacyclic_exact(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a * b mod X^N + 1 in exact int64 arithmetic (|coefficients| < 2^62 here)."""
    n = len(a)
    full = np.convolve(a, b)  # int64, length 2N - 1
    out = full[:n].copy()
    out[: n - 1] -= full[n:]
    return out


def _monomial(n: int, e: int) -> np.ndarray:
    """X^e - 1 mod X^N + 1 (0 <= e < 2N) as an int64 coefficient vector."""
    m = np.zeros(n, np.int64)
    m[e % n] += 1 if e < n else -1
    m[0] -= 1
    return m


@pytest.mark.parametrize("preset,mb", [("3x12", 1), ("2x18", 1), ("2x18", 2)])
def test_limb_products_round_exactly_in_fp64(pkg, preset, mb):
    """The arithmetic the split kernel relies on, restated with numpy's FP64 FFT: digit
    polynomials at the largest balanced digits, key limbs at the largest balanced limbs, summed
    over the 2 digits rows and multiplied by the step's monomials (X^a - 1, or c0 K0 + c1 K1 +
    c0 c1 K01 for mb = 2), computed through one complex product per row in the frequency domain
    and one inverse transform.  Every coefficient must sit within a small fraction of 1/2 of the
    exact integer product; the worst distance is reported."""
    p = pkg.preset_params(preset)
    limbs, lb, bound = pkg.split_fft_plan(p, mb)
    g = int(p.base_g).bit_length() - 1
    n, rows = int(p.N), 2 * int(p.digits_g)
    rng = np.random.default_rng(7 + mb)
    # extreme-valued inputs (+-2^(g-1), +-2^(lb-1)): every term at its largest magnitude
    dig = rng.choice([-(1 << (g - 1)), (1 << (g - 1)) - 1], size=(rows, n)).astype(np.int64)
    keys = 3 if mb == 2 else 1
    lim = rng.choice([-(1 << (lb - 1)), (1 << (lb - 1))], size=(keys, rows, n)).astype(np.int64)
    a0, a1 = (int(x) for x in rng.integers(1, 2 * n, size=2))
    monos = [_monomial(n, a0)] if mb == 1 else [_monomial(n, a0), _monomial(n, a1),
                                                 _negacyclic_exact(_monomial(n, a0), _monomial(n, a1))]
    exact = np.zeros(n, np.int64)
    for k in range(keys):
        t = np.zeros(n, np.int64)
        for r in range(rows):
            t += _negacyclic_exact(dig[r], lim[k, r])
        exact += _negacyclic_exact(t, monos[k])
    assert np.abs(exact).max() < 2.0 ** bound
    # FP64: length-4N transforms of the zero-padded operands (the linear product of three
    # length-N factors has 3N - 2 terms), folded negacyclically
    f = lambda v: np.fft.fft(np.concatenate([v.astype(np.float64), np.zeros(3 * n)]))  # noqa: E731
    spec = np.zeros(4 * n, np.complex128)
    for k in range(keys):
        fm = f(monos[k])
        for r in range(rows):
            spec += f(dig[r]) * f(lim[k, r]) * fm
    lin = np.fft.ifft(spec).real
    approx = lin[:n] - lin[n:2 * n] + lin[2 * n:3 * n] - lin[3 * n:]
    err = np.abs(approx - exact).max()
    print(f"{preset} mb={mb}: |exact| max 2^{np.log2(np.abs(exact).max()):.1f} (bound 2^{bound}), "
          f"FP64 distance from the exact integers {err:.3g}")
    assert err < 0.125
    assert np.array_equal(np.rint(approx).astype(np.int64), exact)
