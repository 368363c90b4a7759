"""The 2^18 x 2 blind-rotation gadget (cbs_params_preset(CBS_PARAMS_AES_2X18)): the exact NTT
blind rotation bit-exact against the oracle, the grouped FP64 FFT blind rotation within its
phase-error bound of the oracle's exact grouped rotation, and AES-128 end to end on the
headline configuration (FFT backend, mb = 2) with the decryption-failure probability implied
by the measured noise of the output bits."""
from __future__ import annotations

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_decrypt_bits, lwe_encrypt_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

# Grouped FFT blind rotation, max |phase error| against the exact grouped oracle over all
# coefficients (before the N^-1 finalize).  With 18-bit digits (|d| <= 2^17) each product of a
# digit spectrum by a 54-bit key spectrum is 2^6 larger than with 12-bit digits, and so is its
# FP64 rounding error: ~2^22-2^24 per coefficient and group, ~2^34 rms and ~2^36-2^37 max over
# 315 groups (the 2^12 x 3 gadget measures 2^30.7 max).  Only the constant coefficient of each
# multi-value RLWE survives the trace, where it adds to the ~2^27 rms HomTrace noise of the RGSW
# rows' constant term only; in a CMux it is multiplied by one digit per row instead of being
# convolved over N coefficients, so it contributes like 2^34 / sqrt(N) ~ 2^28.5 would on every
# coefficient.  Bound: 2^39.
FFT_PHASE_TOL_LOG2_2X18 = 39.0
# AES: per-bit failure probability of the output LWEs (Gaussian tail of the measured error at
# the decision margin q/4) must stay at or below 2^-40
PFAIL_LOG2_MAX = -40.0


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


@pytest.fixture(scope="module")
def wctx(pkg):
    c = pkg.Context(params=pkg.preset_params("2x18"), max_batch=2048)
    c.keygen(47)
    yield c
    c.close()


@pytest.fixture(scope="module")
def wkeys(wctx):
    return wctx.export_keys()


@pytest.fixture(scope="module")
def woc(oracle, wctx, wkeys):
    return OracleCbs(oracle, wctx.params, wkeys)


def test_preset_values(pkg):
    p = pkg.preset_params("2x18")
    d = pkg.default_params()
    assert (p.base_g, p.digits_g) == (1 << 18, 2)
    assert pkg.preset_params("3x12").as_dict() == d.as_dict()
    for k, v in d.as_dict().items():
        if k not in ("base_g", "digits_g"):
            assert getattr(p, k) == v, k


def test_exact_blind_rotate_bit_exact(pkg, wctx, wkeys, woc):
    p = wctx.params
    rng = np.random.default_rng(5)
    a, b = lwe_encrypt_bits(rng, wkeys["s_lwe"], [1, 0], p.q_lwe)
    mv = torch.zeros((2, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    da, db = _dev(a), _dev(b)
    pkg.call("cbs_blind_rotate_batch_device", wctx.handle, da.data_ptr(), db.data_ptr(), 2, p.n, mv.data_ptr(), None)
    torch.cuda.synchronize()
    want = woc.br_mv(a, b)
    assert np.array_equal(mv.cpu().numpy().view(np.uint64).reshape(want.shape), want)


@pytest.mark.parametrize("mb", [3, 4])
def test_grouped_fft_blind_rotate_phase_error_mb3_mb4(pkg, wctx, wkeys, woc, mb):
    """The generic grouped kernel on the two-digit gadget: mb = 3 and the staged mb = 4 (an mb = 3
    step and a one-bit step per group of 4) against the oracle's exact grouped rotation."""
    p = wctx.params
    bits = [1, 0, 1]
    B = len(bits)
    pkg.call("cbs_context_set_br_backend", wctx.handle, pkg.BR_FFT64)
    wctx.set_br_multibit(mb)
    try:
        mbk = wctx.export_mb_bsk()
        rng = np.random.default_rng(60 + mb)
        a, b = lwe_encrypt_bits(rng, wkeys["s_lwe"], bits, p.q_lwe)
        mv = torch.zeros((B, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
        da, db = _dev(a), _dev(b)
        pkg.call("cbs_blind_rotate_batch_device", wctx.handle, da.data_ptr(), db.data_ptr(), B, p.n, mv.data_ptr(),
                 None)
        torch.cuda.synchronize()
    finally:
        wctx.set_br_multibit(2)
        pkg.call("cbs_context_set_br_backend", wctx.handle, pkg.BR_NTT)
    got = mv.cpu().numpy().view(np.uint64).reshape(B, p.num_lut, 2, p.N)
    want = woc.br_acc_mb(a, b, mbk, mb)
    Q, N = p.Q, p.N
    worst = 0
    for i in range(B):
        d = woc.phase_coef(got[i, 0]) - woc.phase_coef(want[i])
        e = [((int(x) * N + Q // 2) % Q) - Q // 2 for x in d]
        worst = max(worst, max(abs(x) for x in e))
    log2 = np.log2(worst + 1)
    print(f"2x18 grouped FFT blind rotation (mb = {mb}): max |phase error| 2^{log2:.1f}")
    assert log2 < FFT_PHASE_TOL_LOG2_2X18


@pytest.mark.parametrize("schedule,bits", [("digitwise", [0, 1, 1]), ("lockstep", [0, 1, 1]),
                                           ("paired", [0, 1, 1]), ("paired", [1, 0, 1, 1])])
def test_grouped_fft_blind_rotate_phase_error(pkg, wctx, wkeys, woc, schedule, bits):
    """Every schedule of the two-digit grouped rotation; the paired one (two ciphertexts per CTA)
    on an odd batch (its last CTA runs a copy of the last ciphertext and writes nothing for it)
    and an even one."""
    p = wctx.params
    sched = {"digitwise": pkg.BR_SCHEDULE_DIGITWISE, "lockstep": pkg.BR_SCHEDULE_LOCKSTEP,
             "paired": pkg.BR_SCHEDULE_PAIRED}[schedule]
    B = len(bits)
    pkg.call("cbs_context_set_br_backend", wctx.handle, pkg.BR_FFT64)
    wctx.set_br_multibit(2)
    wctx.set_br_schedule(sched)
    try:
        mbk = wctx.export_mb_bsk()
        rng = np.random.default_rng(6)
        a, b = lwe_encrypt_bits(rng, wkeys["s_lwe"], bits, p.q_lwe)
        mv = torch.full((B + 1, p.num_lut, 2, p.N), 7, dtype=torch.int64, device="cuda")
        da, db = _dev(a), _dev(b)
        pkg.call("cbs_blind_rotate_batch_device", wctx.handle, da.data_ptr(), db.data_ptr(), B, p.n, mv.data_ptr(),
                 None)
        torch.cuda.synchronize()
    finally:
        wctx.set_br_schedule(pkg.BR_SCHEDULE_AUTO)
        pkg.call("cbs_context_set_br_backend", wctx.handle, pkg.BR_NTT)
    allv = mv.cpu().numpy().view(np.uint64)
    assert (allv[B] == 7).all()  # nothing written past the batch
    got = allv[:B].reshape(B, p.num_lut, 2, p.N)
    want = woc.br_acc_mb(a, b, mbk, 2)
    Q, N = p.Q, p.N
    worst, sq, cnt = 0, 0.0, 0
    for i in range(B):
        d = woc.phase_coef(got[i, 0]) - woc.phase_coef(want[i])
        e = [((int(x) * N + Q // 2) % Q) - Q // 2 for x in d]
        worst = max(worst, max(abs(x) for x in e))
        sq += sum(float(x) * float(x) for x in e)
        cnt += len(e)
    log2 = np.log2(worst + 1)
    print(f"2x18 grouped FFT blind rotation ({schedule}, batch {B}): phase error rms 2^{0.5 * np.log2(sq / cnt):.1f}, max 2^{log2:.1f}")
    assert log2 < FFT_PHASE_TOL_LOG2_2X18


def test_aes128_16_blocks_grouped_fft_pfail(pkg, wctx, wkeys):
    """16 seeded random blocks under a seeded random key on the headline configuration: every
    keystream block equals OpenSSL AES-128, and the Gaussian tail of the output bits' measured
    error (2048 bits, sigma over all of them) at the decision margin q/4 is below 2^-40."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    p = wctx.params
    rng = np.random.default_rng(1818)
    key = rng.bytes(16)
    blocks = 16
    pkg.call("cbs_context_set_br_backend", wctx.handle, pkg.BR_FFT64)
    wctx.set_br_multibit(2)
    try:
        pkg.call("cbs_aes128_setup_device", wctx.handle, key, rng.bytes(32))
        ctrs = [rng.bytes(16) for _ in range(blocks)]
        bits = np.array([[(c[t // 8] >> (t % 8)) & 1 for t in range(128)] for c in ctrs], np.uint8).reshape(-1)
        oa = torch.zeros((blocks * 128, p.n), dtype=torch.int64, device="cuda")
        ob = torch.zeros(blocks * 128, dtype=torch.int64, device="cuda")
        dbits = torch.from_numpy(bits).cuda()
        pkg.call("cbs_aes128_ctr_transcipher_device", wctx.handle, dbits.data_ptr(), blocks, oa.data_ptr(),
                 ob.data_ptr(), 1, None)
        torch.cuda.synchronize()
    finally:
        pkg.call("cbs_context_set_br_backend", wctx.handle, pkg.BR_NTT)
    got_bits, err = lwe_decrypt_bits(wkeys["s_lwe"], oa.cpu().numpy().view(np.uint64),
                                     ob.cpu().numpy().view(np.uint64), p.q_lwe)
    enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    for blk in range(blocks):
        out = bytes(int(sum(int(got_bits[blk * 128 + i * 8 + b]) << b for b in range(8))) for i in range(16))
        assert out == enc.update(ctrs[blk]), blk
    e = np.asarray(err, np.float64)
    sigma = float(np.sqrt(np.mean(e * e)))
    lp = pkg.log2_pfail_gaussian(sigma, p.q_lwe / 4)
    print(f"2x18 AES 16 blocks: output error sigma {sigma:.1f}, max {e.max():.0f} (margin {p.q_lwe // 4}); "
          f"p_fail per bit 2^{lp:.0f}")
    assert lp <= PFAIL_LOG2_MAX
