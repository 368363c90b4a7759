"""Exact split-FFT blind rotation (BR_FFT64_SPLIT, the reference's CIRBTS_USE_SPLIT_FFT backend,
bitwise/src/cirbts/cirbts-init.cu:1084-1140 and cirbts-bootstrap.cu:939-1085): the key is cut
into balanced limbs small enough that every FP64 digit x limb product rounds to its exact
integer, so the blind rotation must be bit-identical to the oracle's exact blind rotation and
to the exact NTT kernel -- no tolerance.  A wrong rounding anywhere in 630 steps x 2 polynomials
x N coefficients x 3 limbs changes the output words."""
from __future__ import annotations

import time

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_decrypt_bits, lwe_encrypt_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _blind_rotate(pkg, ctx, a, b):
    p = ctx.params
    batch = a.shape[0]
    da, db = _dev(a), _dev(b)
    mv = torch.zeros((batch, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    pkg.call("cbs_blind_rotate_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), batch, a.shape[1],
             mv.data_ptr(), None)
    torch.cuda.synchronize()
    return mv.cpu().numpy().view(np.uint64).reshape(batch, p.num_lut, 2, p.N)


@pytest.fixture(scope="module", params=["3x12", "2x18"])
def sctx(pkg, request):
    c = pkg.Context(params=pkg.preset_params(request.param), max_batch=512)
    c.keygen(31)
    pkg.call("cbs_context_set_br_backend", c.handle, pkg.BR_FFT64_SPLIT)
    c.preset = request.param
    yield c
    c.close()


def test_split_plan_of_the_context(pkg, sctx):
    limbs, lb, bound = pkg.split_fft_plan(sctx.params)
    print(f"{sctx.preset}: {limbs} limbs of {lb} bits, limb products below 2^{bound}")
    assert limbs == 3 and lb == 18 and bound <= 50


def test_split_blind_rotate_equals_oracle(pkg, oracle, sctx):
    """Bit-identical to the oracle's exact blind rotation (orc_blind_rotate_mv)."""
    p = sctx.params
    keys = sctx.export_keys()
    oc = OracleCbs(oracle, p, keys)
    rng = np.random.default_rng(5)
    bits = [1, 0, 1]
    a, b = lwe_encrypt_bits(rng, keys["s_lwe"], bits, p.q_lwe)
    got = _blind_rotate(pkg, sctx, a, b)
    want = oc.br_mv(a, b)
    assert np.array_equal(got, want)


def test_split_blind_rotate_equals_ntt_kernel_at_296(pkg, sctx):
    """296 ciphertexts (two per SM) of uniformly random masks, split backend against the exact NTT
    kernel on the same keys: every output word equal."""
    p = sctx.params
    rng = np.random.default_rng(11)
    batch = 296
    a = rng.integers(0, p.q_lwe, size=(batch, p.n), dtype=np.uint64)
    b = rng.integers(0, p.q_lwe, size=batch, dtype=np.uint64)
    got = _blind_rotate(pkg, sctx, a, b)
    pkg.call("cbs_context_set_br_backend", sctx.handle, pkg.BR_NTT)
    try:
        want = _blind_rotate(pkg, sctx, a, b)
    finally:
        pkg.call("cbs_context_set_br_backend", sctx.handle, pkg.BR_FFT64_SPLIT)
    diff = int(np.count_nonzero(got != want))
    assert diff == 0, f"{diff} of {got.size} words differ"


def test_split_grouped_blind_rotate_equals_oracle(pkg, oracle, sctx):
    """Grouped mb = 2 on the split backend (keys for {0} {1} {0,1}, combined per spectrum slot as
    c0 (K0 + c1 K01) + c1 K1): bit-identical to the oracle's exact grouped rotation
    (orc_blind_rotate_mb) with the same grouped keys, for encryptions and for uniform masks."""
    p = sctx.params
    limbs, lb, bound = pkg.split_fft_plan(p, 2)
    print(f"{sctx.preset} mb = 2: {limbs} limbs of {lb} bits, limb products below 2^{bound}")
    assert bound <= 50
    keys = sctx.export_keys()
    oc = OracleCbs(oracle, p, keys)
    sctx.set_br_multibit(2)
    try:
        mbk = sctx.export_mb_bsk()
        rng = np.random.default_rng(17)
        a1, b1 = lwe_encrypt_bits(rng, keys["s_lwe"], [1, 0, 1], p.q_lwe)
        a2 = rng.integers(0, p.q_lwe, size=(3, p.n), dtype=np.uint64)
        b2 = rng.integers(0, p.q_lwe, size=3, dtype=np.uint64)
        a, b = np.vstack([a1, a2]), np.concatenate([b1, b2])
        got = _blind_rotate(pkg, sctx, a, b)
    finally:
        sctx.set_br_multibit(1)
    want = oc.br_acc_mb(a, b, mbk, 2)
    assert np.array_equal(got[:, 0], want)


def test_split_grouped_aes128(pkg, sctx):
    """AES-128 CTR with the grouped split blind rotation: keystream equal to OpenSSL's."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    p = sctx.params
    key = bytes(range(96, 112))
    rng = np.random.default_rng(23)
    ctr = rng.bytes(16)
    h = np.frombuffer(ctr, np.uint8).copy()
    sctx.set_br_multibit(2)
    try:
        pkg.call("cbs_aes128_setup", sctx.handle, key, 5)
        oa = np.zeros((128, p.n), np.uint64)
        ob = np.zeros(128, np.uint64)
        pkg.call("cbs_aes128_ctr_transcipher", sctx.handle, h.ctypes.data, 1, oa.ctypes.data, ob.ctypes.data)
    finally:
        sctx.set_br_multibit(1)
    got_bits, err = lwe_decrypt_bits(sctx.export_keys()["s_lwe"], oa, ob, p.q_lwe)
    out = bytes(int(sum(int(got_bits[i * 8 + k]) << k for k in range(8))) for i in range(16))
    assert out == Cipher(algorithms.AES(key), modes.ECB()).encryptor().update(ctr)
    assert max(err) < p.q_lwe // 8


def test_split_aes128_equals_ntt_backend(pkg, sctx):
    """AES-128 CTR on the split backend: the keystream equals OpenSSL's and every output LWE word
    equals the exact NTT backend's on the same keys and counters."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    p = sctx.params
    key = bytes(range(64, 80))
    blocks = 1
    rng = np.random.default_rng(21)
    ctrs = [rng.bytes(16) for _ in range(blocks)]
    h = np.frombuffer(b"".join(ctrs), np.uint8).copy()

    def run():
        pkg.call("cbs_aes128_setup", sctx.handle, key, 5)
        oa = np.zeros((blocks * 128, p.n), np.uint64)
        ob = np.zeros(blocks * 128, np.uint64)
        pkg.call("cbs_aes128_ctr_transcipher", sctx.handle, h.ctypes.data, blocks, oa.ctypes.data, ob.ctypes.data)
        return oa, ob

    sa, sb = run()
    pkg.call("cbs_context_set_br_backend", sctx.handle, pkg.BR_NTT)
    try:
        na, nb = run()
    finally:
        pkg.call("cbs_context_set_br_backend", sctx.handle, pkg.BR_FFT64_SPLIT)
    keys = sctx.export_keys()
    got_bits, err = lwe_decrypt_bits(keys["s_lwe"], sa, sb, p.q_lwe)
    enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    for blk in range(blocks):
        out = bytes(int(sum(int(got_bits[blk * 128 + i * 8 + k]) << k for k in range(8))) for i in range(16))
        assert out == enc.update(ctrs[blk])
    assert np.array_equal(sa, na) and np.array_equal(sb, nb)


def test_split_blind_rotate_timing(pkg, sctx):
    """Per-bootstrap time of the split backend beside the exact NTT and the FP64 FFT one-bit
    kernels, 296 ciphertexts, CUDA events (printed, not asserted)."""
    p = sctx.params
    rng = np.random.default_rng(3)
    batch = 296
    a = _dev(rng.integers(0, p.q_lwe, size=(batch, p.n), dtype=np.uint64))
    b = _dev(rng.integers(0, p.q_lwe, size=batch, dtype=np.uint64))
    mv = torch.zeros((batch, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")

    def time_backend(backend, reps=3):
        pkg.call("cbs_context_set_br_backend", sctx.handle, backend)
        args = (sctx.handle, a.data_ptr(), b.data_ptr(), batch, p.n, mv.data_ptr(), None)
        pkg.call("cbs_blind_rotate_batch_device", *args)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            pkg.call("cbs_blind_rotate_batch_device", *args)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / batch * 1e3

    t0 = time.time()
    try:
        split_us = time_backend(pkg.BR_FFT64_SPLIT)
        sctx.set_br_multibit(2)
        split2_us = time_backend(pkg.BR_FFT64_SPLIT)
        ntt_us = time_backend(pkg.BR_NTT)
        fft_us = time_backend(pkg.BR_FFT64)
    finally:
        pkg.call("cbs_context_set_br_backend", sctx.handle, pkg.BR_FFT64_SPLIT)
        sctx.set_br_multibit(1)
    print(f"{sctx.preset} blind rotation, {batch} cts: split FFT (exact) one-bit {split_us:.1f} us, mb = 2 "
          f"{split2_us:.1f} us, exact NTT {ntt_us:.1f} us, FP64 FFT one-bit (approximate) {fft_us:.1f} us per "
          f"bootstrap ({time.time() - t0:.1f} s)")
    assert split_us > 0 and split2_us > 0 and ntt_us > 0
