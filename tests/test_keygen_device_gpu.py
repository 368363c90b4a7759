"""Key generation on the device (cbs_keygen_device): every word equal to the oracle's
restatement on the same ChaCha20 stream (secrets, bootstrapping, HomTrace, SchemeSwitch and
extraction keys, and the grouped keys), and AES-128 transciphering with a device-generated key
set decrypting to OpenSSL's keystream."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import RNG_KEY, lwe_decrypt_bits, oracle_chacha_keys, orc_params

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

def test_device_keygen_matches_oracle_word_for_word(pkg, oracle):
    p = pkg.preset_params("2x18")
    p.n = 64  # the same generator at a smaller LWE dimension, so the oracle finishes in seconds
    c = pkg.Context(params=p, max_batch=8)
    try:
        c.keygen_device(RNG_KEY)
        got = c.export_keys()
        want = oracle_chacha_keys(oracle, p, RNG_KEY)
        for f in ("s_lwe", "s_rlwe", "bsk", "ht", "ss", "ksk"):
            assert np.array_equal(np.asarray(got[f]).reshape(-1), want[f].reshape(-1).astype(np.asarray(got[f]).dtype)), f
        assert set(np.unique(want["s_rlwe"])) <= {-1, 0, 1} and 0 < want["s_lwe"].sum() < p.n
        # grouped keys from the same stream (mb = 2: domain 8; the staged mb = 4: domain 10)
        c.set_br_backend(pkg.BR_FFT64)
        vp = ctypes.c_void_p
        oracle.orc_cbs_keygen_chacha_mb.argtypes = [vp, ctypes.c_double, vp, vp, vp, ctypes.c_uint32, vp]
        kw = np.frombuffer(RNG_KEY, np.uint32).copy()
        op = orc_params(p)
        for mb in (2, 4):
            c.set_br_multibit(mb)
            mbk = c.export_mb_bsk()
            wm = np.zeros_like(mbk)
            oracle.orc_cbs_keygen_chacha_mb(ctypes.byref(op), p.sigma_rlwe, kw.ctypes.data, want["s_lwe"].ctypes.data,
                                            want["s_rlwe"].ctypes.data, mb, wm.ctypes.data)
            assert np.array_equal(mbk, wm), mb
    finally:
        c.close()


def test_device_keygen_aes128_decrypts(pkg):
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    import time
    p = pkg.preset_params("2x18")
    c = pkg.Context(params=p, max_batch=256)
    try:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c.keygen_device(None)  # a fresh key from the operating system
        t1 = time.perf_counter()
        c.set_br_backend(pkg.BR_FFT64)
        c.set_br_multibit(2)
        t2 = time.perf_counter()
        print(f"device keygen {1e3 * (t1 - t0):.0f} ms, FFT and grouped key preparation {1e3 * (t2 - t1):.0f} ms")
        keys = c.export_keys()
        key = bytes(range(7, 23))
        pkg.call("cbs_aes128_setup_device", c.handle, key, None)
        blocks = 2
        rng = np.random.default_rng(2)
        ctrs = [rng.bytes(16) for _ in range(blocks)]
        h = np.frombuffer(b"".join(ctrs), np.uint8).copy()
        oa = np.zeros((blocks * 128, p.n), np.uint64)
        ob = np.zeros(blocks * 128, np.uint64)
        pkg.call("cbs_aes128_ctr_transcipher", c.handle, h.ctypes.data, blocks, oa.ctypes.data, ob.ctypes.data)
        got_bits, err = lwe_decrypt_bits(keys["s_lwe"], oa, ob, p.q_lwe)
        enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
        for blk in range(blocks):
            out = bytes(int(sum(int(got_bits[blk * 128 + i * 8 + b]) << b for b in range(8))) for i in range(16))
            assert out == enc.update(ctrs[blk]), blk
        assert max(err) < p.q_lwe // 8
    finally:
        c.close()
