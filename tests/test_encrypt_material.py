"""Device encryption of the AES material (cbs_aes128_setup_device) and its CPU restatement.

CPU: the oracle's ChaCha20 block function is pinned against OpenSSL's ChaCha20 (through
`cryptography`: 16-byte nonce = 4-byte little-endian block counter + 12-byte nonce), the
library's noise table equals the oracle's, and the sampled noise has the discrete Gaussian's
moments.  GPU: every table / round-key / round-0-bit sample the device writes equals the
oracle's restatement word for word, and the AES transcipher on device-encrypted material
decrypts to AES-128."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import oracle_tables

vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
RNG_KEY = bytes(range(100, 132))


@pytest.fixture(scope="module")
def orc(oracle):
    oracle.orc_chacha20_block.argtypes = [vp, u32, vp, vp]
    oracle.orc_uniform_mod.argtypes = [vp, u64]
    oracle.orc_uniform_mod.restype = u64
    oracle.orc_cdt_table.argtypes = [ctypes.c_double, vp, u32]
    oracle.orc_cdt_table.restype = u32
    oracle.orc_cdt_sample.argtypes = [u64, vp, u32]
    oracle.orc_cdt_sample.restype = ctypes.c_int64
    oracle.orc_encrypt_words_rlwe.argtypes = [vp, vp, u32, u32, u32, u64, vp, vp, vp, u32, vp]
    oracle.orc_encrypt_bits_lwe.argtypes = [vp, vp, u32, u32, u64, vp, vp, u32, vp, vp]
    return oracle


def _key_words(key: bytes) -> np.ndarray:
    return np.frombuffer(key, dtype="<u4").astype(np.uint32).copy()


def _orc_cdt(orc, sigma: float) -> np.ndarray:
    T = np.zeros(256, np.uint64)
    n = orc.orc_cdt_table(sigma, T.ctypes.data, 256)
    return T[:n].copy()


@pytest.mark.parametrize("counter,nonce", [(0, (0, 0, 0)), (1, (7, 1, 0)), (2047, (2091, 1, 0)),
                                           (0xFFFFFFFF, (0xDEADBEEF, 2, 0x12345678))])
def test_chacha20_block_matches_openssl(orc, counter, nonce):
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    key = RNG_KEY
    iv = counter.to_bytes(4, "little") + b"".join(x.to_bytes(4, "little") for x in nonce)
    want = Cipher(algorithms.ChaCha20(key, iv), mode=None).encryptor().update(bytes(64))
    out = np.zeros(16, np.uint32)
    kw = _key_words(key)
    nw = np.array(nonce, np.uint32)
    orc.orc_chacha20_block(kw.ctypes.data, counter, nw.ctypes.data, out.ctypes.data)
    assert out.astype("<u4").tobytes() == want


def test_uniform_mod_is_floor_of_scaled_128_bit_word(orc):
    rng = np.random.default_rng(5)
    for q in (2 ** 14, (1 << 54) - 33, 3, (1 << 62) + 1):
        for _ in range(50):
            w = rng.integers(0, 2 ** 32, 4, dtype=np.uint64).astype(np.uint32)
            x = sum(int(w[i]) << (32 * i) for i in range(4))
            assert orc.orc_uniform_mod(w.ctypes.data, q) == (x * q) >> 128
    w = np.full(4, 0xFFFFFFFF, np.uint32)
    assert orc.orc_uniform_mod(w.ctypes.data, 12289) == 12288


@pytest.mark.parametrize("sigma", [0.5, 3.19, 0.0])
def test_cdt_table_library_equals_oracle(pkg, lib, orc, sigma):
    want = _orc_cdt(orc, sigma)
    n = ctypes.c_uint32(0)
    assert lib.cbs_cdt_table_host(sigma, None, 0, ctypes.byref(n)) == 0
    got = np.zeros(max(1, n.value), np.uint64)
    assert lib.cbs_cdt_table_host(sigma, got.ctypes.data, got.size, ctypes.byref(n)) == 0
    assert np.array_equal(got[:n.value], want)
    if sigma > 0:
        assert (np.diff(want.astype(object)) > 0).all() and int(want[-1]) < 2 ** 63


@pytest.mark.parametrize("sigma", [0.5, 3.19])
def test_cdt_sampler_moments(orc, sigma):
    T = _orc_cdt(orc, sigma)
    rng = np.random.default_rng(9)
    u = rng.integers(0, 2 ** 63, 40000, dtype=np.uint64) * 2 + rng.integers(0, 2, 40000, dtype=np.uint64)
    x = np.array([orc.orc_cdt_sample(int(v), T.ctypes.data, T.size) for v in u], np.float64)
    xs = np.arange(-60, 61, dtype=np.float64)
    rho = np.exp(-xs ** 2 / (2 * sigma ** 2))
    var = float((xs ** 2 * rho).sum() / rho.sum())
    assert abs(x.mean()) < 4 * np.sqrt(var / x.size)
    assert abs(x.var() / var - 1) < 0.05


# ------------------------------------------------------------------ GPU


@pytest.fixture(scope="module")
def dev_ctx(pkg):
    pytest.importorskip("torch")
    c = pkg.Context(max_batch=256)
    c.keygen(23)
    yield c
    c.close()


@pytest.mark.gpu
def test_device_material_equals_oracle(pkg, orc, dev_ctx):
    p = dev_ctx.params
    N, n, Q = p.N, p.n, p.Q
    key = bytes(range(16))
    pkg.call("cbs_aes128_setup_device", dev_ctx.handle, key, RNG_KEY)
    tables = np.zeros((8, 256, 2, N), np.uint64)
    rkw = np.zeros((11, 4, 2, N), np.uint64)
    rk0a = np.zeros((128, n), np.uint64)
    rk0b = np.zeros(128, np.uint64)
    pkg.call("cbs_aes128_export_material", dev_ctx.handle, tables.ctypes.data, rkw.ctypes.data, rk0a.ctypes.data,
             rk0b.ctypes.data)
    keys = dev_ctx.export_keys()
    rp = oracle_tables(orc, N, Q)[0]
    s = (np.asarray(keys["s_rlwe"]).reshape(-1).astype(np.int64) % Q).astype(np.uint64)
    s_ntt = s.copy()
    orc.orc_ntt_forward(s_ntt, 1, N, Q, rp)
    kw = _key_words(RNG_KEY)
    Tr, Tl = _orc_cdt(orc, p.sigma_rlwe), _orc_cdt(orc, p.sigma_lwe)
    te = np.zeros((8, 256), np.uint32)
    orc.orc_aes_enc_tables(te)
    # tables: a sample from each table, first and last entries
    for tb, x in [(0, 0), (0, 255), (3, 17), (7, 255)]:
        r = tb * 256 + x
        want = np.zeros(2 * N, np.uint64)
        w = np.array([te[tb, x]], np.uint32)
        orc.orc_encrypt_words_rlwe(kw.ctypes.data, w.ctypes.data, 1, r, N, Q, rp.ctypes.data, s_ntt.ctypes.data,
                                   Tr.ctypes.data, Tr.size, want.ctypes.data)
        assert np.array_equal(tables[tb, x].reshape(-1), want), (tb, x)
    # round-key words: samples 2048 + r*4 + col
    rks = np.zeros((11, 16), np.uint8)
    orc.orc_aes128_key_expand(key, rks.ctypes.data_as(ctypes.c_char_p))
    for r, col in [(0, 0), (5, 2), (10, 3)]:
        b = rks[r, col * 4:col * 4 + 4]
        w = np.array([(int(b[0]) << 24) | (int(b[1]) << 16) | (int(b[2]) << 8) | int(b[3])], np.uint32)
        want = np.zeros(2 * N, np.uint64)
        orc.orc_encrypt_words_rlwe(kw.ctypes.data, w.ctypes.data, 1, 2048 + r * 4 + col, N, Q, rp.ctypes.data,
                                   s_ntt.ctypes.data, Tr.ctypes.data, Tr.size, want.ctypes.data)
        assert np.array_equal(rkw[r, col].reshape(-1), want), (r, col)
    # round-0 key bits: all 128 LWE samples
    bits = np.array([(rks[0, t // 8] >> (t % 8)) & 1 for t in range(128)], np.uint8)
    sl = np.asarray(keys["s_lwe"]).reshape(-1).astype(np.int32)
    wa = np.zeros((128, n), np.uint64)
    wb = np.zeros(128, np.uint64)
    orc.orc_encrypt_bits_lwe(kw.ctypes.data, bits.ctypes.data, 128, n, p.q_lwe, sl.ctypes.data, Tl.ctypes.data,
                             Tl.size, wa.ctypes.data, wb.ctypes.data)
    assert np.array_equal(rk0a, wa) and np.array_equal(rk0b, wb)


@pytest.mark.gpu
def test_device_material_transciphers(pkg, dev_ctx):
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    p = dev_ctx.params
    key = bytes(range(16, 32))
    pkg.call("cbs_aes128_setup_device", dev_ctx.handle, key, RNG_KEY[::-1])
    ctrs = np.frombuffer(bytes(range(32)), np.uint8).copy()
    oa = np.zeros((256, p.n), np.uint64)
    ob = np.zeros(256, np.uint64)
    pkg.call("cbs_aes128_ctr_transcipher", dev_ctx.handle, ctrs.ctypes.data, 2, oa.ctypes.data, ob.ctypes.data)
    dec = np.zeros(256, np.uint8)
    pkg.call("cbs_lwe_decrypt_bits", dev_ctx.handle, oa.ctypes.data, ob.ctypes.data, 256, p.n, dec.ctypes.data)
    got = np.packbits(dec.reshape(2, 128), axis=1, bitorder="little").tobytes()
    enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    assert got == enc.update(ctrs.tobytes())
