"""GPU parity of the circuit-bootstrapping path through the C ABI against the CPU oracle:
blind rotation + multi-value split, HomTrace + SchemeSwitch, the full CBS view, the CMux
LUT, sample extract + key switch (all bit-exact), plus the decryption semantics of the RGSW
rows and end-to-end AES-128 CTR transciphering checked against plaintext AES."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_decrypt_bits, lwe_encrypt_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a: np.ndarray):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32)).cuda()
    if a.dtype == np.uint8:
        return torch.from_numpy(a).cuda()
    raise TypeError(a.dtype)


def host(t, shape=None) -> np.ndarray:
    x = t.cpu().numpy().view(np.uint64)
    return x.reshape(shape) if shape is not None else x


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(max_batch=256)
    c.keygen(11)
    yield c
    c.close()


@pytest.fixture(scope="module")
def keys(ctx):
    return ctx.export_keys()


@pytest.fixture(scope="module")
def oc(oracle, ctx, keys):
    return OracleCbs(oracle, ctx.params, keys)


def test_keygen_matches_host_keygen(pkg, ctx, keys):
    hk = pkg.generate_keys_host(ctx.params, 11)
    for k in pkg.KEY_FIELDS:
        assert np.array_equal(hk[k], keys[k]), k


def _lwe(ctx, keys, bits, seed):
    rng = np.random.default_rng(seed)
    return lwe_encrypt_bits(rng, keys["s_lwe"], bits, ctx.params.q_lwe)


@pytest.mark.parametrize("batch", [1, 3])
def test_blind_rotate_mv_bit_exact(pkg, ctx, keys, oc, batch):
    p = ctx.params
    a, b = _lwe(ctx, keys, [i & 1 for i in range(batch)], 100 + batch)
    da, db = dev(a), dev(b)
    mv = torch.zeros((batch, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    pkg.call("cbs_blind_rotate_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), batch, p.n, mv.data_ptr(),
             None)
    torch.cuda.synchronize()
    want = oc.br_mv(a, b)
    assert np.array_equal(host(mv, want.shape), want)


def test_blind_rotate_strided_input(pkg, ctx, keys, oc):
    """a_stride > n (the reference's a_stride argument) reads only the first n entries."""
    p = ctx.params
    a, b = _lwe(ctx, keys, [1, 0], 5)
    wide = np.zeros((2, p.n + 37), np.uint64)
    wide[:, :p.n] = a
    wide[:, p.n:] = 12345  # junk that must be ignored
    mv = torch.zeros((2, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    dw, db = dev(wide), dev(b)
    pkg.call("cbs_blind_rotate_batch_device", ctx.handle, dw.data_ptr(), db.data_ptr(), 2, p.n + 37,
             mv.data_ptr(), None)
    torch.cuda.synchronize()
    assert np.array_equal(host(mv, (2, p.num_lut, 2, p.N)), oc.br_mv(a, b))


def test_trace_schemeswitch_bit_exact(pkg, ctx, keys, oc):
    p = ctx.params
    rng = np.random.default_rng(3)
    count = 5
    mv = rng.integers(0, p.Q, size=(count, 2, p.N), dtype=np.uint64)
    out = torch.zeros((count, 2, 2, p.N), dtype=torch.int64, device="cuda")
    dmv = dev(mv)
    pkg.call("cbs_trace_schemeswitch_device", ctx.handle, dmv.data_ptr(), count, out.data_ptr(), None)
    torch.cuda.synchronize()
    want = oc.trace_ss(mv)
    assert np.array_equal(host(out, want.shape), want)


def test_circuit_bootstrap_view_and_semantics(pkg, ctx, keys, oc):
    p = ctx.params
    bits = [0, 1, 1, 0, 1]
    a, b = _lwe(ctx, keys, bits, 21)
    view = ctypes.c_void_p()
    da, db = dev(a), dev(b)
    pkg.call("cbs_circuit_bootstrap_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), len(bits), p.n,
             ctypes.byref(view), None)
    torch.cuda.synchronize()
    per = p.num_lut * 4 * p.N
    tmp = torch.empty(len(bits) * per, dtype=torch.int64, device="cuda")
    _copy_d2d(tmp.data_ptr(), view.value, len(bits) * per * 8)
    got = host(tmp).reshape(len(bits), p.num_lut, 2, 2, p.N)
    want = oc.trace_ss(oc.br_mv(a, b)).reshape(len(bits), p.num_lut, 2, 2, p.N)
    assert np.array_equal(got, want)
    # decryption semantics: row 2j+1 -> m*g_j, row 2j -> -m*g_j*s (up to the CBS noise)
    g = [int(x) for x in keys["gpow"]]
    s = keys["s_rlwe"].astype(object)
    for i, m in enumerate(bits):
        for j in range(p.num_lut):
            ph1 = oc.phase_coef(got[i, j, 1])
            ph1[0] -= m * g[j]
            ph0 = oc.phase_coef(got[i, j, 0]) + m * g[j] * s
            assert max(abs(int(x)) for x in ph1) < g[0] // 2
            assert max(abs(int(x)) for x in ph0) < g[0] * 2


_CUDART = None


def _copy_d2d(dst: int, src: int, nbytes: int) -> None:
    """cudaMemcpy device-to-device (copies a context-owned view into a test buffer)."""
    global _CUDART
    if _CUDART is None:
        _CUDART = ctypes.CDLL("libcudart.so.12")
        _CUDART.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    torch.cuda.synchronize()
    assert _CUDART.cudaMemcpy(dst, src, nbytes, 3) == 0  # cudaMemcpyDeviceToDevice


def test_cbs_rejects_oversized_batch(pkg, ctx):
    p = ctx.params
    view = ctypes.c_void_p()
    x = torch.zeros(8, dtype=torch.int64, device="cuda")
    st = pkg.load().cbs_circuit_bootstrap_batch_device(ctx.handle, x.data_ptr(), x.data_ptr(), ctx.max_batch + 1, p.n,
                                                       ctypes.byref(view), None)
    assert st == 2  # CBS_ERR_SHAPE_MISMATCH
    assert b"max_batch" in pkg.load().cbs_last_error()


@pytest.fixture(scope="module")
def aes_ctx(pkg, ctx):
    key = bytes(range(16))
    pkg.call("cbs_aes128_setup", ctx.handle, key, 99)
    p = ctx.params
    tables = np.zeros((8, 256, 2, p.N), np.uint64)
    rkw = np.zeros((11, 4, 2, p.N), np.uint64)
    pkg.call("cbs_aes128_export_material", ctx.handle, tables.ctypes.data, rkw.ctypes.data, None, None)
    return key, tables, rkw


def test_lut8x32_bit_exact_and_decrypts(pkg, ctx, keys, oc, aes_ctx):
    p = ctx.params
    _, tables, _ = aes_ctx
    # CBS of 16 random bits -> controls of two LUTs (bits 0..7 and 8..15)
    rng = np.random.default_rng(8)
    bits = rng.integers(0, 2, size=16)
    a, b = _lwe(ctx, keys, bits, 31)
    view = ctypes.c_void_p()
    da, db = dev(a), dev(b)
    pkg.call("cbs_circuit_bootstrap_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), 16, p.n,
             ctypes.byref(view), None)
    per = p.num_lut * 4 * p.N
    rg = torch.empty(16 * per, dtype=torch.int64, device="cuda")
    _copy_d2d(rg.data_ptr(), view.value, 16 * per * 8)
    torch.cuda.synchronize()
    d_tables = dev(tables)
    sel = np.array([0, 5], np.uint32)
    ctrl = np.array([list(range(8)), list(range(8, 16))], np.uint32)
    out = torch.zeros((2, 2, p.N), dtype=torch.int64, device="cuda")
    pkg.call("cbs_lut8x32_batch_device", ctx.handle, d_tables.data_ptr(), 8, sel.ctypes.data, rg.data_ptr(), 16, per,
             ctrl.ctypes.data, 2, out.data_ptr(), None)
    bad = ctrl.copy()
    bad[1, 3] = 16
    assert pkg.load().cbs_lut8x32_batch_device(ctx.handle, d_tables.data_ptr(), 8, sel.ctypes.data, rg.data_ptr(), 16,
                                               per, bad.ctypes.data, 2, out.data_ptr(), None) == 1
    torch.cuda.synchronize()
    got = host(out, (2, 2, p.N))
    rgh = host(rg, (16, per))
    te = np.zeros(8 * 256, np.uint32)
    oc.o.orc_aes_enc_tables(te)
    te = te.reshape(8, 256)
    for u in range(2):
        ctrls = [np.ascontiguousarray(rgh[8 * u + k]) for k in range(8)]
        want = oc.lut(np.ascontiguousarray(tables[sel[u]]), ctrls)
        assert np.array_equal(got[u], want)
        x = int(sum(int(bits[8 * u + k]) << k for k in range(8)))
        ph = oc.phase_coef(got[u])
        dec = 0
        for bt in range(32):
            v = int(ph[bt]) % p.Q
            dec |= (((2 * v + p.Q // 2) // p.Q) & 1) << bt
        assert dec == int(te[sel[u], x])


def test_extract_keyswitch_bit_exact(pkg, ctx, keys, oc):
    p = ctx.params
    rng = np.random.default_rng(4)
    W = 3
    words = rng.integers(0, p.Q, size=(W, 2, p.N), dtype=np.uint64)
    info = np.array([(w << 16) | c for w, c in [(0, 0), (1, 5), (2, 2047), (0, 31), (2, 1000), (1, 0), (0, 1)]],
                    np.uint32)
    T = len(info)
    oa = torch.zeros((T, p.n), dtype=torch.int64, device="cuda")
    ob = torch.zeros(T, dtype=torch.int64, device="cuda")
    dw = dev(words)
    pkg.call("cbs_extract_keyswitch_device", ctx.handle, dw.data_ptr(), W, info.ctypes.data, T, oa.data_ptr(),
             ob.data_ptr(), p.n, None)
    torch.cuda.synchronize()
    wa, wb = oc.extract(words, info)
    assert np.array_equal(host(oa, (T, p.n)), wa)
    assert np.array_equal(host(ob), wb)


def test_extract_rejects_bad_info(pkg, ctx):
    p = ctx.params
    info = np.array([(5 << 16) | 3], np.uint32)
    x = torch.zeros(16, dtype=torch.int64, device="cuda")
    st = pkg.load().cbs_extract_keyswitch_device(ctx.handle, x.data_ptr(), 2, info.ctypes.data, 1, x.data_ptr(),
                                                 x.data_ptr(), p.n, None)
    assert st == 1


def _aes_ecb(key: bytes, blocks: list[bytes]) -> list[bytes]:
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    return [enc.update(b) for b in blocks]


@pytest.mark.parametrize("blocks,graphs", [(1, 0), (3, 1)])
def test_aes128_ctr_transcipher_device(pkg, ctx, keys, aes_ctx, blocks, graphs):
    p = ctx.params
    key, _, _ = aes_ctx
    rng = np.random.default_rng(blocks)
    ctrs = [rng.bytes(16) for _ in range(blocks)]
    bits = np.array([[(c[t // 8] >> (t % 8)) & 1 for t in range(128)] for c in ctrs], np.uint8).reshape(-1)
    oa = torch.zeros((blocks * 128, p.n), dtype=torch.int64, device="cuda")
    ob = torch.zeros(blocks * 128, dtype=torch.int64, device="cuda")
    dbits = dev(bits)
    stream = torch.cuda.Stream()
    for rep in range(2 if graphs else 1):  # the second call replays the captured graphs
        oa.zero_()
        ob.zero_()
        torch.cuda.synchronize()
        pkg.call("cbs_aes128_ctr_transcipher_device", ctx.handle, dbits.data_ptr(), blocks, oa.data_ptr(),
                 ob.data_ptr(), graphs, stream.cuda_stream)
        stream.synchronize()
        torch.cuda.synchronize()
        got_bits, err = lwe_decrypt_bits(keys["s_lwe"], host(oa, (blocks * 128, p.n)), host(ob), p.q_lwe)
        want = _aes_ecb(key, ctrs)
        for blk in range(blocks):
            out = bytes(int(sum(int(got_bits[blk * 128 + i * 8 + b]) << b for b in range(8))) for i in range(16))
            assert out == want[blk], f"block {blk} rep {rep}"
        assert max(err) < p.q_lwe // 8, max(err)


def test_aes128_ctr_transcipher_host_api(pkg, ctx, keys, aes_ctx):
    p = ctx.params
    key, _, _ = aes_ctx
    ctrs = [bytes([0] * 15 + [i]) for i in range(2)]
    h = np.frombuffer(b"".join(ctrs), np.uint8).copy()
    oa = np.zeros((2 * 128, p.n), np.uint64)
    ob = np.zeros(2 * 128, np.uint64)
    pkg.call("cbs_aes128_ctr_transcipher", ctx.handle, h.ctypes.data, 2, oa.ctypes.data, ob.ctypes.data)
    dec = np.zeros(256, np.uint8)
    pkg.call("cbs_lwe_decrypt_bits", ctx.handle, oa.ctypes.data, ob.ctypes.data, 256, p.n, dec.ctypes.data)
    want = _aes_ecb(key, ctrs)
    for blk in range(2):
        out = bytes(int(sum(int(dec[blk * 128 + i * 8 + b]) << b for b in range(8))) for i in range(16))
        assert out == want[blk]


@pytest.mark.parametrize("blocks", [1, 3, 1000])
def test_aes128_ctr_add_ciphertext_device_bit_exact(pkg, ctx, blocks):
    """b[t] + q/2 mod q exactly where bit t of the public ciphertext is set (main.cu:1569-1582),
    nothing else touched; 1000 blocks leave a partial last CTA."""
    p = ctx.params
    rng = np.random.default_rng(70 + blocks)
    T = blocks * 128
    b = rng.integers(0, p.q_lwe, T, dtype=np.uint64)
    b[:3] = [0, p.q_lwe // 2, p.q_lwe - 1]  # wrap edges
    cipher = rng.integers(0, 256, blocks * 16, dtype=np.uint8)
    cipher[0] = 0x07
    db, dc = dev(b), dev(cipher)  # both held until the kernel has run
    pkg.call("cbs_aes128_ctr_add_ciphertext_device", ctx.handle, dc.data_ptr(), blocks, db.data_ptr(), None)
    torch.cuda.synchronize()
    bits = np.unpackbits(cipher, bitorder="little").astype(np.uint64)
    want = (b + bits * (p.q_lwe // 2)) % p.q_lwe
    assert np.array_equal(host(db), want)
    assert pkg.load().cbs_aes128_ctr_add_ciphertext_device(ctx.handle, None, 0, None, None) == 0  # empty


def test_aes128_ctr_transcipher_ciphertext_decrypts_to_plaintext(pkg, ctx, keys, aes_ctx):
    """Counters + a public AES-CTR ciphertext in, LWE encryptions of the plaintext bits out:
    the reference's download -> EvalAddConstEq -> Decrypt sequence with the add on the GPU."""
    p = ctx.params
    key, _, _ = aes_ctx
    rng = np.random.default_rng(77)
    blocks = 2
    ctrs = [rng.bytes(16) for _ in range(blocks)]
    plain = [rng.bytes(16) for _ in range(blocks)]
    ks = _aes_ecb(key, ctrs)
    cipher = [bytes(x ^ y for x, y in zip(pt, k)) for pt, k in zip(plain, ks)]
    hc = np.frombuffer(b"".join(ctrs), np.uint8).copy()
    hx = np.frombuffer(b"".join(cipher), np.uint8).copy()
    oa = np.zeros((blocks * 128, p.n), np.uint64)
    ob = np.zeros(blocks * 128, np.uint64)
    pkg.call("cbs_aes128_ctr_transcipher_ciphertext", ctx.handle, hc.ctypes.data, hx.ctypes.data, blocks,
             oa.ctypes.data, ob.ctypes.data)
    dec = np.zeros(blocks * 128, np.uint8)
    pkg.call("cbs_lwe_decrypt_bits", ctx.handle, oa.ctypes.data, ob.ctypes.data, blocks * 128, p.n, dec.ctypes.data)
    for blk in range(blocks):
        out = bytes(int(sum(int(dec[blk * 128 + i * 8 + b]) << b for b in range(8))) for i in range(16))
        assert out == plain[blk]
    # the keystream path on the same counters: same a, b differing by q/2 exactly where the
    # ciphertext bit is set
    ka = np.zeros_like(oa)
    kb = np.zeros_like(ob)
    pkg.call("cbs_aes128_ctr_transcipher", ctx.handle, hc.ctypes.data, blocks, ka.ctypes.data, kb.ctypes.data)
    bits = np.unpackbits(hx, bitorder="little").astype(np.uint64)
    assert np.array_equal((kb + bits * (p.q_lwe // 2)) % p.q_lwe, ob)
