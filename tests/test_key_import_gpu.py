"""Key import (cbs_import_keys, cbs_import_mb_bsk, cbs_aes128_import_material): a context
loaded with another context's evaluation keys, without the secrets, computes bit-identical
blind rotations (exact NTT and FFT, one-bit and grouped) and transciphers AES-128 to the
same ciphertexts as the key owner; what needs a secret refuses; malformed keys are
rejected."""
from __future__ import annotations

import numpy as np
import pytest

from cbs_harness import lwe_decrypt_bits, lwe_encrypt_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


@pytest.fixture(scope="module")
def owner(pkg):
    a = pkg.Context(max_batch=256)
    a.keygen(21)
    yield a
    a.close()


@pytest.fixture(scope="module")
def okeys(owner):
    return owner.export_keys()


@pytest.fixture(scope="module")
def server(pkg, okeys):
    b = pkg.Context(max_batch=256)
    b.import_keys(okeys, with_secrets=False)
    yield b
    b.close()


def _br(pkg, ctx, a, b):
    p = ctx.params
    mv = torch.zeros((len(b), p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    da, db = _dev(a), _dev(b)
    pkg.call("cbs_blind_rotate_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), len(b), p.n, mv.data_ptr(),
             None)
    torch.cuda.synchronize()
    return mv.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("backend", ["ntt", "fft64"])
def test_imported_keys_blind_rotate_identically(pkg, owner, server, okeys, backend):
    be = pkg.BR_NTT if backend == "ntt" else pkg.BR_FFT64
    a, b = lwe_encrypt_bits(np.random.default_rng(3), okeys["s_lwe"], [1, 0, 1], owner.params.q_lwe)
    try:
        owner.set_br_backend(be)
        server.set_br_backend(be)
        assert np.array_equal(_br(pkg, owner, a, b), _br(pkg, server, a, b))
    finally:
        owner.set_br_backend(pkg.BR_NTT)
        server.set_br_backend(pkg.BR_NTT)


def test_secret_operations_refuse_without_secrets(pkg, server):
    server.set_br_backend(pkg.BR_FFT64)
    try:
        with pytest.raises(pkg.CbsError, match="secret"):
            server.set_br_multibit(2)
    finally:
        server.set_br_backend(pkg.BR_NTT)
    with pytest.raises(pkg.CbsError, match="secret"):
        pkg.call("cbs_aes128_setup", server.handle, bytes(16), 1)
    x = np.zeros(server.params.n, np.uint64)
    out = np.zeros(1, np.uint8)
    with pytest.raises(pkg.CbsError, match="secret"):
        pkg.call("cbs_lwe_decrypt_bits", server.handle, x.ctypes.data, x.ctypes.data, 1, server.params.n,
                 out.ctypes.data)


def test_imported_grouped_keys_blind_rotate_identically(pkg, owner, server, okeys):
    a, b = lwe_encrypt_bits(np.random.default_rng(4), okeys["s_lwe"], [0, 1], owner.params.q_lwe)
    try:
        owner.set_br_backend(pkg.BR_FFT64)
        owner.set_br_multibit(2)
        server.set_br_backend(pkg.BR_FFT64)
        server.import_mb_bsk(2, owner.export_mb_bsk())
        assert np.array_equal(server.export_mb_bsk(), owner.export_mb_bsk())
        assert np.array_equal(_br(pkg, owner, a, b), _br(pkg, server, a, b))
    finally:
        owner.set_br_backend(pkg.BR_NTT)
        server.set_br_backend(pkg.BR_NTT)


def test_imported_aes_material_transciphers_identically(pkg, owner, server, okeys):
    """Owner: keys + AES material (the AES key stays here).  Server: evaluation keys, grouped
    keys and the encrypted material only.  Both transcipher two counter blocks on the FFT
    path with the grouped rotation; the outputs are identical and decrypt to AES_K(ctr)."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    p = owner.params
    key = bytes(range(100, 116))
    try:
        for c in (owner, server):
            c.set_br_backend(pkg.BR_FFT64)
        owner.set_br_multibit(2)
        server.import_mb_bsk(2, owner.export_mb_bsk())
        pkg.call("cbs_aes128_setup", owner.handle, key, 5)
        server.aes_import_material(owner.aes_export_material())
        ctrs = [bytes([7] * 15 + [i]) for i in range(2)]
        h = np.frombuffer(b"".join(ctrs), np.uint8).copy()
        outs = []
        for c in (owner, server):
            oa = np.zeros((256, p.n), np.uint64)
            ob = np.zeros(256, np.uint64)
            pkg.call("cbs_aes128_ctr_transcipher", c.handle, h.ctypes.data, 2, oa.ctypes.data, ob.ctypes.data)
            outs.append((oa, ob))
    finally:
        owner.set_br_backend(pkg.BR_NTT)
        server.set_br_backend(pkg.BR_NTT)
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    got, _ = lwe_decrypt_bits(okeys["s_lwe"], outs[1][0], outs[1][1], p.q_lwe)
    enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    for blk, ctr in enumerate(ctrs):
        want = enc.update(ctr)
        out = bytes(int(sum(int(got[blk * 128 + i * 8 + b]) << b for b in range(8))) for i in range(16))
        assert out == want, blk


def test_import_with_secrets_equals_keygen(pkg, okeys):
    c = pkg.Context(max_batch=4)
    try:
        c.import_keys(okeys, with_secrets=True)
        again = c.export_keys()
        for k in pkg.KEY_FIELDS:
            assert np.array_equal(again[k], okeys[k]), k
    finally:
        c.close()


def test_import_rejects_malformed_keys(pkg, owner, okeys):
    c = pkg.Context(max_batch=4)
    try:
        bad = {k: v.copy() for k, v in okeys.items()}
        bad["bsk"].reshape(-1)[17] = owner.params.Q  # not a residue
        with pytest.raises(pkg.CbsError, match="residues mod Q"):
            c.import_keys(bad, with_secrets=False)
        bad = {k: v.copy() for k, v in okeys.items()}
        bad["ksk"].reshape(-1)[3] = owner.params.qks
        with pytest.raises(pkg.CbsError, match="qks"):
            c.import_keys(bad, with_secrets=False)
        bad = {k: v.copy() for k, v in okeys.items()}
        bad["s_rlwe"].reshape(-1)[0] = 2
        with pytest.raises(pkg.CbsError, match="ternary"):
            c.import_keys(bad, with_secrets=True)
        x = okeys["bsk"]
        with pytest.raises(pkg.CbsError, match="both secrets"):
            pkg.call("cbs_import_keys", c.handle, okeys["s_lwe"].ctypes.data, None, x.ctypes.data, x.ctypes.data,
                     x.ctypes.data, okeys["ksk"].ctypes.data)
        c.import_keys(okeys, with_secrets=False)
        c.set_br_backend(pkg.BR_FFT64)
        with pytest.raises(pkg.CbsError):
            c.import_mb_bsk(2, np.zeros(10, np.uint64))  # wrong size
    finally:
        c.close()
