"""The LMKCDEY blind rotation on the GPU (k_lmkcdey, the reference's method = LMKCDEY:
bitwise/src/cirbts/cirbts-lmkcdey.cu:105-407) against the oracle's restatement, word for word:
the whole bootstrapping rotation (finalized, MV layout), the EvalAcc primitive on random
accumulators for several automorphism-key counts, and circuit bootstrapping end to end
(LMKCDEY rotation, then HomTrace + SchemeSwitch) with the rows' decryption semantics.  The
oracle's EvalAcc is pinned to the reference's own LMKCDEY kernels in
tests/test_ref_cirbts_gpu.py.  Parameters: the 2^18 x 2 preset (g (digits + 1) = 54 covers
Q) with a one-slot test vector (num_lut = 1; LMKCDEY's odd masks cannot respect the
multi-value rotation quantum)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_encrypt_bits, oracle_lmkcdey_keys

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
NUM_AUTO = 10
SEED = 53


def _dev(a: np.ndarray):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32)).cuda()
    raise TypeError(a.dtype)


def _host(t, shape):
    return t.cpu().numpy().view(np.uint64).reshape(shape)


def _params(pkg):
    p = pkg.preset_params("2x18")
    p.num_lut = 1
    return p


@pytest.fixture(scope="module")
def lctx(pkg):
    c = pkg.Context(params=_params(pkg), max_batch=64)
    c.keygen(SEED)
    c.set_br_method(pkg.BR_LMKCDEY, NUM_AUTO)
    yield c
    c.close()


@pytest.fixture(scope="module")
def lkeys(lctx):
    return lctx.export_keys()


@pytest.fixture(scope="module")
def loc(oracle, lctx, lkeys):
    return OracleCbs(oracle, lctx.params, lkeys)


@pytest.fixture(scope="module")
def lmk(oracle, lctx, lkeys):
    return oracle_lmkcdey_keys(oracle, lctx.params, lkeys, NUM_AUTO, SEED)


def test_lmkcdey_keys_match_oracle(lctx, lmk):
    ev, au = lctx.export_lmkcdey_keys()
    assert np.array_equal(ev, lmk["eval"]) and np.array_equal(au, lmk["auto"])


def test_lmkcdey_blind_rotation_matches_oracle(pkg, lctx, lkeys, loc, lmk):
    p = lctx.params
    bits = [1, 0, 1]
    a, b = lwe_encrypt_bits(np.random.default_rng(4), lkeys["s_lwe"], bits, p.q_lwe)
    mv = torch.zeros((len(bits), p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    da, db = _dev(a), _dev(b)
    pkg.call("cbs_blind_rotate_batch_device", lctx.handle, da.data_ptr(), db.data_ptr(), len(bits), p.n, mv.data_ptr(),
             None)
    torch.cuda.synchronize()
    want = loc.br_acc_lmkcdey(a, b, lmk)
    assert np.array_equal(_host(mv, (len(bits), 2, p.N)), want)


@pytest.mark.parametrize("num_auto,window", [(1, 0), (NUM_AUTO, 0), (200, 0), (NUM_AUTO, 32), (NUM_AUTO, 5)])
def test_lmkcdey_eval_acc_matches_oracle(pkg, oracle, lctx, lkeys, num_auto, window):
    """EvalAcc on random NTT-domain accumulators and random masks: every automorphism-key count
    changes where the walk places its automorphisms (1: one per step; 200: only at buckets), and
    the windowed key sets close long runs with two automorphisms (5^(q w), then 5^r)."""
    p = lctx.params
    N, Q, n = p.N, p.Q, p.n
    changed = (num_auto, window) != (NUM_AUTO, 0)
    if changed:
        lctx.set_br_method(pkg.BR_LMKCDEY, num_auto, window)
    try:
        keys = oracle_lmkcdey_keys(oracle, p, lkeys, num_auto, SEED, window)
        rng = np.random.default_rng(num_auto)
        batch, stride = 2, n + 3
        acc = rng.integers(0, Q, size=(batch, 2, N), dtype=np.uint64)
        a_neg = rng.integers(0, 2 * N, size=(batch, stride), dtype=np.uint32)
        a_neg[0, :64] = a_neg[0, 0]  # a crowded bucket: 64 coefficients of one logarithm
        d_acc, d_a = _dev(acc), _dev(a_neg)
        pkg.call("cbs_lmkcdey_eval_acc_batch_device", lctx.handle, d_a.data_ptr(), stride, d_acc.data_ptr(), batch,
                 None)
        torch.cuda.synchronize()
        got = _host(d_acc, (batch, 2, N))
        vp, u32 = ctypes.c_void_p, ctypes.c_uint32
        oracle.orc_lmkcdey_eval_acc.argtypes = [vp, vp, vp, vp, u32, u32, vp, u32, vp]
        op = OracleCbs(oracle, p, lkeys).op
        for i in range(batch):
            want = np.ascontiguousarray(acc[i])
            row = np.ascontiguousarray(a_neg[i, :n])
            oracle.orc_lmkcdey_eval_acc(ctypes.byref(op), keys["eval"].ctypes.data, keys["auto"].ctypes.data,
                                        keys["maps"].ctypes.data, num_auto, window, row.ctypes.data, n,
                                        want.ctypes.data)
            assert np.array_equal(got[i], want), i
    finally:
        if changed:
            lctx.set_br_method(pkg.BR_LMKCDEY, NUM_AUTO)


def test_lmkcdey_circuit_bootstrap_rows(pkg, lctx, lkeys, loc, lmk):
    """CBS with the LMKCDEY rotation: the RGSW rows equal the oracle's HomTrace + SchemeSwitch of
    the oracle's LMKCDEY accumulator, and decrypt to m g_0 (row 1) and -m g_0 s (row 0)."""
    p = lctx.params
    bits = [0, 1, 1, 0]
    a, b = lwe_encrypt_bits(np.random.default_rng(9), lkeys["s_lwe"], bits, p.q_lwe)
    view = ctypes.c_void_p()
    da, db = _dev(a), _dev(b)
    pkg.call("cbs_circuit_bootstrap_batch_device", lctx.handle, da.data_ptr(), db.data_ptr(), len(bits), p.n,
             ctypes.byref(view), None)
    torch.cuda.synchronize()
    per = p.num_lut * 4 * p.N
    got = np.zeros(len(bits) * per, np.uint64)
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    assert cudart.cudaMemcpy(got.ctypes.data, view.value, got.nbytes, 2) == 0  # device to host
    got = got.reshape(len(bits), p.num_lut, 2, 2, p.N)
    want = loc.trace_ss(loc.br_acc_lmkcdey(a, b, lmk)).reshape(len(bits), p.num_lut, 2, 2, p.N)
    assert np.array_equal(got, want)
    g0 = int(lkeys["gpow"][0])
    s = lkeys["s_rlwe"].astype(object)
    for i, m in enumerate(bits):
        ph1 = loc.phase_coef(got[i, 0, 1])
        ph1[0] -= m * g0
        ph0 = loc.phase_coef(got[i, 0, 0]) + m * g0 * s
        assert max(abs(int(x)) for x in ph1) < g0 // 2
        assert max(abs(int(x)) for x in ph0) < g0 * 2


def test_lmkcdey_import_on_a_server_without_secrets(pkg, lctx, lkeys):
    """A context holding evaluation keys only takes the LMKCDEY keys by import and rotates as the
    key owner does."""
    p = lctx.params
    ev, au = lctx.export_lmkcdey_keys()
    srv = pkg.Context(params=p, max_batch=4)
    try:
        pkg.call("cbs_import_keys", srv.handle, None, None, *(np.ascontiguousarray(lkeys[k]).ctypes.data
                                                               for k in ("bsk", "ht", "ss", "ksk")))
        assert pkg.load().cbs_context_set_br_method(srv.handle, pkg.BR_LMKCDEY, NUM_AUTO, 0) == 7  # no secret
        srv.import_lmkcdey_keys(NUM_AUTO, ev, au)
        a, b = lwe_encrypt_bits(np.random.default_rng(2), lkeys["s_lwe"], [1, 1], p.q_lwe)
        outs = []
        for c in (lctx, srv):
            mv = torch.zeros((2, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
            da, db = _dev(a), _dev(b)
            pkg.call("cbs_blind_rotate_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 2, p.n, mv.data_ptr(),
                     None)
            torch.cuda.synchronize()
            outs.append(_host(mv, (2, 2, p.N)))
        assert np.array_equal(outs[0], outs[1])
    finally:
        srv.close()


def test_lmkcdey_preconditions(pkg):
    lib = pkg.load()
    c = pkg.Context(params=pkg.preset_params("2x18"), max_batch=4)  # num_lut = 4
    try:
        assert lib.cbs_context_set_br_method(c.handle, pkg.BR_LMKCDEY, NUM_AUTO, 0) == 6
        assert b"num_lut" in lib.cbs_last_error()
    finally:
        c.close()
    p = pkg.default_params()  # 2^12 x 3: the approximate digits do not cover Q
    p.num_lut = 1
    c = pkg.Context(params=p, max_batch=4)
    try:
        assert lib.cbs_context_set_br_method(c.handle, pkg.BR_LMKCDEY, NUM_AUTO, 0) == 6
        assert b"log2 Q" in lib.cbs_last_error()
    finally:
        c.close()
    c = pkg.Context(params=_params(pkg), max_batch=4)
    try:
        assert lib.cbs_context_set_br_method(c.handle, pkg.BR_LMKCDEY, 0, 0) == 1
        assert lib.cbs_context_set_br_method(c.handle, 7, NUM_AUTO, 0) == 1
        assert lib.cbs_context_set_br_method(c.handle, pkg.BR_LMKCDEY, NUM_AUTO, c.params.N // 2) == 1
        c.set_br_backend(pkg.BR_FFT64)
        assert lib.cbs_context_set_br_method(c.handle, pkg.BR_LMKCDEY, NUM_AUTO, 0) == 6
        c.set_br_backend(pkg.BR_NTT)
        c.set_br_method(pkg.BR_LMKCDEY, NUM_AUTO)  # keys follow at keygen
        c.keygen(3)
        ev, au = c.export_lmkcdey_keys()
        assert ev.shape[0] == c.params.n and au.shape[0] == NUM_AUTO + 1
        c.set_br_backend(pkg.BR_FFT64)  # resets the method
        st = lib.cbs_export_lmkcdey_keys(c.handle, None, None, ctypes.byref(ctypes.c_size_t()),
                                         ctypes.byref(ctypes.c_size_t()))
        assert st == 7
    finally:
        c.close()
