"""Functional bootstrapping on the GPU (csrc/gate_func.cu: the reference's BatchGPUBootstrapFunc,
BatchGPUEvalFunc / Floor / Sign / Decomp, bitwise/src/binfhe-base-scheme-batch.cu:215-712)
against the oracle's restatement (tests/gate_harness.py OracleGateFunc over
orc_gate_bootstrap_func), bit for bit: the programmable bootstrap and every evaluator on
the same keys and ciphertexts (LWE dimension 100, so the exact oracle finishes in seconds), plus
the evaluators' semantics at the default gate parameters (n = 636)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from gate_harness import OracleGateFunc, declare_gate, lut_via_function, lwe_encrypt_mod, phase_mod

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
BETA = 128


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, np.uint32).view(np.int32)).cuda()


def _host(t, shape):
    return t.cpu().numpy().view(np.uint32).reshape(shape)


def _centred(x, bits):
    x = np.asarray(x, np.int64) % (1 << bits)
    return np.where(x >= 1 << (bits - 1), x - (1 << bits), x)


@pytest.fixture(scope="module")
def fctx(pkg, oracle):
    p = pkg.gate_default_params()
    p.n = 100
    c = pkg.GateContext(params=p, max_batch=16)
    c.keygen(29)
    keys = c.export_keys()
    yield c, keys, OracleGateFunc(declare_gate(oracle), p, keys)
    c.close()


def _outs(count, n, digits=1):
    return (torch.zeros(digits * count * n, dtype=torch.int32, device="cuda"),
            torch.zeros(digits * count, dtype=torch.int32, device="cuda"))


def test_bootstrap_func_matches_oracle(pkg, fctx):
    c, keys, fo = fctx
    p = c.params
    rng = np.random.default_rng(1)
    in_bits, f_bits = 11, 20
    lut = rng.integers(0, 1 << f_bits, 1 << (in_bits - 1), dtype=np.uint64)
    a, b = lwe_encrypt_mod(rng, keys["s_lwe"], rng.integers(0, 1 << in_bits, 6), in_bits, sigma_units=1)
    oa, ob = _outs(6, p.n)
    da, db = _dev(a), _dev(b)  # held: a temporary's memory could be reused before the kernels run
    pkg.call("cbs_gate_bootstrap_func_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 6,
             1 << in_bits, lut.ctypes.data, 1 << f_bits, oa.data_ptr(), ob.data_ptr(), None)
    torch.cuda.synchronize()
    wa, wb = fo.bootstrap(a, b, in_bits, lut, f_bits)
    assert np.array_equal(_host(oa, (6, p.n)), wa) and np.array_equal(_host(ob, (6,)), wb)
    # fmod = 2^32: no final rounding
    lut32 = rng.integers(0, 1 << 32, 1 << (in_bits - 1), dtype=np.uint64)
    pkg.call("cbs_gate_bootstrap_func_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 6,
             1 << in_bits, lut32.ctypes.data, 1 << 32, oa.data_ptr(), ob.data_ptr(), None)
    torch.cuda.synchronize()
    wa, wb = fo.bootstrap(a, b, in_bits, lut32, 32)
    assert np.array_equal(_host(oa, (6, p.n)), wa) and np.array_equal(_host(ob, (6,)), wb)


@pytest.mark.parametrize("kind", ["negacyclic", "periodic", "arbitrary"])
def test_eval_func_matches_oracle(pkg, fctx, kind):
    c, keys, fo = fctx
    p = c.params
    P, q = 4, 1024
    f = {"negacyclic": lambda m, p_: [1, 2, 3, 2][m], "periodic": lambda m, p_: m % 2,
         "arbitrary": lambda m, p_: (3 * m) % 4}[kind]
    lut = lut_via_function(f, P, q)
    ms = np.array([0, 1, 2, 3, 3, 0], np.int64)
    a, b = lwe_encrypt_mod(np.random.default_rng(2), keys["s_lwe"], ms * (q // P), 10, sigma_units=3)
    oa, ob = _outs(6, p.n)
    da, db = _dev(a), _dev(b)
    pkg.call("cbs_gate_eval_func_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 6, q,
             lut.ctypes.data, BETA, oa.data_ptr(), ob.data_ptr(), None)
    torch.cuda.synchronize()
    ga, gb = _host(oa, (6, p.n)), _host(ob, (6,))
    wa, wb = fo.eval_func(a, b, q, lut, BETA)
    assert np.array_equal(ga, wa) and np.array_equal(gb, wb)
    dec = ((phase_mod(keys["s_lwe"], ga, gb, 10) + q // (2 * P)) // (q // P)) % P
    assert list(dec) == [f(int(m), P) for m in ms]


def test_eval_floor_sign_decomp_match_oracle(pkg, fctx):
    c, keys, fo = fctx
    p = c.params
    s = keys["s_lwe"]
    mod_bits, q_bits = 14, 10
    x = np.array([300, 4000, 8000, 8500, 12000, 16000], np.int64)
    a, b = lwe_encrypt_mod(np.random.default_rng(3), s, x, mod_bits, sigma_units=2)
    da, db = _dev(a), _dev(b)
    oa, ob = _outs(6, p.n)
    pkg.call("cbs_gate_eval_floor_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 6, 1 << mod_bits,
             1 << q_bits, 0, BETA, oa.data_ptr(), ob.data_ptr(), None)
    torch.cuda.synchronize()
    wa, wb = fo.eval_floor(a, b, mod_bits, q_bits, BETA)
    assert np.array_equal(_host(oa, (6, p.n)), wa) and np.array_equal(_host(ob, (6,)), wb)
    for ss in (0, 1):
        pkg.call("cbs_gate_eval_sign_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 6, 1 << mod_bits,
                 1 << q_bits, BETA, ss, oa.data_ptr(), ob.data_ptr(), None)
        torch.cuda.synchronize()
        wa, wb = fo.eval_sign(a, b, mod_bits, q_bits, BETA, bool(ss))
        assert np.array_equal(_host(oa, (6, p.n)), wa) and np.array_equal(_host(ob, (6,)), wb), ss
    digits = ctypes.c_uint32(4)
    oa, ob = _outs(6, p.n, 4)
    pkg.call("cbs_gate_eval_decomp_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 6, 1 << mod_bits,
             1 << q_bits, BETA, oa.data_ptr(), ob.data_ptr(), ctypes.byref(digits), None)
    torch.cuda.synchronize()
    want = fo.eval_decomp(a, b, mod_bits, q_bits, BETA)
    assert digits.value == len(want) == 3
    ga, gb = _host(oa, (4, 6, p.n)), _host(ob, (4, 6))
    for k, ((wa, wb), _) in enumerate(want):
        assert np.array_equal(ga[k], wa) and np.array_equal(gb[k], wb), k
    # too small an output is refused and reports the digits needed
    small = ctypes.c_uint32(2)
    st = pkg.load().cbs_gate_eval_decomp_batch_device(c.handle, da.data_ptr(), db.data_ptr(), 6, 1 << mod_bits,
                                                      1 << q_bits, BETA, oa.data_ptr(), ob.data_ptr(),
                                                      ctypes.byref(small), None)
    assert st == 1 and small.value == 3


def test_eval_sign_semantics_default_parameters(pkg):
    """EvalSign at the default gate parameters (n = 636, N = 1024): the sign of 64 random
    14-bit values, every one right."""
    c = pkg.GateContext(max_batch=64)
    try:
        c.keygen(31)
        s = c.export_keys()["s_lwe"]
        rng = np.random.default_rng(6)
        mod_bits, q_bits = 14, 10
        x = rng.integers(0, 1 << mod_bits, 64)
        x = np.where(np.abs(x - (1 << (mod_bits - 1))) < 256, x + 512, x) % (1 << mod_bits)  # off the boundary
        x = np.where(x < 256, x + 512, x)
        x = np.where(x > (1 << mod_bits) - 256, x - 512, x)
        a, b = lwe_encrypt_mod(rng, s, x, mod_bits, sigma_units=2)
        oa, ob = _outs(64, c.params.n)
        da, db = _dev(a), _dev(b)

        def run():
            pkg.call("cbs_gate_eval_sign_batch_device", c.handle, da.data_ptr(), db.data_ptr(), 64,
                     1 << mod_bits, 1 << q_bits, BETA, 0, oa.data_ptr(), ob.data_ptr(), None)

        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        print(f"\nEvalSign, 14-bit values, 64 ciphertexts (5 bootstraps each): {e0.elapsed_time(e1):.2f} ms")
        ph = phase_mod(s, _host(oa, (64, c.params.n)), _host(ob, (64,)), q_bits)
        msb = (x >= (1 << (mod_bits - 1))).astype(np.int64)
        err = _centred(ph - msb * (1 << (q_bits - 1)), q_bits)
        print(f"EvalSign, n = 636: max |phase error| {np.abs(err).max()} of q/4 = {1 << (q_bits - 2)}")
        assert np.abs(err).max() < 1 << (q_bits - 3)
    finally:
        c.close()


def test_functional_bootstrap_preconditions(pkg, fctx):
    c, keys, fo = fctx
    lib = pkg.load()
    x = torch.zeros(64, dtype=torch.int32, device="cuda")
    lut = np.zeros(2048, np.uint64)
    lut32 = np.zeros(4096, np.uint32)
    lut32[0] = 1  # neither negacyclic nor periodic
    assert lib.cbs_gate_bootstrap_func_batch_device(c.handle, x.data_ptr(), x.data_ptr(), 1, 4096, lut.ctypes.data,
                                                    1 << 10, x.data_ptr(), x.data_ptr(), None) == 1  # q_in > 2N
    assert lib.cbs_gate_eval_func_batch_device(c.handle, x.data_ptr(), x.data_ptr(), 1, 2048, lut32.ctypes.data,
                                               BETA, x.data_ptr(), x.data_ptr(), None) == 1  # arbitrary, q > N
    assert lib.cbs_gate_eval_sign_batch_device(c.handle, x.data_ptr(), x.data_ptr(), 1, 1024, 1024, BETA, 0,
                                               x.data_ptr(), x.data_ptr(), None) == 1  # mod <= q
    c.set_fft_mode("fp32-split")
    try:
        assert lib.cbs_gate_eval_floor_batch_device(c.handle, x.data_ptr(), x.data_ptr(), 1, 1 << 14, 1024, 0, BETA,
                                                    x.data_ptr(), x.data_ptr(), None) == 6
    finally:
        c.set_fft_mode("fp64")
