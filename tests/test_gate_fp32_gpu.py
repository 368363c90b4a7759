"""GPU checks of the FP32 external products of the torus-32 gate bootstrap
(cbs_gate_set_fft_mode) against the FP64 path, which is bit-exact to the exact-integer oracle
(test_gate_gpu.py; re-checked here on four ciphertexts): the noise of the extracted LWE
(its phase under the RLWE key minus the expected +-1/8) in each mode, decryption of the
key-switched outputs, gates, the ragged launch, and the argument checks.

The accumulators of the two paths are not compared coefficient by coefficient: once one
FP32 rounding differs, the gadget digits of the next step differ and the accumulator becomes
another encryption of (nearly) the same phase, with unrelated coefficients.  What carries
over is the phase.  Split FP32 (keys k = lo + 2^S hi, S = log2 N + 14, the hi limb's
products exact) adds its lo-limb rounding (about 2^11 rms per external product on the 2^32
torus, ~2^20.7 of phase after n = 636 steps) to the bootstrapping-key noise (~2^23 of
phase): the output noise barely moves.  Plain FP32 (whole keys, ~2^19 rms per product)
adds ~2^28.7 of phase, at the 2^29 margin itself: it is measured, not required to decrypt."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle
from gate_harness import OracleGate, declare_gate

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

# split FP32: output noise within this factor of the FP64 path's, and its max far below the
# 2^29 margin
SPLIT_SIGMA_RATIO = 1.25
SPLIT_NOISE_MAX = 2 ** 27


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _centre(d):
    d = np.asarray(d, np.int64) % (1 << 32)
    return np.where(d >= 1 << 31, d - (1 << 32), d)


@pytest.fixture(scope="module")
def fctx(pkg):
    c = pkg.GateContext(max_batch=512)
    c.keygen(11)
    yield c
    c.close()


@pytest.fixture(scope="module")
def fkeys(fctx):
    return fctx.export_keys()


def _bootstrap(pkg, ctx, a, b):
    p = ctx.params
    cnt = len(b)
    da, db = _dev(a), _dev(b)
    ext = torch.zeros((cnt, p.N + 1), dtype=torch.int32, device="cuda")
    oa = torch.zeros((cnt, p.n), dtype=torch.int32, device="cuda")
    ob = torch.zeros(cnt, dtype=torch.int32, device="cuda")
    pkg.call("cbs_gate_bootstrap_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), cnt, ext.data_ptr(),
             oa.data_ptr(), ob.data_ptr(), None)
    torch.cuda.synchronize()
    return _host(ext), _host(oa), _host(ob)


def _in_mode(ctx, mode, fn):
    ctx.set_fft_mode(mode)
    try:
        return fn()
    finally:
        ctx.set_fft_mode("fp64")


@pytest.mark.parametrize("mode", ["fp32-split", "fp32"])
def test_fp32_noise_against_exact(pkg, fctx, fkeys, mode):
    p = fctx.params
    rng = np.random.default_rng(7)
    bits = rng.integers(0, 2, 512).astype(np.uint8)
    a, b = fctx.encrypt(bits, seed=21)
    ext64, _, _ = _bootstrap(pkg, fctx, a, b)
    # the FP64 path is the exact product (bit-exact to the oracle): re-check four ciphertexts
    og = OracleGate(declare_gate(load_oracle()), p, fkeys)
    assert np.array_equal(ext64[:4], og.blind_rotate(a[:4], b[:4]))
    ext32, oa32, ob32 = _in_mode(fctx, mode, lambda: _bootstrap(pkg, fctx, a, b))
    z = fkeys["z_rlwe"].astype(np.int64)
    want = np.where(bits == 1, 1 << 29, -(1 << 29))

    def noise(ext):
        ph = ext[:, p.N].astype(np.int64) - ext[:, : p.N].astype(np.int64) @ z
        return _centre(ph - want).astype(np.float64)

    n64, n32 = noise(ext64), noise(ext32)
    s64, s32 = n64.std(), n32.std()
    wrong = int(np.count_nonzero(fctx.decrypt(oa32, ob32) != bits))
    print(f"{mode}: output noise sigma 2^{np.log2(s32):.2f} max 2^{np.log2(np.abs(n32).max()):.2f}; "
          f"FP64 sigma 2^{np.log2(s64):.2f} max 2^{np.log2(np.abs(n64).max()):.2f} (margin 2^29); "
          f"{wrong}/512 bits wrong")
    if mode == "fp32-split":
        assert s32 < SPLIT_SIGMA_RATIO * s64
        assert np.abs(n32).max() < SPLIT_NOISE_MAX
        assert wrong == 0
    else:
        assert s32 > 4 * s64  # the whole-key FP32 error dominates the output noise


@pytest.fixture(scope="module")
def quiet(pkg):
    """A context whose bootstrapping keys carry no noise: the output noise is then the gadget
    rounding (FP64) plus the FP32 rounding of the external products."""
    gp = pkg.gate_default_params()
    gp.sigma_rlwe = 0.0
    c = pkg.GateContext(gp, max_batch=256)
    c.keygen(12)
    yield c, c.export_keys()
    c.close()


# output-noise sigma with noise-free keys (log2, torus 2^32): FP64 ~ 2^18.4 (gadget rounding),
# split FP32 ~ 2^21 (+ the lo limb's rounding), plain FP32 ~ 2^28.7
QUIET_SIGMA_MAX = {"fp64": 19.5, "fp32-split": 22.5}
QUIET_SIGMA_MIN_FP32 = 26.0


def test_fp32_rounding_noise_with_noise_free_keys(pkg, quiet):
    ctx, keys = quiet
    p = ctx.params
    bits = np.random.default_rng(8).integers(0, 2, 256).astype(np.uint8)
    a, b = ctx.encrypt(bits, seed=22)
    z = keys["z_rlwe"].astype(np.int64)
    want = np.where(bits == 1, 1 << 29, -(1 << 29))
    sig = {}
    for mode in ("fp64", "fp32-split", "fp32"):
        ext, _, _ = _in_mode(ctx, mode, lambda: _bootstrap(pkg, ctx, a, b))
        nz = _centre(ext[:, p.N].astype(np.int64) - ext[:, : p.N].astype(np.int64) @ z - want).astype(np.float64)
        sig[mode] = np.log2(nz.std())
        print(f"noise-free keys, {mode}: output noise sigma 2^{sig[mode]:.2f} max 2^{np.log2(np.abs(nz).max()):.2f}")
    assert sig["fp64"] < QUIET_SIGMA_MAX["fp64"]
    assert sig["fp32-split"] < QUIET_SIGMA_MAX["fp32-split"]
    assert sig["fp32"] > QUIET_SIGMA_MIN_FP32


def test_fp32_split_gates(pkg, fctx):
    p = fctx.params
    rng = np.random.default_rng(31)
    cnt = 256
    x = rng.integers(0, 2, cnt).astype(np.uint8)
    y = rng.integers(0, 2, cnt).astype(np.uint8)
    a1, b1 = fctx.encrypt(x, seed=32)
    a2, b2 = fctx.encrypt(y, seed=33)
    da1, db1, da2, db2 = _dev(a1), _dev(b1), _dev(a2), _dev(b2)
    truth = {pkg.GATE_NAND: 1 - (x & y), pkg.GATE_XOR: x ^ y, pkg.GATE_OR: x | y}

    def run():
        outs = {}
        for g in truth:
            oa = torch.zeros((cnt, p.n), dtype=torch.int32, device="cuda")
            ob = torch.zeros(cnt, dtype=torch.int32, device="cuda")
            pkg.call("cbs_gate_eval_batch_device", fctx.handle, g, da1.data_ptr(), db1.data_ptr(), da2.data_ptr(),
                     db2.data_ptr(), cnt, oa.data_ptr(), ob.data_ptr(), None)
            torch.cuda.synchronize()
            outs[g] = (_host(oa), _host(ob))
        return outs

    outs = _in_mode(fctx, "fp32-split", run)
    for g, want in truth.items():
        assert np.array_equal(fctx.decrypt(*outs[g]), want), g


def test_fp32_split_ragged_launch(pkg, fctx):
    """The ragged (request-table) launch runs the same FP32 kernel."""
    p = fctx.params
    sizes = [3, 17, 1, 40]
    reqs, keep, bits_all = [], [], []
    for i, cnt in enumerate(sizes):
        bits = np.random.default_rng(50 + i).integers(0, 2, cnt).astype(np.uint8)
        a, b = fctx.encrypt(bits, seed=60 + i)
        da, db = _dev(a), _dev(b)
        oa = torch.zeros((cnt, p.n), dtype=torch.int32, device="cuda")
        ob = torch.zeros(cnt, dtype=torch.int32, device="cuda")
        keep.append((da, db, oa, ob))
        bits_all.append(bits)
        reqs.append((da.data_ptr(), db.data_ptr(), oa.data_ptr(), ob.data_ptr(), cnt))

    def run():
        fctx.ragged_plan(reqs, grid_ctas=16)  # fewer CTAs than ciphertexts: CTAs loop
        fctx.ragged_launch()
        torch.cuda.synchronize()

    _in_mode(fctx, "fp32-split", run)
    for (da, db, oa, ob), bits in zip(keep, bits_all):
        assert np.array_equal(fctx.decrypt(_host(oa), _host(ob)), bits)


def test_fft_mode_argument_checks(pkg, fctx):
    with pytest.raises(pkg.CbsError):
        pkg.call("cbs_gate_set_fft_mode", fctx.handle, 7)
    fctx.set_multibit(2)
    try:
        with pytest.raises(pkg.CbsError):
            fctx.set_fft_mode("fp32-split")
    finally:
        fctx.set_multibit(1)
    fctx.set_fft_mode("fp32-split")
    try:
        with pytest.raises(pkg.CbsError):
            fctx.set_multibit(2)
    finally:
        fctx.set_fft_mode("fp64")
    # 8-bit digits: the split's top limb would not round exactly
    gp = pkg.gate_default_params()
    gp.bg_bits, gp.levels = 8, 3
    c = pkg.GateContext(gp, max_batch=4)
    try:
        with pytest.raises(pkg.CbsError):
            c.set_fft_mode("fp32-split")
        c.set_fft_mode("fp32")  # no exactness claim: allowed
    finally:
        c.close()
