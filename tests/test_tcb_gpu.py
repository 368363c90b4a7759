"""GPU torus circuit bootstrap with PFKS: the level-2 LWEs match the exact oracle within the
FP64 rounding of the 64-bit-torus products, the PFKS rows are bit-exact against the oracle
on the same inputs, the RGSW rows decrypt to m g_k / -m g_k z1, and an external product with
the output RGSW selects the message (a CMux works with it)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle
from tcb_harness import OracleTcb, centered, declare_tcb, lwe64_phase_top, rgsw_row_errors, rlwe_phase

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev32(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _run(pkg, ctx, bits, seed):
    p = ctx.params
    a, b = ctx.encrypt(bits, seed=seed)
    da, db = _dev32(a), _dev32(b)
    cnt = len(bits)
    ext = torch.zeros((cnt, p.cb_levels, p.N2 + 1), dtype=torch.int64, device="cuda")
    rgsw = torch.zeros((cnt, p.cb_levels, 2, 2, p.N1), dtype=torch.int32, device="cuda")
    pkg.call("cbs_tcb_circuit_bootstrap_device", ctx.handle, da.data_ptr(), db.data_ptr(), cnt, ext.data_ptr(),
             rgsw.data_ptr(), None)
    torch.cuda.synchronize()
    return a, b, ext.cpu().numpy().view(np.uint64), rgsw.cpu().numpy().view(np.uint32)


def test_small_parity_against_oracle(pkg):
    p = pkg.tcb_default_params()
    p.n, p.N2, p.N1 = 64, 1024, 256
    ctx = pkg.TcbContext(p, max_batch=4)
    ctx.keygen(21)
    keys = ctx.export_keys(with_pfks=True)
    bits = np.array([1, 0, 1], np.uint8)
    a, b, ext, rgsw = _run(pkg, ctx, bits, 5)
    ot = OracleTcb(declare_tcb(load_oracle()), p, keys)
    want = ot.blind_rotate(a, b)
    for i, m in enumerate(int(x) for x in bits):
        for k in range(p.cb_levels):
            # The FP64 products on the 64-bit torus perturb the accumulator by ~2^-38; where a
            # coefficient sits at a rounding boundary of the 37 bits the gadget drops, the
            # digits then differ by one, which moves the phase by a sample of the gadget
            # rounding noise itself (~2^-21 here).  So the GPU and the exact phases agree to
            # within that noise, and both sit within it of m g_k.
            g = 2.0 ** (32 - (k + 1) * p.cb_bits)
            ph_gpu = lwe64_phase_top(ext[i, k], keys["z2"])
            ph_ref = lwe64_phase_top(want[i, k], keys["z2"])
            assert abs(ph_gpu - ph_ref) < 2 ** 14
            assert abs(ph_gpu - m * g) < 2 ** 14 and abs(ph_ref - m * g) < 2 ** 14
    assert np.array_equal(rgsw, ot.pfks(ext))  # the switch itself is exact
    err = rgsw_row_errors(rgsw, bits, keys["z1"], p.cb_bits, p.cb_levels)
    assert np.max(np.abs(err)) < 2 ** 16
    ctx.close()


def _ext_product(rgsw_k, ct, cb_bits, levels):
    """RGSW [levels][2][2][N] (row 2k+c: message on component c) x RLWE (a, b) -> RLWE, exact."""
    N = ct.shape[1]
    out = np.zeros((2, N), np.int64)
    off = (1 << (32 - levels * cb_bits - 1))
    for k in range(levels):
        off += (1 << (cb_bits - 1)) << (32 - (k + 1) * cb_bits)
    for c in range(2):
        w = (ct[c].astype(np.int64) + off) % (1 << 32)
        for k in range(levels):
            d = ((w >> (32 - (k + 1) * cb_bits)) & ((1 << cb_bits) - 1)) - (1 << (cb_bits - 1))
            for comp in range(2):
                full = np.convolve(d, centered(rgsw_k[k, c, comp]))
                prod = full[:N].copy()
                prod[:N - 1] -= full[N:]
                out[comp] = (out[comp] + prod) % (1 << 32)
    return out.astype(np.uint32)


def test_default_rows_and_cmux(pkg):
    """The configuration's parameters (n=630, N2=2048, 2^9 x 3, N1=1024, PFKS 2^4 x 8): row
    errors, and RGSW(m) (x) RLWE(1/4) decrypts to m/4."""
    ctx = pkg.TcbContext(max_batch=8)
    ctx.keygen(22)
    p = ctx.params
    keys = ctx.export_keys(with_pfks=False)
    bits = np.array([1, 0, 1, 1, 0, 0, 1, 0], np.uint8)
    _, _, _, rgsw = _run(pkg, ctx, bits, 6)
    err = rgsw_row_errors(rgsw, bits, keys["z1"], p.cb_bits, p.cb_levels)
    sigma = float(np.std(err))
    print(f"RGSW row error: sigma 2^{np.log2(sigma):.1f}, max 2^{np.log2(np.max(np.abs(err))):.1f} (units 2^-32)")
    assert np.max(np.abs(err)) < 2 ** 22
    rng = np.random.default_rng(1)
    z1 = keys["z1"].astype(np.int64)
    N1 = p.N1
    for i, m in enumerate(int(x) for x in bits):
        a = rng.integers(0, 1 << 32, N1, dtype=np.int64)
        msg = np.zeros(N1, np.int64)
        msg[0] = 1 << 30  # 1/4
        from tcb_harness import negacyclic_binary
        b = (negacyclic_binary(centered(a), z1) + msg + rng.integers(-8, 9, N1)) % (1 << 32)
        ct = np.stack([a % (1 << 32), b]).astype(np.uint32)
        out = _ext_product(rgsw[i], ct, p.cb_bits, p.cb_levels)
        ph = rlwe_phase(out, keys["z1"])
        assert abs(int(centered(ph[0] - m * (1 << 30)))) < 1 << 27  # within 1/32 of m/4
    ctx.close()


@pytest.mark.parametrize("mb", [2, 3])
def test_multibit_level2_parity_against_oracle(pkg, mb):
    """Grouped (multi-bit) level-2 blind rotation against the oracle's exact grouped rotation:
    the same FP64 digit-boundary argument as the one-bit test, and the PFKS rows it feeds decrypt
    to m g_k / -m g_k z1."""
    p = pkg.tcb_default_params()
    p.n, p.N2, p.N1 = 64, 1024, 256
    ctx = pkg.TcbContext(p, max_batch=4)
    try:
        ctx.keygen(23)
        ctx.set_multibit(mb)
        keys = ctx.export_keys(with_pfks=True)
        mbk = ctx.export_mb_bsk()
        bits = np.array([1, 0, 1], np.uint8)
        a, b, ext, rgsw = _run(pkg, ctx, bits, 7)
    finally:
        ctx.close()
    ot = OracleTcb(declare_tcb(load_oracle()), p, keys)
    want = ot.blind_rotate_mb(a, b, mbk, mb)
    for i, m in enumerate(int(x) for x in bits):
        for k in range(p.cb_levels):
            g = 2.0 ** (32 - (k + 1) * p.cb_bits)
            ph_gpu = lwe64_phase_top(ext[i, k], keys["z2"])
            ph_ref = lwe64_phase_top(want[i, k], keys["z2"])
            assert abs(ph_gpu - ph_ref) < 2 ** 14
            assert abs(ph_gpu - m * g) < 2 ** 14 and abs(ph_ref - m * g) < 2 ** 14
    assert np.array_equal(rgsw, ot.pfks(ext))
    err = rgsw_row_errors(rgsw, bits, keys["z1"], p.cb_bits, p.cb_levels)
    assert np.max(np.abs(err)) < 2 ** 16
