"""The CMux entry point (one LUT-tree level of the reference's kernel_LUT_CMUX_Delta +
kernel_LUT_CMUX_ExternalProduct, examples/aes_transcipher/gpu_lut.cuh:521-595) on both
backends: the exact NTT CMux bit-exact against the oracle's CMux, and the FP64 FFT CMux of
the AES path checked level by level against the exact CMux on the same inputs."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_encrypt_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

# Tolerance on one FFT CMux: max |phase(FFT) - phase(exact)| over all coefficients.  The
# products of 6-bit digits by 54-bit row spectra (8 rows, N = 2048) round with ~2^14-2^16 of
# FP64 error per output coefficient; the phase b - a*s multiplies the mask error by the
# ternary secret (|s|_2 ~ 2^5.2), so the phase error stays near 2^20-2^22.  A CMux itself adds
# ~2^11.2 x the rows' noise (~2^40 at these parameters): the FFT error is 2^-18 of that.
CMUX_PHASE_TOL = 2 ** 26


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t, shape):
    return t.cpu().numpy().view(np.uint64).reshape(shape)


@pytest.fixture(scope="module")
def cctx(pkg):
    c = pkg.Context(max_batch=64)
    c.keygen(31)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ckeys(cctx):
    return cctx.export_keys()


@pytest.fixture(scope="module")
def coc(oracle, cctx, ckeys):
    return OracleCbs(oracle, cctx.params, ckeys)


@pytest.fixture(scope="module")
def controls(pkg, cctx, ckeys):
    """RGSW rows of 8 random bits from the exact CBS (NTT backend), [8][num_lut][2][2][N]."""
    p = cctx.params
    rng = np.random.default_rng(41)
    bits = rng.integers(0, 2, 8)
    a, b = lwe_encrypt_bits(rng, ckeys["s_lwe"], bits, p.q_lwe)
    da, db = _dev(a), _dev(b)
    view = ctypes.c_void_p()
    pkg.call("cbs_circuit_bootstrap_batch_device", cctx.handle, da.data_ptr(), db.data_ptr(), 8, p.n,
             ctypes.byref(view), None)
    per = p.num_lut * 4 * p.N
    out = torch.empty(8 * per, dtype=torch.int64, device="cuda")
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    torch.cuda.synchronize()
    assert cudart.cudaMemcpy(out.data_ptr(), view.value, 8 * per * 8, 3) == 0
    return bits, _host(out, (8, per))


def _exact_cmux(coc, p, ct0, ct1, rgsw):
    Q = p.Q
    delta = ((ct1.astype(object) - ct0.astype(object)) % Q).astype(np.uint64)
    prod = np.zeros((2, p.N), np.uint64)
    coc.o.orc_external_product(np.ascontiguousarray(delta).ctypes.data, np.ascontiguousarray(rgsw).ctypes.data,
                               prod.ctypes.data, p.N, Q, coc.rp.ctypes.data, coc.irp.ctypes.data, int(coc.ninv[0]),
                               p.base_cc, p.num_lut)
    return ((ct0.astype(object) + prod.astype(object)) % Q).astype(np.uint64)


def test_cmux_ntt_bit_exact(pkg, cctx, coc, controls):
    """Exact backend: every output equals the oracle's CMux word for word; per-item controls."""
    p = cctx.params
    _, rg = controls
    rng = np.random.default_rng(42)
    count = 5
    ct0 = rng.integers(0, p.Q, size=(count, 2, p.N), dtype=np.uint64)
    ct1 = rng.integers(0, p.Q, size=(count, 2, p.N), dtype=np.uint64)
    ctrl = np.ascontiguousarray(rg[[3, 0, 7, 3, 1]])
    out = torch.zeros((count, 2, p.N), dtype=torch.int64, device="cuda")
    d0, d1, dc = _dev(ct0), _dev(ct1), _dev(ctrl)  # held: a freed temporary's block would be reused
    pkg.call("cbs_cmux_batch_device", cctx.handle, d0.data_ptr(), d1.data_ptr(), dc.data_ptr(), rg.shape[1], count,
             out.data_ptr(), None)
    torch.cuda.synchronize()
    got = _host(out, (count, 2, p.N))
    for u in range(count):
        want = _exact_cmux(coc, p, ct0[u], ct1[u], ctrl[u].reshape(-1))
        assert np.array_equal(got[u], want), u


def test_cmux_fft_phase_error_per_level(pkg, cctx, coc, controls):
    """FFT backend, a 256-leaf LUT tree run level by level through the FFT CMux: at every
    level each output is compared with the exact CMux of the same inputs (the FFT path's own
    previous-level outputs), so the bound holds per CMux and errors do not compound in the
    comparison; the selected leaf is checked at the end by decryption."""
    p = cctx.params
    bits, rg = controls
    Q = p.Q
    rng = np.random.default_rng(43)
    leaves = np.zeros((256, 2, p.N), np.uint64)
    # leaf x encrypts bit c of x times Q/2 in coefficient c (c < 8): a random mask, b = a*s + m in
    # the NTT domain, no noise
    leaves[:, 0] = rng.integers(0, Q, size=(256, p.N), dtype=np.uint64)
    s_ntt = (coc.k["s_rlwe"].astype(np.int64) % Q).astype(np.uint64)
    coc.o.orc_ntt_forward(s_ntt, 1, p.N, Q, coc.rp)
    for x in range(256):
        m = np.zeros(p.N, np.uint64)
        m[:8] = [((x >> c) & 1) * (Q // 2) for c in range(8)]
        coc.o.orc_ntt_forward(m, 1, p.N, Q, coc.rp)
        prod = (leaves[x, 0].astype(object) * s_ntt.astype(object)) % Q
        leaves[x, 1] = ((prod + m.astype(object)) % Q).astype(np.uint64)
    pkg.call("cbs_context_set_br_backend", cctx.handle, pkg.BR_FFT64)
    try:
        cur = leaves
        worst = []
        for level in range(8):
            pairs = cur.shape[0] // 2
            ct0 = np.ascontiguousarray(cur[0::2])
            ct1 = np.ascontiguousarray(cur[1::2])
            out = torch.zeros((pairs, 2, p.N), dtype=torch.int64, device="cuda")
            ctrl, d0, d1 = _dev(rg[level]), _dev(ct0), _dev(ct1)
            pkg.call("cbs_cmux_batch_device", cctx.handle, d0.data_ptr(), d1.data_ptr(), ctrl.data_ptr(), 0, pairs,
                     out.data_ptr(), None)
            torch.cuda.synchronize()
            got = _host(out, (pairs, 2, p.N))
            w = 0
            for u in range(0, pairs, max(1, pairs // 8)):  # up to 8 CMuxes checked per level
                want = _exact_cmux(coc, p, ct0[u], ct1[u], rg[level])
                d = coc.phase_coef(got[u]) - coc.phase_coef(want)
                w = max(w, max(abs(((int(v) + Q // 2) % Q) - Q // 2) for v in d))
            worst.append(w)
            cur = got
        print("FFT CMux max |phase error| per level (log2):",
              " ".join(f"{np.log2(w + 1):.1f}" for w in worst))
        assert max(worst) < CMUX_PHASE_TOL
        sel = int(sum(int(bits[k]) << k for k in range(8)))
        ph = coc.phase_coef(cur[0])
        dec = sum(((((2 * (int(ph[c]) % Q) + Q // 2) // Q) & 1) << c) for c in range(8))
        assert dec == sel
    finally:
        pkg.call("cbs_context_set_br_backend", cctx.handle, pkg.BR_NTT)


def test_cmux_rejects_bad_stride(pkg, cctx):
    x = torch.zeros(16, dtype=torch.int64, device="cuda")
    st = pkg.load().cbs_cmux_batch_device(cctx.handle, x.data_ptr(), x.data_ptr(), x.data_ptr(), 7, 1, x.data_ptr(),
                                          None)
    assert st == 1
    assert pkg.load().cbs_cmux_batch_device(cctx.handle, None, None, None, 0, 0, None, None) == 0
