"""The product's sample extract + LWE key switch (cbs_extract_keyswitch_device) against the
reference's own kernel, kernel_SampleExtractKeySwitchToLWE (bitwise/examples/aes_gpu_ks.cuh:
538-607), rebuilt for sm_100a by `make -C oracle ref_gpu_extract` from the reference header
(ref_gpu_extract_shim.cu): the same random coefficient-domain words mod Q, the product's
key-switching key (the packed [2][N][base_ks][n+1] u16 layout both use) and the same
(word, coefficient) list give bit-identical LWE outputs, through both of the reference's
launch variants (coefficient index computed in the kernel, or read from its pre-encoded
map).  This pins a14 against the reference itself, not only against the oracle."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

REF_SO = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libref_extract.so"


@pytest.fixture(scope="module")
def ref():
    if not REF_SO.exists():
        pytest.skip("reference extraction kernel not built (make -C oracle ref_gpu_extract)")
    lib = ctypes.CDLL(str(REF_SO))
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    lib.ref_gpu_extract_keyswitch.argtypes = [vp, u32, u32, u32, u32, vp, vp, vp, u32, u64, u64, vp, vp, u32,
                                              ctypes.c_int]
    lib.ref_gpu_extract_keyswitch.restype = ctypes.c_int
    return lib


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(max_batch=256)
    c.keygen(17)
    yield c
    c.close()


def _dev(a):
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int64) if a.dtype == np.uint64 else a.view(np.int16)).cuda()


@pytest.mark.parametrize("mapped", [0, 1])
def test_extract_keyswitch_matches_reference_kernel(pkg, ref, ctx, mapped):
    p = ctx.params
    N, n = p.N, p.n
    keys = ctx.export_keys()
    ksk = np.ascontiguousarray(keys["ksk"]).reshape(-1)
    rng = np.random.default_rng(40 + mapped)
    W, count = 8, 256
    words = rng.integers(0, p.Q, size=(W, 2, N), dtype=np.uint64)
    word = rng.integers(0, W, count, dtype=np.uint32)
    idx = rng.integers(0, N, count, dtype=np.uint32)
    idx[:4] = [0, 1, N - 1, N // 2]  # edges of the extraction index
    info = ((word << 16) | idx).astype(np.uint32)
    stride = n + 3  # a row stride above n, as both entry points take

    d_words = _dev(words)
    oa = torch.zeros((count, stride), dtype=torch.int64, device="cuda")
    ob = torch.zeros(count, dtype=torch.int64, device="cuda")
    pkg.call("cbs_extract_keyswitch_device", ctx.handle, d_words.data_ptr(), W, info.ctypes.data, count,
             oa.data_ptr(), ob.data_ptr(), stride, None)
    torch.cuda.synchronize()

    d_ksk = _dev(ksk)
    d_a = _dev(words[:, 0, :])
    d_b = _dev(words[:, 1, :])
    d_info = torch.from_numpy(info.view(np.int32)).cuda()
    ra = torch.zeros((count, stride), dtype=torch.int64, device="cuda")
    rb = torch.zeros(count, dtype=torch.int64, device="cuda")
    st = ref.ref_gpu_extract_keyswitch(d_ksk.data_ptr(), n, N, p.base_ks, p.qks, d_a.data_ptr(), d_b.data_ptr(),
                                       d_info.data_ptr(), count, p.Q, p.q_lwe, ra.data_ptr(), rb.data_ptr(), stride,
                                       mapped)
    torch.cuda.synchronize()
    assert st == 0
    got_a = oa.cpu().numpy()[:, :n]
    want_a = ra.cpu().numpy()[:, :n]
    assert np.array_equal(got_a, want_a)
    assert np.array_equal(ob.cpu().numpy(), rb.cpu().numpy())
    assert (want_a >= 0).all() and (want_a < p.q_lwe).all()
