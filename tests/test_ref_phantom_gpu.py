"""GPU parity against the reference's own Phantom NTT kernels (src/ntt/ntt_1d.cu,
src/ntt/fntt_2d.cu, src/ntt/intt_2d.cu) rebuilt for sm_100a by `make -C oracle ref_gpu`:
the product's 1-D batched NTT and its multi-prime NTT give the same words as the reference's
kernels on the same inputs and tables.  Skipped when that library was not built here."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ORACLE_DIR, load_pkg

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
REF_SO = ORACLE_DIR / "_ref" / "libref_phantom_ntt.so"


@pytest.fixture(scope="module")
def ref():
    if not REF_SO.exists():
        pytest.skip("reference Phantom NTT library not built (make -C oracle ref_gpu)")
    lib = ctypes.CDLL(str(REF_SO))
    vp, sz, u32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32
    lib.ref_gpu_fnwt_1d_opt_batched.argtypes = [vp, vp, vp, vp, sz, sz, vp]
    lib.ref_gpu_inwt_1d_opt_batched.argtypes = [vp, vp, vp, vp, vp, vp, sz, sz, vp]
    lib.ref_gpu_ntt2d_create.argtypes = [u32, u32, vp]
    lib.ref_gpu_ntt2d_create.restype = vp
    lib.ref_gpu_ntt2d_forward.argtypes = [vp, vp, u32, u32, vp]
    lib.ref_gpu_ntt2d_backward.argtypes = [vp, vp, u32, u32, vp]
    lib.ref_gpu_ntt2d_destroy.argtypes = [vp]
    return lib


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def test_1d_batched_matches_reference_kernel(ref):
    pkg = load_pkg()
    n, q = 2048, None
    primes = np.zeros(1, np.uint64)
    pkg.call("cbs_get_primes", n, 54, 1, primes.ctypes.data)
    q = int(primes[0])
    tabs = [np.zeros(n, np.uint64) for _ in range(4)]
    ninv = np.zeros(2, np.uint64)
    dm = pkg.DModulus()
    pkg.call("cbs_ntt_tables_host", n, q, *(t.ctypes.data for t in tabs), ninv.ctypes.data, ctypes.addressof(dm))
    d_tabs = [_dev(t) for t in tabs]
    dmod = np.array([dm.value, dm.const_ratio[0], dm.const_ratio[1]], np.uint64)
    d_mod = torch.from_numpy(dmod.view(np.int64)).cuda()
    d_ninv = _dev(ninv)
    rng = np.random.default_rng(4)
    x = rng.integers(0, q, size=(37, n), dtype=np.uint64)
    mine, theirs = _dev(x), _dev(x)
    pkg.call("cbs_fnwt_1d_opt_batched", mine.data_ptr(), d_tabs[0].data_ptr(), d_tabs[1].data_ptr(), d_mod.data_ptr(),
             n, 37, None)
    assert ref.ref_gpu_fnwt_1d_opt_batched(theirs.data_ptr(), d_tabs[0].data_ptr(), d_tabs[1].data_ptr(),
                                           d_mod.data_ptr(), n, 37, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_host(mine), _host(theirs))
    pkg.call("cbs_inwt_1d_opt_batched", mine.data_ptr(), d_tabs[2].data_ptr(), d_tabs[3].data_ptr(), d_mod.data_ptr(),
             d_ninv.data_ptr(), d_ninv.data_ptr() + 8, n, 37, None)
    assert ref.ref_gpu_inwt_1d_opt_batched(theirs.data_ptr(), d_tabs[2].data_ptr(), d_tabs[3].data_ptr(),
                                           d_mod.data_ptr(), d_ninv.data_ptr(), d_ninv.data_ptr() + 8, n, 37,
                                           None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_host(mine), _host(theirs))
    assert np.array_equal(_host(mine).reshape(x.shape), x)


@pytest.mark.parametrize("logn,limbs", [(12, 3), (16, 24)])
def test_2d_matches_reference_kernel(ref, logn, limbs):
    pkg = load_pkg()
    n = 1 << logn
    chain = np.zeros(limbs + 2, np.uint64)
    pkg.call("cbs_get_primes", n, 50, limbs + 2, chain.ctypes.data)
    q, p = chain[:limbs], chain[limbs:]
    ctx = pkg.RnsContext(n, q, p)
    table = ref.ref_gpu_ntt2d_create(logn, limbs + 2, chain.ctypes.data)
    assert table
    rng = np.random.default_rng(logn)
    x = np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in chain])
    mine, theirs = _dev(x), _dev(x)
    # limbs 1 .. limbs of the chain (start index 1), the reference's calling convention
    pkg.call("cbs_nwt_2d_radix8_forward_inplace", ctx.handle, mine.data_ptr(), limbs, 1, None)
    assert ref.ref_gpu_ntt2d_forward(table, theirs.data_ptr(), limbs, 1, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_host(mine), _host(theirs))
    pkg.call("cbs_nwt_2d_radix8_backward_inplace", ctx.handle, mine.data_ptr(), limbs, 1, None)
    assert ref.ref_gpu_ntt2d_backward(table, theirs.data_ptr(), limbs, 1, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_host(mine), _host(theirs))
    assert np.array_equal(_host(mine).reshape(x.shape), x)
    ref.ref_gpu_ntt2d_destroy(table)
    ctx.close()
