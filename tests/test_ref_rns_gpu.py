"""The product's modup and moddown (cbs_rns_modup, cbs_rns_moddown_from_ntt; a4 and a6) against
the reference's own Phantom RNS tool -- a PhantomContext built from CKKS EncryptionParameters
and its DRNSTool::modup / moddown_from_NTT (include/rns.cuh:156-164, src/rns_bconv.cu:530-634,
776-828) -- rebuilt for sm_100a by `make -C oracle ref_gpu_rns` (ref_gpu_rns_shim.cu): the same
random NTT-domain inputs give the same words, at the shapes of the product's RNS tests and at
the Phantom-core size (N = 2^16, 24 + 2 and 24 + 8 primes)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ORACLE_DIR

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
REF_SO = ORACLE_DIR / "_ref" / "libref_rns.so"

CASES = [  # (logn, size_q, size_p, size_ql, count)
    (13, 5, 2, 5, 3),
    (13, 5, 2, 4, 1),
    (14, 6, 3, 5, 2),
    (12, 3, 2, 3, 2),
    (16, 24, 2, 24, 2),
    (16, 24, 8, 24, 1),
]


@pytest.fixture(scope="module")
def ref():
    if not REF_SO.exists():
        pytest.skip("reference Phantom RNS tool not built (make -C oracle ref_gpu_rns)")
    lib = ctypes.CDLL(str(REF_SO))
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    lib.ref_rns_create.argtypes = [u32, vp, u32, u32]
    lib.ref_rns_create.restype = vp
    lib.ref_rns_destroy.argtypes = [vp]
    lib.ref_rns_modup.argtypes = [vp, u32, vp, vp, u32, vp]
    lib.ref_rns_moddown_from_ntt.argtypes = [vp, u32, vp, vp, u32, vp]
    lib.ref_rns_rescale.argtypes = [vp, u32, vp, vp, u32, vp]
    return lib


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t, shape):
    return t.cpu().numpy().view(np.uint64).reshape(shape)


def _limbs(rng, mods, n, lead):
    """uniform residues [*lead][len(mods)][n], limb i below mods[i]"""
    x = rng.integers(0, 2 ** 62, size=(*lead, len(mods), n), dtype=np.uint64)
    return (x % mods.reshape(1, -1, 1)).astype(np.uint64) if lead else x % mods.reshape(-1, 1)


@pytest.mark.parametrize("logn,size_q,size_p,size_ql,count", CASES)
def test_modup_moddown_match_reference_rns_tool(pkg, ref, logn, size_q, size_p, size_ql, count):
    n = 1 << logn
    chain = np.zeros(size_q + size_p, np.uint64)
    pkg.call("cbs_get_primes", n, 50, size_q + size_p, chain.ctypes.data)  # Phantom chain order
    q, p = chain[:size_q].copy(), chain[size_q:].copy()
    ctx = pkg.RnsContext(n, q, p)
    rctx = ref.ref_rns_create(logn, chain.ctypes.data, size_q, size_p)
    assert rctx
    try:
        rng = np.random.default_rng(logn * 100 + size_ql)
        qlp = size_ql + size_p
        beta = ctx.beta(size_ql)
        ql_p = np.concatenate([q[:size_ql], p])
        # modup: c2 [count][ql][n] -> [count][beta][ql + p][n]
        c2 = _limbs(rng, q[:size_ql], n, (count,))
        mine = torch.zeros((count, beta, qlp, n), dtype=torch.int64, device="cuda")
        theirs = torch.zeros_like(mine)
        d_c2 = _dev(c2)
        pkg.call("cbs_rns_modup", ctx.handle, mine.data_ptr(), d_c2.data_ptr(), size_ql, count, None)
        assert ref.ref_rns_modup(rctx, size_ql, theirs.data_ptr(), d_c2.data_ptr(), count, None) == 0
        torch.cuda.synchronize()
        assert np.array_equal(_host(mine, mine.shape), _host(theirs, theirs.shape))
        # moddown_from_NTT (overwrite form): cx [polys][ql + p][n] -> [polys][ql][n]; the
        # reference works on cx in place, so each side gets its own copy
        polys = 2 * count
        cx = _limbs(rng, ql_p, n, (polys,))
        d_cx_m, d_cx_t = _dev(cx), _dev(cx)
        out_m = torch.zeros((polys, size_ql, n), dtype=torch.int64, device="cuda")
        out_t = torch.zeros_like(out_m)
        pkg.call("cbs_rns_moddown_from_ntt", ctx.handle, out_m.data_ptr(), d_cx_m.data_ptr(), size_ql, polys, 0, None)
        assert ref.ref_rns_moddown_from_ntt(rctx, size_ql, out_t.data_ptr(), d_cx_t.data_ptr(), polys, None) == 0
        torch.cuda.synchronize()
        assert np.array_equal(_host(out_m, out_m.shape), _host(out_t, out_t.shape))
    finally:
        ref.ref_rns_destroy(rctx)
        ctx.close()


@pytest.mark.parametrize("logn,size_q,size_ql", [(13, 5, 5), (14, 6, 4), (16, 24, 24)])
def test_rescale_matches_reference_rns_tool(pkg, ref, logn, size_q, size_ql):
    """cbs_ckks_rescale_to_next against the reference's DRNSTool::divide_and_round_q_last_ntt
    (src/rns.cu:1183-1208) on the same NTT-domain ciphertext: the same words."""
    n, size_p, size = 1 << logn, 2, 2
    chain = np.zeros(size_q + size_p, np.uint64)
    pkg.call("cbs_get_primes", n, 50, size_q + size_p, chain.ctypes.data)
    q, p = chain[:size_q].copy(), chain[size_q:].copy()
    ctx = pkg.RnsContext(n, q, p)
    rctx = ref.ref_rns_create(logn, chain.ctypes.data, size_q, size_p)
    assert rctx
    try:
        rng = np.random.default_rng(logn * 31 + size_ql)
        src = _limbs(rng, q[:size_ql], n, (size,))
        d_src_m, d_src_t = _dev(src), _dev(src)
        out_m = torch.zeros((size, size_ql - 1, n), dtype=torch.int64, device="cuda")
        out_t = torch.zeros_like(out_m)
        pkg.call("cbs_ckks_rescale_to_next", ctx.handle, out_m.data_ptr(), d_src_m.data_ptr(), size, size_ql, None)
        assert ref.ref_rns_rescale(rctx, size_ql, out_t.data_ptr(), d_src_t.data_ptr(), size, None) == 0
        torch.cuda.synchronize()
        assert np.array_equal(_host(out_m, out_m.shape), _host(out_t, out_t.shape))
    finally:
        ref.ref_rns_destroy(rctx)
        ctx.close()
