"""The oracle's one-bit GINX blind rotation against the reference's own CirBTS kernels
(bitwise/src/cirbts/kernel.cu: kernel_SpecialMS_IndexPos_Batch, kernel_SignedDigitDecompose2_
FusedFNWT_Batch, kernel_EvalAccCore_Binary_Batch; Phantom's inwt_1d_opt_outofplace_batched),
rebuilt for sm_100a by `make -C oracle ref_gpu_cirbts` and launched in the reference's
per-step sequence (ref_gpu_cirbts_shim.cu).  From the same initial accumulator, with the
product's keys (its [n][2 digits][2][N] NTT-domain layout is the reference's AoS RF key),
n = 630 steps of the reference kernels give the oracle's accumulator word for word.  The
product's exact-NTT blind rotation is bit-identical to the oracle (test_cbs_gpu.py), so this
pins a9's arithmetic -- modulus switch, signed gadget decomposition, key products, monomial
multiplication -- against the reference itself."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import OracleCbs
from conftest import ORACLE_DIR

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
REF_SO = ORACLE_DIR / "_ref" / "libref_cirbts.so"


@pytest.fixture(scope="module")
def ref():
    if not REF_SO.exists():
        pytest.skip("reference CirBTS kernels not built (make -C oracle ref_gpu_cirbts)")
    lib = ctypes.CDLL(str(REF_SO))
    vp, u32, u64, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
    lib.ref_cirbts_shoup.argtypes = [vp, vp, sz, u64]
    lib.ref_cirbts_blind_rotate_steps.argtypes = [vp, vp, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                                  u32, u64, u32, u32, u64, u32, vp]
    lib.ref_cirbts_blind_rotate_steps.restype = ctypes.c_int
    return lib


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def test_blind_rotation_matches_reference_kernels(pkg, oracle, ref):
    p = pkg.default_params()
    N, n, Q = p.N, p.n, p.Q
    keys = pkg.generate_keys_host(p, 23)
    oc = OracleCbs(oracle, p, keys)
    batch = 2
    rng = np.random.default_rng(9)
    a = rng.integers(0, p.q_lwe, size=(batch, n), dtype=np.uint64)
    b = rng.integers(0, p.q_lwe, batch, dtype=np.uint64)

    def orc_acc(steps):
        op = type(oc.op).from_buffer_copy(oc.op)
        op.n = steps
        out = np.zeros((batch, 2, N), np.uint64)
        oracle.orc_blind_rotate(ctypes.byref(op), ctypes.byref(oc.ok), a.ctypes.data, b.ctypes.data, batch, n,
                                out.ctypes.data, 0)
        return out

    init, want = orc_acc(0), orc_acc(n)

    # Phantom tables of Q (pinned to the reference's host code elsewhere) and the monomial
    # table NTT(X^k - 1), k < 2N, with X^(N+j) = -X^j (cirbts-init.cu:991-1010)
    tabs = [np.zeros(N, np.uint64) for _ in range(4)]
    ninv = np.zeros(2, np.uint64)
    dm = pkg.DModulus()
    pkg.call("cbs_ntt_tables_host", N, Q, *(t.ctypes.data for t in tabs), ninv.ctypes.data, ctypes.addressof(dm))
    monic = np.zeros((2 * N, N), np.uint64)
    k = np.arange(1, N)
    monic[k, k] = 1
    monic[1:N, 0] = Q - 1
    monic[N, 0] = Q - 2
    monic[N + k, k] = Q - 1
    monic[N + k, 0] = Q - 1
    oracle.orc_ntt_forward.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64,
                                       ctypes.c_void_p]
    oracle.orc_ntt_forward(monic.ctypes.data, 2 * N, N, Q, oc.rp.ctypes.data)

    ek = np.ascontiguousarray(keys["bsk"]).reshape(-1)
    eks = np.zeros_like(ek)
    ref.ref_cirbts_shoup(ek.ctypes.data, eks.ctypes.data, ek.size, Q)
    dmod = np.array([dm.value, dm.const_ratio[0], dm.const_ratio[1]], np.uint64)
    bitwidth = max(0, (p.num_lut - 1).bit_length())
    dev = {name: _dev(v) for name, v in [("acc", init), ("a", a), ("ek", ek), ("eks", eks), ("monic", monic),
                                         ("mod", dmod), ("tw", tabs[0]), ("tws", tabs[1]), ("itw", tabs[2]),
                                         ("itws", tabs[3]), ("ninv", ninv)]}
    st = ref.ref_cirbts_blind_rotate_steps(
        dev["acc"].data_ptr(), dev["a"].data_ptr(), n, n, batch, dev["ek"].data_ptr(), dev["eks"].data_ptr(),
        dev["monic"].data_ptr(), dev["mod"].data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(),
        dev["itw"].data_ptr(), dev["itws"].data_ptr(), dev["ninv"].data_ptr(), dev["ninv"].data_ptr() + 8, N, Q,
        p.base_g, p.digits_g, p.q_lwe, bitwidth, None)
    torch.cuda.synchronize()
    assert st == 0
    got = dev["acc"].cpu().numpy().view(np.uint64).reshape(batch, 2, N)
    assert not np.array_equal(got, init)
    assert np.array_equal(got, want)
