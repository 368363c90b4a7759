"""The oracle's blind rotation (a9) and HomTrace + SchemeSwitch (a10) against the reference's
own CirBTS kernels (bitwise/src/cirbts/kernel.cu) and Phantom's 1-D NTT (src/ntt/ntt_1d.cu),
rebuilt for sm_100a by `make -C oracle ref_gpu_cirbts` and launched in the reference's launch
sequences (ref_gpu_cirbts_shim.cu):
* blind rotation: kernel_SpecialMS_IndexPos_Batch, then per step inwt_1d_opt_outofplace_batched,
  kernel_SignedDigitDecompose2_FusedFNWT_Batch and kernel_EvalAccCore_Binary_Batch with the
  product's keys (its [n][2 digits][2][N] NTT-domain layout is the reference's AoS RF key):
  from the same initial accumulator, n = 630 steps give the oracle's accumulator word for word;
  likewise the grouped mb = 2 sequence (kernel_EvalAccCore_Binary_MB2_Grouped_Batch), the staged
  mb = 4 sequence (MB3 grouped kernel, then a one-key step) and the AES example's mb = 3 SoA
  sequence against the oracle's exact grouped rotation; and LMKCDEY_EvalAcc
  (cirbts-lmkcdey.cu:105-407: host buckets, kernel_Permute_Only, the LMKCDEY decompositions,
  kernel_MultAdd, kernel_AddInPlace) against the oracle's LMKCDEY accumulator;
* HomTrace + SchemeSwitch: kernel_GenerateCoefficientAutoMaps, per round the permuting INTT,
  kernel_Fused_Permute_Decompose, the NTT and kernel_MultAddUpdate_HT_PermuteC1, then
  kernel_MultAddUpdate_SS and kernel_SaveToRGSW: the oracle's RGSW rows word for word, and the
  product's automorphism maps.
The product's exact-NTT kernels are bit-identical to the oracle (test_cbs_gpu.py), so these pin
a9 and a10 against the reference itself."""
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


def _tables(pkg, N, Q):
    """Phantom tables of Q (pinned to the reference's host code elsewhere) and the DModulus."""
    tabs = [np.zeros(N, np.uint64) for _ in range(4)]
    ninv = np.zeros(2, np.uint64)
    dm = pkg.DModulus()
    pkg.call("cbs_ntt_tables_host", N, Q, *(t.ctypes.data for t in tabs), ninv.ctypes.data, ctypes.addressof(dm))
    return tabs, ninv, np.array([dm.value, dm.const_ratio[0], dm.const_ratio[1]], np.uint64)


def _monic(oracle, oc, N, Q):
    """NTT(X^k - 1) for k < 2N with X^(N+j) = -X^j (cirbts-init.cu:991-1010)."""
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
    return monic


def _orc_acc(oracle, oc, a, b, steps, mbk=None, mb=1):
    """The oracle's accumulator after `steps` LWE coefficients, not finalized (NTT domain)."""
    op = type(oc.op).from_buffer_copy(oc.op)
    op.n = steps
    batch, stride = a.shape
    out = np.zeros((batch, 2, oc.p.N), np.uint64)
    if mbk is None:
        oracle.orc_blind_rotate(ctypes.byref(op), ctypes.byref(oc.ok), a.ctypes.data, b.ctypes.data, batch, stride,
                                out.ctypes.data, 0)
    else:
        oracle.orc_blind_rotate_mb(ctypes.byref(op), ctypes.byref(oc.ok), mbk.ctypes.data, mb, a.ctypes.data,
                                   b.ctypes.data, batch, stride, out.ctypes.data, 0)
    return out


@pytest.mark.parametrize("preset", ["3x12", "2x18"])
def test_blind_rotation_matches_reference_kernels(pkg, oracle, ref, preset):
    """Both blind-rotation gadgets (2^12 x 3, the default set, and 2^18 x 2)."""
    p = pkg.preset_params(preset)
    N, n, Q = p.N, p.n, p.Q
    keys = pkg.generate_keys_host(p, 23)
    oc = OracleCbs(oracle, p, keys)
    batch = 2
    rng = np.random.default_rng(9)
    a = rng.integers(0, p.q_lwe, size=(batch, n), dtype=np.uint64)
    b = rng.integers(0, p.q_lwe, batch, dtype=np.uint64)

    init, want = _orc_acc(oracle, oc, a, b, 0), _orc_acc(oracle, oc, a, b, n)
    tabs, ninv, dmod = _tables(pkg, N, Q)
    monic = _monic(oracle, oc, N, Q)

    ek = np.ascontiguousarray(keys["bsk"]).reshape(-1)
    eks = np.zeros_like(ek)
    ref.ref_cirbts_shoup(ek.ctypes.data, eks.ctypes.data, ek.size, Q)
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


def test_trace_schemeswitch_matches_reference_kernels(pkg, oracle, ref):
    """HomTrace + SchemeSwitch (a10) in the reference's default launch sequence on the same
    MV RLWEs and keys give the oracle's RGSW rows word for word, and the reference's own
    automorphism-map kernel gives the product's maps."""
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    ref.ref_cirbts_trace_schemeswitch.argtypes = [vp, vp, u32, vp, vp, vp, vp, u32, u32, u32, u32, u32, vp, vp, vp,
                                                  vp, vp, vp, vp, vp, u32, u64, vp, vp]
    ref.ref_cirbts_trace_schemeswitch.restype = ctypes.c_int
    oracle.orc_trace_schemeswitch.argtypes = [vp, vp, vp, u32, vp]
    p = pkg.default_params()
    N, Q = p.N, p.Q
    rounds = N.bit_length() - 1 - p.trace_shift
    keys = pkg.generate_keys_host(p, 29)
    oc = OracleCbs(oracle, p, keys)
    count = 4
    ct = np.random.default_rng(10).integers(0, Q, size=(count, 2, N), dtype=np.uint64)
    want = np.zeros((count, 2, 2, N), np.uint64)
    oracle.orc_trace_schemeswitch(ctypes.byref(oc.op), ctypes.byref(oc.ok), ct.ctypes.data, count, want.ctypes.data)

    tabs, ninv, dmod = _tables(pkg, N, Q)
    ht = np.ascontiguousarray(keys["ht"]).reshape(-1)
    ss = np.ascontiguousarray(keys["ss"]).reshape(-1)
    hts, sss = np.zeros_like(ht), np.zeros_like(ss)
    ref.ref_cirbts_shoup(ht.ctypes.data, hts.ctypes.data, ht.size, Q)
    ref.ref_cirbts_shoup(ss.ctypes.data, sss.ctypes.data, ss.size, Q)
    dev = {name: _dev(v) for name, v in [("c0", ct[:, 0, :]), ("c1", ct[:, 1, :]), ("ht", ht), ("hts", hts),
                                         ("ss", ss), ("sss", sss), ("mod", dmod), ("tw", tabs[0]), ("tws", tabs[1]),
                                         ("itw", tabs[2]), ("itws", tabs[3]), ("ninv", ninv)]}
    maps = torch.zeros((rounds, N), dtype=torch.int32, device="cuda")
    rows = torch.zeros((count, 2, 2, N), dtype=torch.int64, device="cuda")
    st = ref.ref_cirbts_trace_schemeswitch(
        dev["c0"].data_ptr(), dev["c1"].data_ptr(), count, dev["ht"].data_ptr(), dev["hts"].data_ptr(),
        dev["ss"].data_ptr(), dev["sss"].data_ptr(), rounds, p.base_ht, p.digits_ht, p.base_ss, p.digits_ss,
        maps.data_ptr(), dev["mod"].data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(), dev["itw"].data_ptr(),
        dev["itws"].data_ptr(), dev["ninv"].data_ptr(), dev["ninv"].data_ptr() + 8, N, Q, rows.data_ptr(), None)
    torch.cuda.synchronize()
    assert st == 0
    assert np.array_equal(maps.cpu().numpy().view(np.uint32), np.asarray(keys["maps"]).reshape(rounds, N))
    assert np.array_equal(rows.cpu().numpy().view(np.uint64), want)


@pytest.mark.parametrize("preset,mb,steps", [("3x12", 2, 630), ("2x18", 2, 630), ("3x12", 4, 630),
                                              ("2x18", 4, 629), ("2x18", 4, 627)])
def test_grouped_blind_rotation_matches_reference_kernels(pkg, oracle, ref, preset, mb, steps):
    """The grouped blind rotation: mb = 2 (CIRBTS_PBS_MULTIBIT=2), the reference's
    kernel_EvalAccCore_Binary_MB2_Grouped_Batch sequence, and the staged mb = 4
    (CIRBTS_PBS_MULTIBIT=4: kernel_EvalAccCore_Binary_MB3_Grouped_Batch on coefficients 0-2 of a
    group, then a fresh decomposition and the one-key kernel with key 3), with the product's
    grouped keys re-laid [subset][group] as the reference's RF key, reproduce the oracle's exact
    grouped accumulator word for word.  The mb = 4 cases end on a group of 2 (the reference's
    MB2 tail), 1 (its one-key tail) and 3 coefficients (no one-bit step).  The product's FFT form
    is checked against that oracle within its phase-error bound (test_cbs_fft_gpu.py)."""
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    fn = ref.ref_cirbts_blind_rotate_mb2 if mb == 2 else ref.ref_cirbts_blind_rotate_mb4
    fn.argtypes = [vp, vp, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32, u64, u32, u32, u64, u32, vp]
    fn.restype = ctypes.c_int
    oracle.orc_blind_rotate_mb.argtypes = [vp, vp, vp, u32, vp, vp, u32, u32, vp, ctypes.c_int]
    p = pkg.preset_params(preset)
    N, n, Q = p.N, p.n, p.Q
    keys = pkg.generate_keys_host(p, 31)
    K = 3 if mb == 2 else 8
    groups = -(-steps // mb)
    mbk = np.asarray(pkg.generate_mb_bsk_host(p, 31, mb)).reshape(-1, K, 2 * p.digits_g * 2 * N)[:groups]
    mbk = np.ascontiguousarray(mbk)
    oc = OracleCbs(oracle, p, keys)
    batch = 2
    rng = np.random.default_rng(12 + mb)
    a = rng.integers(0, p.q_lwe, size=(batch, n), dtype=np.uint64)
    b = rng.integers(0, p.q_lwe, batch, dtype=np.uint64)
    init = _orc_acc(oracle, oc, a, b, 0)
    want = _orc_acc(oracle, oc, a, b, steps, mbk=mbk, mb=mb)
    tabs, ninv, dmod = _tables(pkg, N, Q)
    monic = _monic(oracle, oc, N, Q)
    ek = np.ascontiguousarray(mbk.transpose(1, 0, 2)).reshape(-1)  # [subset][group][...]
    eks = np.zeros_like(ek)
    ref.ref_cirbts_shoup(ek.ctypes.data, eks.ctypes.data, ek.size, Q)
    bitwidth = max(0, (p.num_lut - 1).bit_length())
    dev = {name: _dev(v) for name, v in [("acc", init), ("a", a), ("ek", ek), ("eks", eks), ("monic", monic),
                                         ("mod", dmod), ("tw", tabs[0]), ("tws", tabs[1]), ("itw", tabs[2]),
                                         ("itws", tabs[3]), ("ninv", ninv)]}
    st = fn(dev["acc"].data_ptr(), dev["a"].data_ptr(), n, steps, batch, dev["ek"].data_ptr(), dev["eks"].data_ptr(),
            dev["monic"].data_ptr(), dev["mod"].data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(),
            dev["itw"].data_ptr(), dev["itws"].data_ptr(), dev["ninv"].data_ptr(), dev["ninv"].data_ptr() + 8, N, Q,
            p.base_g, p.digits_g, p.q_lwe, bitwidth, None)
    torch.cuda.synchronize()
    assert st == 0
    got = dev["acc"].cpu().numpy().view(np.uint64).reshape(batch, 2, N)
    assert not np.array_equal(got, init)
    assert np.array_equal(got, want)


def _mb3_soa_keys(mbk, p):
    """The grouped mb = 3 keys [groups][7][2 digits][2][N] re-laid as the reference's 7 SoA subset
    keys [groups][N/32 tiles][2 digits][2][32 lanes] (kernel_SwizzleRFKey, kernel.cu:2383-2404)."""
    groups = -(-p.n // 3)
    l2 = 2 * p.digits_g
    k = np.asarray(mbk).reshape(groups, 7, l2, 2, p.N // 32, 32)
    return [np.ascontiguousarray(k[:, s].transpose(0, 3, 1, 2, 4)).reshape(-1) for s in range(7)]


@pytest.mark.parametrize("preset", ["3x12", "2x18"])
def test_grouped_mb3_soa_matches_reference_kernels(pkg, oracle, ref, preset):
    """The reference's AES-default grouping (CIRBTS_PBS_MULTIBIT=3 with SoA keys and N-major
    index positions: kernel_EvalAccCore_Binary_MB3_Grouped_Batch_SoA_NMajor, kernel.cu:4585-4771,
    fused-NTT threads per block 384, EvalAcc block X 128) with the product's grouped mb = 3 keys
    reproduces the oracle's exact grouped accumulator word for word; the product's FFT mb = 3
    rotation is checked against that oracle within its phase-error bound (test_cbs_fft_gpu.py)."""
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    ref.ref_cirbts_index_nmajor.argtypes = [vp, u32, u32, u32, u32, u64, u32, vp, vp]
    ref.ref_cirbts_index_nmajor.restype = ctypes.c_int
    ref.ref_cirbts_blind_rotate_mb3_soa.argtypes = [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32, u64,
                                                    u32, u32, vp, u32, u32, vp, vp, vp]
    ref.ref_cirbts_blind_rotate_mb3_soa.restype = ctypes.c_int
    oracle.orc_blind_rotate_mb.argtypes = [vp, vp, vp, u32, vp, vp, u32, u32, vp, ctypes.c_int]
    p = pkg.preset_params(preset)
    N, n, Q = p.N, p.n, p.Q
    keys = pkg.generate_keys_host(p, 37)
    mbk = np.ascontiguousarray(pkg.generate_mb_bsk_host(p, 37, 3))
    oc = OracleCbs(oracle, p, keys)
    batch = 2
    rng = np.random.default_rng(14)
    a = rng.integers(0, p.q_lwe, size=(batch, n), dtype=np.uint64)
    b = rng.integers(0, p.q_lwe, batch, dtype=np.uint64)
    init = _orc_acc(oracle, oc, a, b, 0)
    want = _orc_acc(oracle, oc, a, b, n, mbk=mbk, mb=3)
    tabs, ninv, dmod = _tables(pkg, N, Q)
    monic = _monic(oracle, oc, N, Q)
    soa = _mb3_soa_keys(mbk, p)
    shoups = []
    for k in soa:
        ks = np.zeros_like(k)
        ref.ref_cirbts_shoup(k.ctypes.data, ks.ctypes.data, k.size, Q)
        shoups.append(ks)
    d_keys = [_dev(k) for k in soa]
    d_shoups = [_dev(k) for k in shoups]
    kp = (ctypes.c_void_p * 7)(*[t.data_ptr() for t in d_keys])
    ksp = (ctypes.c_void_p * 7)(*[t.data_ptr() for t in d_shoups])
    bitwidth = max(0, (p.num_lut - 1).bit_length())
    dev = {name: _dev(v) for name, v in [("acc", init), ("a", a), ("monic", monic), ("mod", dmod), ("tw", tabs[0]),
                                         ("tws", tabs[1]), ("itw", tabs[2]), ("itws", tabs[3]), ("ninv", ninv)]}
    idx = torch.zeros(n * batch, dtype=torch.int32, device="cuda")
    ct = torch.zeros(2 * batch * N, dtype=torch.int64, device="cuda")
    dct = torch.zeros(2 * p.digits_g * batch * N, dtype=torch.int64, device="cuda")
    assert ref.ref_cirbts_index_nmajor(dev["a"].data_ptr(), n, n, batch, N, p.q_lwe, bitwidth, idx.data_ptr(),
                                       None) == 0
    st = ref.ref_cirbts_blind_rotate_mb3_soa(
        dev["acc"].data_ptr(), n, batch, kp, ksp, dev["monic"].data_ptr(), dev["mod"].data_ptr(), dev["tw"].data_ptr(),
        dev["tws"].data_ptr(), dev["itw"].data_ptr(), dev["itws"].data_ptr(), dev["ninv"].data_ptr(),
        dev["ninv"].data_ptr() + 8, N, Q, p.base_g, p.digits_g, idx.data_ptr(), 384, 128, ct.data_ptr(),
        dct.data_ptr(), None)
    torch.cuda.synchronize()
    assert st == 0
    got = dev["acc"].cpu().numpy().view(np.uint64).reshape(batch, 2, N)
    assert not np.array_equal(got, init)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("num_auto,window", [(10, 0), (1, 0), (10, 32)])
def test_lmkcdey_eval_acc_matches_reference_kernels(pkg, oracle, ref, num_auto, window):
    """LMKCDEY_EvalAcc in the reference's launch sequence over its own kernels, with the
    product's LMKCDEY keys and maps, reproduces the oracle's accumulator word for word (the
    product's kernel equals the oracle: tests/test_lmkcdey_gpu.py)."""
    from cbs_harness import oracle_lmkcdey_keys
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    ref.ref_cirbts_lmkcdey_eval_acc.argtypes = [vp, vp, u32, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, u32,
                                                u64, u32, u32, vp]
    ref.ref_cirbts_lmkcdey_eval_acc.restype = ctypes.c_int
    oracle.orc_lmkcdey_eval_acc.argtypes = [vp, vp, vp, vp, u32, u32, vp, u32, vp]
    p = pkg.preset_params("2x18")
    p.num_lut = 1
    N, n, Q = p.N, p.n, p.Q
    keys = pkg.generate_keys_host(p, 61)
    lmk = oracle_lmkcdey_keys(oracle, p, keys, num_auto, 61, window)
    oc = OracleCbs(oracle, p, keys)
    tabs, ninv, dmod = _tables(pkg, N, Q)
    rng = np.random.default_rng(num_auto + 5)
    dev = {name: _dev(v) for name, v in [("eval", lmk["eval"]), ("auto", lmk["auto"]), ("mod", dmod),
                                         ("tw", tabs[0]), ("tws", tabs[1]), ("itw", tabs[2]), ("itws", tabs[3]),
                                         ("ninv", ninv)]}
    d_maps = torch.from_numpy(lmk["maps"].view(np.int32)).cuda()
    for trial in range(2):
        acc = rng.integers(0, Q, size=(2, N), dtype=np.uint64)
        a_neg = np.ascontiguousarray(rng.integers(0, 2 * N, size=n, dtype=np.uint32))
        want = acc.copy()
        oracle.orc_lmkcdey_eval_acc(ctypes.byref(oc.op), lmk["eval"].ctypes.data, lmk["auto"].ctypes.data,
                                    lmk["maps"].ctypes.data, num_auto, window, a_neg.ctypes.data, n,
                                    want.ctypes.data)
        d_acc = _dev(acc)
        st = ref.ref_cirbts_lmkcdey_eval_acc(
            d_acc.data_ptr(), a_neg.ctypes.data, n, dev["eval"].data_ptr(), dev["auto"].data_ptr(), d_maps.data_ptr(),
            num_auto, window, dev["mod"].data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(), dev["itw"].data_ptr(),
            dev["itws"].data_ptr(), dev["ninv"].data_ptr(), dev["ninv"].data_ptr() + 8, N, Q, p.base_g, p.digits_g,
            None)
        torch.cuda.synchronize()
        assert st == 0
        got = d_acc.cpu().numpy().view(np.uint64).reshape(2, N)
        assert not np.array_equal(got, acc)
        assert np.array_equal(got, want), trial
