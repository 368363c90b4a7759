"""Timing beside the reference's own GPU kernels on the same B200: the reference's one-bit and
grouped (mb = 2) blind rotations (bitwise/src/cirbts/kernel.cu + Phantom's ntt_1d.cu, rebuilt
for sm_100a by `make -C oracle ref_gpu_cirbts`, launched in the reference's per-step sequences by
ref_gpu_cirbts_shim.cu) against the product's blind rotation (cbs_blind_rotate_batch_device,
exact-NTT and FP64-FFT backends, one-bit and grouped) at the same batch, N = 2048, n = 630.
Also the 2-D NTT and the sample extract + key switch beside the reference's kernels.  Prints
the times; asserts only that the runs complete (and, where both write comparable outputs, that
they agree).  The reference's blind-rotation timing covers its kernels only (no finalize / MV
split, which the product's includes).

    python -m pytest tests/test_ref_timing_gpu.py -m gpu -s
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import pytest

from conftest import ORACLE_DIR

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
REF_SO = ORACLE_DIR / "_ref" / "libref_cirbts.so"
BATCH = 1184  # 8 waves of the one-CTA-per-SM grouped kernel


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _time_ms(fn, reps=2):
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def test_blind_rotation_timing_beside_reference_kernels(pkg):
    if not REF_SO.exists():
        pytest.skip("reference CirBTS kernels not built (make -C oracle ref_gpu_cirbts)")
    ref = ctypes.CDLL(str(REF_SO))
    vp, u32, u64, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
    argt = [vp, vp, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32, u64, u32, u32, u64, u32, vp]
    for f in (ref.ref_cirbts_blind_rotate_steps, ref.ref_cirbts_blind_rotate_mb2):
        f.argtypes = argt
        f.restype = ctypes.c_int
    ref.ref_cirbts_shoup.argtypes = [vp, vp, sz, u64]

    ctx = pkg.Context(max_batch=BATCH)
    ctx.keygen(41)
    p = ctx.params
    N, n, Q = p.N, p.n, p.Q
    keys = ctx.export_keys()
    rng = np.random.default_rng(3)
    a = rng.integers(0, p.q_lwe, size=(BATCH, n), dtype=np.uint64)
    b = rng.integers(0, p.q_lwe, BATCH, dtype=np.uint64)
    da, db = _dev(a), _dev(b)
    mv = torch.empty((BATCH, p.num_lut, 2, N), dtype=torch.int64, device="cuda")
    results = {}

    def ours():
        pkg.call("cbs_blind_rotate_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), BATCH, n, mv.data_ptr(),
                 None)

    for name, backend, mb in [("product exact NTT, one-bit", pkg.BR_NTT, 1),
                              ("product FP64 FFT, one-bit", pkg.BR_FFT64, 1),
                              ("product FP64 FFT, mb = 2", pkg.BR_FFT64, 2)]:
        ctx.set_br_backend(backend)
        ctx.set_br_multibit(mb)
        results[name] = _time_ms(ours)
    mbk = ctx.export_mb_bsk()
    ctx.set_br_backend(pkg.BR_NTT)

    # the reference's kernels: tables, monomials NTT(X^k - 1), keys with Shoup tables
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
    d_monic = _dev(monic)
    dev = {nm: _dev(v) for nm, v in [("tw", tabs[0]), ("tws", tabs[1]), ("itw", tabs[2]), ("itws", tabs[3]),
                                     ("ninv", ninv),
                                     ("mod", np.array([dm.value, dm.const_ratio[0], dm.const_ratio[1]], np.uint64))]}
    pkg.call("cbs_fnwt_1d_opt_batched", d_monic.data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(),
             dev["mod"].data_ptr(), N, 2 * N, None)
    bitwidth = max(0, (p.num_lut - 1).bit_length())
    acc = torch.from_numpy(rng.integers(0, Q, size=(BATCH, 2, N), dtype=np.uint64).view(np.int64)).cuda()
    groups = (n + 1) // 2
    for name, fn, key in [("reference kernels, one-bit", ref.ref_cirbts_blind_rotate_steps,
                           np.ascontiguousarray(keys["bsk"]).reshape(-1)),
                          ("reference kernels, mb = 2", ref.ref_cirbts_blind_rotate_mb2,
                           np.ascontiguousarray(mbk.reshape(groups, 3, -1).transpose(1, 0, 2)).reshape(-1))]:
        ks = np.zeros_like(key)
        ref.ref_cirbts_shoup(key.ctypes.data, ks.ctypes.data, key.size, Q)
        d_k, d_ks = _dev(key), _dev(ks)

        def run():
            st = fn(acc.data_ptr(), da.data_ptr(), n, n, BATCH, d_k.data_ptr(), d_ks.data_ptr(), d_monic.data_ptr(),
                    dev["mod"].data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(), dev["itw"].data_ptr(),
                    dev["itws"].data_ptr(), dev["ninv"].data_ptr(), dev["ninv"].data_ptr() + 8, N, Q, p.base_g,
                    p.digits_g, p.q_lwe, bitwidth, None)
            assert st == 0

        results[name] = _time_ms(run, reps=1)
        del d_k, d_ks
    ctx.close()
    print(f"\nblind rotation, N = {N}, n = {n}, batch {BATCH}, one B200 (us per bootstrap):")
    for name, ms in results.items():
        print(f"  {name:32s} {ms * 1e3 / BATCH:9.1f}")
    assert all(v > 0 for v in results.values())


def test_rns_ntt_timing_beside_reference_kernels(pkg):
    """The Phantom-core 2-D NTT (N = 2^16, 32 ciphertexts x 2 polys x 24 limbs, forward +
    inverse, in place) against the reference's nwt_2d_radix8_forward/backward_inplace
    (src/ntt/fntt_2d.cu, intt_2d.cu, rebuilt by `make -C oracle ref_gpu`, one call per
    polynomial as the reference's API takes them); both round trips must give the input back."""
    so = ORACLE_DIR / "_ref" / "libref_phantom_ntt.so"
    if not so.exists():
        pytest.skip("reference Phantom NTT library not built (make -C oracle ref_gpu)")
    lib = ctypes.CDLL(str(so))
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    lib.ref_gpu_ntt2d_create.argtypes = [u32, u32, vp]
    lib.ref_gpu_ntt2d_create.restype = vp
    lib.ref_gpu_ntt2d_forward.argtypes = [vp, vp, u32, u32, vp]
    lib.ref_gpu_ntt2d_backward.argtypes = [vp, vp, u32, u32, vp]
    lib.ref_gpu_ntt2d_destroy.argtypes = [vp]
    logn, size_q, polys = 16, 24, 64
    n = 1 << logn
    q = np.zeros(size_q + 2, np.uint64)
    pkg.call("cbs_get_primes", n, 50, size_q + 2, q.ctypes.data)  # as bench.py rns_chain
    ctx = pkg.RnsContext(n, q[:size_q], q[size_q:])
    x = torch.remainder(torch.randint(0, 2 ** 62, (polys, size_q, n), dtype=torch.int64, device="cuda"),
                        torch.from_numpy(q[:size_q].view(np.int64)).cuda().view(1, -1, 1)).contiguous()
    orig = x.clone()
    y = x.clone()

    def ours():
        pkg.call("cbs_rns_ntt_batched", ctx.handle, x.data_ptr(), polys, size_q * n, size_q, 0, 0, None)
        pkg.call("cbs_rns_ntt_batched", ctx.handle, x.data_ptr(), polys, size_q * n, size_q, 0, 1, None)

    table = lib.ref_gpu_ntt2d_create(logn, len(q), q.ctypes.data)

    def theirs():
        for k in range(polys):
            lib.ref_gpu_ntt2d_forward(table, y.data_ptr() + k * size_q * n * 8, size_q, 0, None)
        for k in range(polys):
            lib.ref_gpu_ntt2d_backward(table, y.data_ptr() + k * size_q * n * 8, size_q, 0, None)

    t_ours, t_ref = _time_ms(ours, reps=3), _time_ms(theirs, reps=3)
    lib.ref_gpu_ntt2d_destroy(table)
    ctx.close()
    print(f"\n2-D NTT N = 2^16, {polys} polys x {size_q} limbs, forward + inverse: product {t_ours:.2f} ms, "
          f"reference kernels {t_ref:.2f} ms ({t_ref / t_ours:.2f}x)")
    assert torch.equal(x, orig) and torch.equal(y, orig)


def test_extraction_timing_beside_reference_kernel(pkg):
    """Sample extract + LWE key switch of one AES round's 16384 bits (128 blocks) from 512
    coefficient-domain words: the product's k_extract_keyswitch against the reference's
    kernel_SampleExtractKeySwitchToLWE (aes_gpu_ks.cuh, `make -C oracle ref_gpu_extract`).  The
    reference's timed call includes its workspace allocation, as its helper makes it."""
    so = ORACLE_DIR / "_ref" / "libref_extract.so"
    if not so.exists():
        pytest.skip("reference extraction kernel not built (make -C oracle ref_gpu_extract)")
    lib = ctypes.CDLL(str(so))
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    lib.ref_gpu_extract_keyswitch.argtypes = [vp, u32, u32, u32, u32, vp, vp, vp, u32, u64, u64, vp, vp, u32,
                                              ctypes.c_int]
    lib.ref_gpu_extract_keyswitch.restype = ctypes.c_int
    ctx = pkg.Context(max_batch=16384)
    ctx.keygen(43)
    p = ctx.params
    N, n = p.N, p.n
    ksk = np.ascontiguousarray(ctx.export_keys()["ksk"]).reshape(-1)
    rng = np.random.default_rng(5)
    W, count = 512, 16384
    words = rng.integers(0, p.Q, size=(W, 2, N), dtype=np.uint64)
    info = ((np.arange(count, dtype=np.uint32) // 32) << 16 | rng.integers(0, 32, count, dtype=np.uint32))
    info = info.astype(np.uint32)
    d_words = _dev(words)
    oa = torch.zeros((count, n), dtype=torch.int64, device="cuda")
    ob = torch.zeros(count, dtype=torch.int64, device="cuda")
    d_ksk = torch.from_numpy(ksk.view(np.int16)).cuda()
    d_a, d_b = _dev(words[:, 0, :]), _dev(words[:, 1, :])
    d_info = torch.from_numpy(info.view(np.int32)).cuda()
    ra = torch.zeros_like(oa)
    rb = torch.zeros_like(ob)

    def ours():
        pkg.call("cbs_extract_keyswitch_device", ctx.handle, d_words.data_ptr(), W, info.ctypes.data, count,
                 oa.data_ptr(), ob.data_ptr(), n, None)

    def theirs():
        assert lib.ref_gpu_extract_keyswitch(d_ksk.data_ptr(), n, N, p.base_ks, p.qks, d_a.data_ptr(), d_b.data_ptr(),
                                             d_info.data_ptr(), count, p.Q, p.q_lwe, ra.data_ptr(), rb.data_ptr(), n,
                                             0) == 0

    t_ours, t_ref = _time_ms(ours, reps=3), _time_ms(theirs, reps=3)
    ctx.close()
    print(f"\nextract + key switch, {count} bits, N = {N}, n = {n}: product {t_ours:.2f} ms, "
          f"reference kernel {t_ref:.2f} ms ({t_ref / t_ours:.2f}x)")
    assert torch.equal(oa, ra) and torch.equal(ob, rb)


def test_trace_schemeswitch_timing_beside_reference_kernels(pkg):
    """HomTrace + SchemeSwitch of 2048 MV RLWEs (N = 2048, 11 rounds, HT 2^9 x 5, SS 2^9 x 5):
    the product's exact-NTT and FFT forms (cbs_trace_schemeswitch_device) against the
    reference's default launch sequence (ref_gpu_cirbts_shim.cu; its call includes its buffer
    allocation).  The exact form and the reference must agree word for word."""
    if not REF_SO.exists():
        pytest.skip("reference CirBTS kernels not built (make -C oracle ref_gpu_cirbts)")
    ref = ctypes.CDLL(str(REF_SO))
    vp, u32, u64, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
    ref.ref_cirbts_trace_schemeswitch.argtypes = [vp, vp, u32, vp, vp, vp, vp, u32, u32, u32, u32, u32, vp, vp, vp,
                                                  vp, vp, vp, vp, vp, u32, u64, vp, vp]
    ref.ref_cirbts_trace_schemeswitch.restype = ctypes.c_int
    ref.ref_cirbts_shoup.argtypes = [vp, vp, sz, u64]
    count = 2048
    ctx = pkg.Context(max_batch=count)
    ctx.keygen(47)
    p = ctx.params
    N, Q = p.N, p.Q
    rounds = N.bit_length() - 1 - p.trace_shift
    keys = ctx.export_keys()
    mv = np.random.default_rng(6).integers(0, Q, size=(count, 2, N), dtype=np.uint64)
    d_mv = _dev(mv)
    rows = {name: torch.zeros((count, 2, 2, N), dtype=torch.int64, device="cuda") for name in ("ntt", "fft", "ref")}
    times = {}
    for name, backend in (("ntt", pkg.BR_NTT), ("fft", pkg.BR_FFT64)):
        ctx.set_br_backend(backend)
        times[name] = _time_ms(lambda: pkg.call("cbs_trace_schemeswitch_device", ctx.handle, d_mv.data_ptr(), count,
                                                rows[name].data_ptr(), None), reps=3)
    ctx.set_br_backend(pkg.BR_NTT)
    tabs = [np.zeros(N, np.uint64) for _ in range(4)]
    ninv = np.zeros(2, np.uint64)
    dm = pkg.DModulus()
    pkg.call("cbs_ntt_tables_host", N, Q, *(t.ctypes.data for t in tabs), ninv.ctypes.data, ctypes.addressof(dm))
    ht = np.ascontiguousarray(keys["ht"]).reshape(-1)
    ss = np.ascontiguousarray(keys["ss"]).reshape(-1)
    hts, sss = np.zeros_like(ht), np.zeros_like(ss)
    ref.ref_cirbts_shoup(ht.ctypes.data, hts.ctypes.data, ht.size, Q)
    ref.ref_cirbts_shoup(ss.ctypes.data, sss.ctypes.data, ss.size, Q)
    dev = {nm: _dev(v) for nm, v in [("c0", mv[:, 0, :]), ("c1", mv[:, 1, :]), ("ht", ht), ("hts", hts), ("ss", ss),
                                     ("sss", sss), ("tw", tabs[0]), ("tws", tabs[1]), ("itw", tabs[2]),
                                     ("itws", tabs[3]), ("ninv", ninv),
                                     ("mod", np.array([dm.value, dm.const_ratio[0], dm.const_ratio[1]], np.uint64))]}
    maps = torch.zeros((rounds, N), dtype=torch.int32, device="cuda")

    def theirs():
        assert ref.ref_cirbts_trace_schemeswitch(
            dev["c0"].data_ptr(), dev["c1"].data_ptr(), count, dev["ht"].data_ptr(), dev["hts"].data_ptr(),
            dev["ss"].data_ptr(), dev["sss"].data_ptr(), rounds, p.base_ht, p.digits_ht, p.base_ss, p.digits_ss,
            maps.data_ptr(), dev["mod"].data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(), dev["itw"].data_ptr(),
            dev["itws"].data_ptr(), dev["ninv"].data_ptr(), dev["ninv"].data_ptr() + 8, N, Q, rows["ref"].data_ptr(),
            None) == 0

    times["ref"] = _time_ms(theirs, reps=3)
    ctx.close()
    print(f"\nHomTrace + SchemeSwitch, {count} MV RLWEs, N = {N} (us per RLWE): product exact NTT "
          f"{times['ntt'] * 1e3 / count:.2f}, product FP64 FFT {times['fft'] * 1e3 / count:.2f}, "
          f"reference kernels {times['ref'] * 1e3 / count:.2f}")
    assert torch.equal(rows["ntt"], rows["ref"])


@pytest.mark.parametrize("preset", ["3x12", "2x18"])
def test_blind_rotation_timing_beside_reference_aes_default(pkg, preset):
    """The reference's fastest shipped blind-rotation configuration for its AES example
    (examples/aes_transcipher/main.cu:107-136: CIRBTS_PBS_MULTIBIT=3, SoA keys, N-major index
    positions, EvalAcc block X 128, fused-NTT threads per block 384;
    kernel_EvalAccCore_Binary_MB3_Grouped_Batch_SoA_NMajor, kernel.cu:4585) beside the product's
    blind rotation (FP64 FFT, mb = 2, the tuned default schedule, and mb = 3) on the same
    parameter set and batch.  The reference's scratch and index positions are prepared outside
    the timed region (its own driver allocates inside every call); best of 3 repeats each.  The
    fused INTT + decomposition kernel for one-digit gadgets (kernel.cu:561, AES2048_D1) does not
    apply to these two- and three-digit gadgets."""
    if not REF_SO.exists():
        pytest.skip("reference CirBTS kernels not built (make -C oracle ref_gpu_cirbts)")
    from test_ref_cirbts_gpu import _mb3_soa_keys
    ref = ctypes.CDLL(str(REF_SO))
    vp, u32, u64, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
    ref.ref_cirbts_shoup.argtypes = [vp, vp, sz, u64]
    ref.ref_cirbts_index_nmajor.argtypes = [vp, u32, u32, u32, u32, u64, u32, vp, vp]
    ref.ref_cirbts_index_nmajor.restype = ctypes.c_int
    ref.ref_cirbts_blind_rotate_mb3_soa.argtypes = [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32, u64,
                                                    u32, u32, vp, u32, u32, vp, vp, vp]
    ref.ref_cirbts_blind_rotate_mb3_soa.restype = ctypes.c_int

    p = pkg.preset_params(preset)
    ctx = pkg.Context(params=p, max_batch=BATCH)
    ctx.keygen(43)
    N, n, Q = p.N, p.n, p.Q
    rng = np.random.default_rng(5)
    a = rng.integers(0, p.q_lwe, size=(BATCH, n), dtype=np.uint64)
    b = rng.integers(0, p.q_lwe, BATCH, dtype=np.uint64)
    da, db = _dev(a), _dev(b)
    mv = torch.empty((BATCH, p.num_lut, 2, N), dtype=torch.int64, device="cuda")
    results = {}

    def ours():
        pkg.call("cbs_blind_rotate_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), BATCH, n, mv.data_ptr(),
                 None)

    ctx.set_br_backend(pkg.BR_FFT64)
    for name, mb in [("product FP64 FFT, mb = 2", 2), ("product FP64 FFT, mb = 4 (staged)", 4),
                     ("product FP64 FFT, mb = 3", 3)]:
        ctx.set_br_multibit(mb)
        results[name] = _time_ms(ours, reps=3)
    mbk = ctx.export_mb_bsk()  # mb = 3 keys
    soa = _mb3_soa_keys(mbk, p)
    del mbk
    d_keys, d_shoups = [], []
    for k in soa:
        ks = np.zeros_like(k)
        ref.ref_cirbts_shoup(k.ctypes.data, ks.ctypes.data, k.size, Q)
        d_keys.append(_dev(k))
        d_shoups.append(_dev(ks))
    kp = (ctypes.c_void_p * 7)(*[t.data_ptr() for t in d_keys])
    ksp = (ctypes.c_void_p * 7)(*[t.data_ptr() for t in d_shoups])
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
    d_monic = _dev(monic)
    dev = {nm: _dev(v) for nm, v in [("tw", tabs[0]), ("tws", tabs[1]), ("itw", tabs[2]), ("itws", tabs[3]),
                                     ("ninv", ninv),
                                     ("mod", np.array([dm.value, dm.const_ratio[0], dm.const_ratio[1]], np.uint64))]}
    pkg.call("cbs_fnwt_1d_opt_batched", d_monic.data_ptr(), dev["tw"].data_ptr(), dev["tws"].data_ptr(),
             dev["mod"].data_ptr(), N, 2 * N, None)
    bitwidth = max(0, (p.num_lut - 1).bit_length())
    acc = torch.from_numpy(rng.integers(0, Q, size=(BATCH, 2, N), dtype=np.uint64).view(np.int64)).cuda()
    idx = torch.zeros(n * BATCH, dtype=torch.int32, device="cuda")
    ct = torch.zeros(2 * BATCH * N, dtype=torch.int64, device="cuda")
    dct = torch.zeros(2 * p.digits_g * BATCH * N, dtype=torch.int64, device="cuda")
    assert ref.ref_cirbts_index_nmajor(da.data_ptr(), n, n, BATCH, N, p.q_lwe, bitwidth, idx.data_ptr(), None) == 0

    def theirs():
        st = ref.ref_cirbts_blind_rotate_mb3_soa(
            acc.data_ptr(), n, BATCH, kp, ksp, d_monic.data_ptr(), dev["mod"].data_ptr(), dev["tw"].data_ptr(),
            dev["tws"].data_ptr(), dev["itw"].data_ptr(), dev["itws"].data_ptr(), dev["ninv"].data_ptr(),
            dev["ninv"].data_ptr() + 8, N, Q, p.base_g, p.digits_g, idx.data_ptr(), 384, 128, ct.data_ptr(),
            dct.data_ptr(), None)
        assert st == 0

    results["reference AES default (MB3 SoA N-major)"] = _time_ms(theirs, reps=3)
    ctx.close()
    print(f"\nblind rotation, {preset} gadget, N = {N}, n = {n}, batch {BATCH}, one B200 (us per bootstrap):")
    for name, ms in results.items():
        print(f"  {name:42s} {ms * 1e3 / BATCH:9.1f}")
    assert all(v > 0 for v in results.values())


def test_modup_moddown_timing_beside_reference_rns_tool(pkg):
    """The product's modup and moddown_from_NTT (cbs_rns_modup, cbs_rns_moddown_from_ntt) against
    the reference's DRNSTool::modup / moddown_from_NTT (include/rns.cuh:156-164, rebuilt by
    `make -C oracle ref_gpu_rns`, one call per ciphertext as the reference's key switch makes
    them) on the key-switching configuration N = 2^16, 24 + 2 primes, 32 ciphertexts; the
    outputs must agree word for word."""
    so = ORACLE_DIR / "_ref" / "libref_rns.so"
    if not so.exists():
        pytest.skip("reference Phantom RNS tool not built (make -C oracle ref_gpu_rns)")
    lib = ctypes.CDLL(str(so))
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    lib.ref_rns_create.argtypes = [u32, vp, u32, u32]
    lib.ref_rns_create.restype = vp
    lib.ref_rns_destroy.argtypes = [vp]
    lib.ref_rns_modup.argtypes = [vp, u32, vp, vp, u32, vp]
    lib.ref_rns_moddown_from_ntt.argtypes = [vp, u32, vp, vp, u32, vp]
    logn, size_q, size_p, count = 16, 24, 2, 32
    n = 1 << logn
    chain = np.zeros(size_q + size_p, np.uint64)
    pkg.call("cbs_get_primes", n, 50, size_q + size_p, chain.ctypes.data)
    q, p = chain[:size_q].copy(), chain[size_q:].copy()
    ctx = pkg.RnsContext(n, q, p)
    rctx = lib.ref_rns_create(logn, chain.ctypes.data, size_q, size_p)
    assert rctx
    try:
        beta, qlp = ctx.beta(size_q), size_q + size_p
        mods_q = torch.from_numpy(q.view(np.int64)).cuda().view(1, -1, 1)
        c2 = torch.remainder(torch.randint(0, 2 ** 62, (count, size_q, n), dtype=torch.int64, device="cuda"), mods_q)
        mine = torch.zeros((count, beta, qlp, n), dtype=torch.int64, device="cuda")
        theirs = torch.zeros_like(mine)
        t_up = _time_ms(lambda: pkg.call("cbs_rns_modup", ctx.handle, mine.data_ptr(), c2.data_ptr(), size_q, count,
                                         None), reps=3)
        r_up = _time_ms(lambda: lib.ref_rns_modup(rctx, size_q, theirs.data_ptr(), c2.data_ptr(), count, None), reps=3)
        assert torch.equal(mine, theirs)
        del mine, theirs
        polys = 2 * count
        mods_qp = torch.from_numpy(chain.view(np.int64)).cuda().view(1, -1, 1)
        cx = torch.remainder(torch.randint(0, 2 ** 62, (polys, qlp, n), dtype=torch.int64, device="cuda"), mods_qp)
        work = torch.empty_like(cx)
        out_m = torch.zeros((polys, size_q, n), dtype=torch.int64, device="cuda")
        out_t = torch.zeros_like(out_m)

        def fresh_ms(run, out):
            # both sides transform the P limbs of cx in place: each repeat starts from a fresh
            # copy (the copy and the clearing of the output are not timed)
            best = float("inf")
            for _ in range(4):
                work.copy_(cx)
                out.zero_()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                run()
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best

        t_dn = fresh_ms(lambda: pkg.call("cbs_rns_moddown_from_ntt", ctx.handle, out_m.data_ptr(), work.data_ptr(),
                                         size_q, polys, 0, None), out_m)
        r_dn = fresh_ms(lambda: lib.ref_rns_moddown_from_ntt(rctx, size_q, out_t.data_ptr(), work.data_ptr(), polys,
                                                             None), out_t)
        assert torch.equal(out_m, out_t)
    finally:
        lib.ref_rns_destroy(rctx)
        ctx.close()
    print(f"\nN = 2^16, {size_q} + {size_p} primes, {count} ciphertexts (modup) / {polys} polynomials (moddown):\n"
          f"  modup            product {t_up:7.2f} ms, reference DRNSTool {r_up:7.2f} ms ({r_up / t_up:.2f}x)\n"
          f"  moddown_from_NTT product {t_dn:7.2f} ms, reference DRNSTool {r_dn:7.2f} ms ({r_dn / t_dn:.2f}x)")


def test_lmkcdey_timing_beside_reference_kernels(pkg):
    """The LMKCDEY accumulator (EvalAcc; N = 2048, n = 630, 2^18 x 2 gadget with the first digit
    dropped, 10 automorphism keys): the product's k_lmkcdey, one CTA per ciphertext over a batch,
    against the reference's LMKCDEY_EvalAcc sequence over its own kernels, one ciphertext per call
    as the reference runs it (ref_gpu_cirbts_shim.cu; its call allocates its scratch and builds the
    buckets on the host).  Both start from the same accumulator and masks and must agree."""
    if not REF_SO.exists():
        pytest.skip("reference CirBTS kernels not built (make -C oracle ref_gpu_cirbts)")
    ref = ctypes.CDLL(str(REF_SO))
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    ref.ref_cirbts_lmkcdey_eval_acc.argtypes = [vp, vp, u32, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, u32,
                                                u64, u32, u32, vp]
    ref.ref_cirbts_lmkcdey_eval_acc.restype = ctypes.c_int
    num_auto, batch = 10, 1184
    p = pkg.preset_params("2x18")
    p.num_lut = 1
    N, n, Q = p.N, p.n, p.Q
    ctx = pkg.Context(params=p, max_batch=batch)
    try:
        ctx.keygen(71)
        ctx.set_br_method(pkg.BR_LMKCDEY, num_auto)
        ev, au = ctx.export_lmkcdey_keys()
        rng = np.random.default_rng(8)
        acc = rng.integers(0, Q, size=(batch, 2, N), dtype=np.uint64)
        a_neg = rng.integers(0, 2 * N, size=(batch, n), dtype=np.uint32)
        d_acc0 = _dev(acc)
        d_acc = d_acc0.clone()
        d_a = torch.from_numpy(a_neg.view(np.int32)).cuda()

        def ours():
            d_acc.copy_(d_acc0)
            pkg.call("cbs_lmkcdey_eval_acc_batch_device", ctx.handle, d_a.data_ptr(), n, d_acc.data_ptr(), batch, None)

        ms_ours = _time_ms(ours, reps=2)
        got = d_acc.cpu().numpy().view(np.uint64).reshape(batch, 2, N)
        # the whole bootstrapping rotation (bootstrap form, finalize and MV output), LMKCDEY and
        # the exact GINX one-bit form on the same parameters
        la = rng.integers(0, p.q_lwe, size=(batch, n), dtype=np.uint64)
        lb = rng.integers(0, p.q_lwe, batch, dtype=np.uint64)
        dla, dlb = _dev(la), _dev(lb)
        mv = torch.empty((batch, p.num_lut, 2, N), dtype=torch.int64, device="cuda")

        def rotate():
            pkg.call("cbs_blind_rotate_batch_device", ctx.handle, dla.data_ptr(), dlb.data_ptr(), batch, n,
                     mv.data_ptr(), None)

        ms_br_lmk = _time_ms(rotate, reps=2)
        ctx.set_br_method(pkg.BR_GINX, 0, 0)
        ms_br_ginx = _time_ms(rotate, reps=2)
        ctx.set_br_method(pkg.BR_LMKCDEY, num_auto)

        tabs = [np.zeros(N, np.uint64) for _ in range(4)]
        ninv = np.zeros(2, np.uint64)
        dm = pkg.DModulus()
        pkg.call("cbs_ntt_tables_host", N, Q, *(t.ctypes.data for t in tabs), ninv.ctypes.data, ctypes.addressof(dm))
        dmod = np.array([dm.value, dm.const_ratio[0], dm.const_ratio[1]], np.uint64)
        maps = pkg.lmkcdey_auto_maps_host(N, num_auto)
        dv = {nm: _dev(v) for nm, v in [("ev", ev), ("au", au), ("mod", dmod), ("tw", tabs[0]), ("tws", tabs[1]),
                                        ("itw", tabs[2]), ("itws", tabs[3]), ("ninv", ninv)]}
        d_maps = torch.from_numpy(maps.view(np.int32)).cuda()
        reps = 2
        r_acc = [_dev(acc[i]) for i in range(reps)]
        rows = [np.ascontiguousarray(a_neg[i]) for i in range(reps)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(reps):
            st = ref.ref_cirbts_lmkcdey_eval_acc(
                r_acc[i].data_ptr(), rows[i].ctypes.data, n, dv["ev"].data_ptr(), dv["au"].data_ptr(),
                d_maps.data_ptr(), num_auto, 0, dv["mod"].data_ptr(), dv["tw"].data_ptr(), dv["tws"].data_ptr(),
                dv["itw"].data_ptr(), dv["itws"].data_ptr(), dv["ninv"].data_ptr(), dv["ninv"].data_ptr() + 8, N, Q,
                p.base_g, p.digits_g, None)
            assert st == 0
        torch.cuda.synchronize()
        ms_ref = (time.perf_counter() - t0) * 1e3 / reps
        for i in range(reps):
            assert np.array_equal(r_acc[i].cpu().numpy().view(np.uint64).reshape(2, N), got[i]), i
    finally:
        ctx.close()
    print(f"\nLMKCDEY EvalAcc, 2x18, N = 2048, n = 630, 10 automorphism keys, one B200 (us per ciphertext):")
    print(f"  product k_lmkcdey, batch {batch:5d}          {ms_ours * 1e3 / batch:9.1f}")
    print(f"  reference kernels, one per call          {ms_ref * 1e3:9.1f}")
    print(f"whole blind rotation (finalize, MV output), same parameters, batch {batch} (us per ciphertext):")
    print(f"  product LMKCDEY                          {ms_br_lmk * 1e3 / batch:9.1f}")
    print(f"  product exact NTT GINX, one-bit          {ms_br_ginx * 1e3 / batch:9.1f}")
