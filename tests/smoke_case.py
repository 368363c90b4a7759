"""The smoke case run by __graft_entry__.smoke(): small slices of the hot path on cuda:0
through the C ABI, checked against the CPU oracle: the NTT bit-exactly, the grouped FFT
blind rotation within its FP64 phase-error bound, the FFT HomTrace / SchemeSwitch rows by
decryption."""
from __future__ import annotations


def run_smoke(pkg, torch, np) -> None:
    from conftest import load_oracle, oracle_primes, oracle_tables

    assert torch.cuda.is_available(), "smoke() needs cuda:0"
    torch.cuda.set_device(0)
    lib = pkg.load()
    oracle = load_oracle()

    # forward + inverse Phantom NTT at the CBS ring size
    n = 2048
    q = oracle_primes(oracle, n, 54, 1)[0]
    rp, rps, irp, irps, ninv = oracle_tables(oracle, n, q)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()  # noqa: E731
    d_rp, d_rps, d_irp, d_irps = dev(rp), dev(rps), dev(irp), dev(irps)
    d_ni, d_nis = dev(ninv[:1].copy()), dev(ninv[1:].copy())
    d_mod = dev(np.array([q, 0, 0], np.uint64))
    rng = np.random.default_rng(0)
    a = rng.integers(0, q, size=(4, n), dtype=np.uint64)
    x = dev(a.copy())
    pkg.call("cbs_fnwt_1d_opt_batched", x.data_ptr(), d_rp.data_ptr(), d_rps.data_ptr(), d_mod.data_ptr(), n, 4, None)
    torch.cuda.synchronize()
    want = a.copy()
    oracle.orc_ntt_forward(want, 4, n, q, rp)
    got = x.cpu().numpy().view(np.uint64)
    assert (got == want).all(), "forward NTT mismatch vs oracle"
    pkg.call("cbs_inwt_1d_opt_batched", x.data_ptr(), d_irp.data_ptr(), d_irps.data_ptr(), d_mod.data_ptr(),
             d_ni.data_ptr(), d_nis.data_ptr(), n, 4, None)
    torch.cuda.synchronize()
    assert (x.cpu().numpy().view(np.uint64) == a).all(), "inverse NTT mismatch"
    print("smoke: NTT N=2048 bit-exact vs oracle")

    # the FFT circuit-bootstrapping path on a small ring (N = 1024, n = 64): grouped (mb = 2)
    # blind rotation against the oracle's exact grouped rotation, then HomTrace +
    # SchemeSwitch in FFT form through the CBS entry point, rows checked by decryption
    import ctypes

    from cbs_harness import OracleCbs, lwe_encrypt_bits
    p = pkg.default_params()
    p.N, p.n = 1024, 64
    p.Q = oracle_primes(oracle, 1024, 54, 1)[0]
    ctx = pkg.Context(p, max_batch=4)
    try:
        ctx.keygen(7)
        ctx.set_br_backend(pkg.BR_FFT64)
        ctx.set_br_multibit(2)
        keys = ctx.export_keys()
        oc = OracleCbs(oracle, p, keys)
        bits = [1, 0]
        a, b = lwe_encrypt_bits(np.random.default_rng(1), keys["s_lwe"], bits, p.q_lwe)
        da, db = dev(a), dev(b)
        mv = torch.zeros((len(bits), p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
        pkg.call("cbs_blind_rotate_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), len(bits), p.n,
                 mv.data_ptr(), None)
        torch.cuda.synchronize()
        got = mv.cpu().numpy().view(np.uint64)
        want = oc.br_acc_mb(a, b, ctx.export_mb_bsk(), 2)
        Q, N = p.Q, p.N
        worst = 0
        for i in range(len(bits)):
            d = oc.phase_coef(got[i, 0]) - oc.phase_coef(want[i])
            worst = max(worst, max(abs(((int(x) * N + Q // 2) % Q) - Q // 2) for x in d))
        assert worst < 2 ** 33, f"grouped FFT blind rotation phase error 2^{np.log2(worst + 1):.1f}"
        print(f"smoke: grouped FFT blind rotation within 2^{np.log2(worst + 1):.1f} of the exact oracle")

        view = ctypes.c_void_p()
        pkg.call("cbs_circuit_bootstrap_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), len(bits), p.n,
                 ctypes.byref(view), None)
        torch.cuda.synchronize()
        per = p.num_lut * 4 * p.N
        rg = np.zeros(len(bits) * per, np.uint64)
        cudart = ctypes.CDLL("libcudart.so.12")
        cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        assert cudart.cudaMemcpy(rg.ctypes.data, view.value, rg.nbytes, 2) == 0  # device to host
        rg = rg.reshape(len(bits), p.num_lut, 2, 2, p.N)
        g = [int(x) for x in keys["gpow"]]
        s = keys["s_rlwe"].astype(object)
        for i, m in enumerate(bits):
            for j in range(p.num_lut):
                ph1 = oc.phase_coef(rg[i, j, 1])
                ph1[0] -= m * g[j]
                ph0 = oc.phase_coef(rg[i, j, 0]) + m * g[j] * s
                assert max(abs(int(x)) for x in ph1) < 2 ** 33 and max(abs(int(x)) for x in ph0) < 2 ** 37
        print("smoke: FFT HomTrace + SchemeSwitch rows decrypt to m g_j / -m g_j s")

        # the exact split-FFT blind rotation (key limbs whose FP64 products round exactly):
        # one-bit and grouped mb = 2, each equal word for word to the oracle's exact rotation
        ctx.set_br_backend(pkg.BR_FFT64_SPLIT)
        for mb in (1, 2):
            ctx.set_br_multibit(mb)
            mv.zero_()
            pkg.call("cbs_blind_rotate_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), len(bits), p.n,
                     mv.data_ptr(), None)
            torch.cuda.synchronize()
            got = mv.cpu().numpy().view(np.uint64)
            if mb == 1:
                assert np.array_equal(got, oc.br_mv(a, b)), "split FFT blind rotation differs from the oracle"
            else:
                want = oc.br_acc_mb(a, b, ctx.export_mb_bsk(), 2)
                assert np.array_equal(got[:, 0], want), "grouped split FFT blind rotation differs from the oracle"
        print("smoke: exact split-FFT blind rotation (one-bit and mb = 2) equal to the oracle word for word")
    finally:
        ctx.close()

    # split-FP32 gate bootstrap (torus 32, N = 1024, n = 64): FP32 transforms with the keys
    # split into a 24-bit and an exact 8-bit limb; the extracted LWE's noise stays within the
    # FP32 bound of the exact FP64 path's, and every bit decrypts
    gp = pkg.gate_default_params()
    gp.n = 64
    g = pkg.GateContext(gp, max_batch=8)
    try:
        g.keygen(5)
        gk = g.export_keys()
        gbits = np.array([1, 0, 0, 1, 1, 0, 1, 0], np.uint8)
        ga, gb = g.encrypt(gbits, seed=6)
        z = gk["z_rlwe"].astype(np.int64)
        want = np.where(gbits == 1, 1 << 29, -(1 << 29))
        noise = {}
        for mode in ("fp64", "fp32-split"):
            g.set_fft_mode(mode)
            dga = torch.from_numpy(ga.view(np.int32)).cuda()
            dgb = torch.from_numpy(gb.view(np.int32)).cuda()
            ext = torch.zeros((len(gbits), gp.N + 1), dtype=torch.int32, device="cuda")
            oa = torch.zeros((len(gbits), gp.n), dtype=torch.int32, device="cuda")
            ob = torch.zeros(len(gbits), dtype=torch.int32, device="cuda")
            pkg.call("cbs_gate_bootstrap_batch_device", g.handle, dga.data_ptr(), dgb.data_ptr(), len(gbits),
                     ext.data_ptr(), oa.data_ptr(), ob.data_ptr(), None)
            torch.cuda.synchronize()
            e = ext.cpu().numpy().view(np.uint32).astype(np.int64)
            ph = (e[:, gp.N] - e[:, : gp.N] @ z - want) % (1 << 32)
            noise[mode] = int(np.abs(np.where(ph >= 1 << 31, ph - (1 << 32), ph)).max())
            got = g.decrypt(oa.cpu().numpy().view(np.uint32), ob.cpu().numpy().view(np.uint32))
            assert np.array_equal(got, gbits), f"{mode} gate bootstrap decrypts wrong"
        g.set_fft_mode("fp64")
        assert noise["fp32-split"] < 2 ** 27, f"split-FP32 output noise 2^{np.log2(noise['fp32-split']):.1f}"
        print(f"smoke: split-FP32 gate bootstrap decrypts; output noise max 2^{np.log2(noise['fp32-split']):.1f} "
              f"(FP64 2^{np.log2(noise['fp64']):.1f})")
    finally:
        g.close()
