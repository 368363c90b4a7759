"""Benchmark: homomorphic AES-128 CTR transciphering throughput (blocks/s) on B200.

Workload (AES-128 transciphering, batches of 16, 128 or 1024 blocks): `--blocks` random 128-bit
counter blocks per GPU (default 128; the configuration also names 16 and 1024), key =
128 uniform bits from a seed, full 10-round homomorphic AES via circuit bootstrapping
(blind rotation + HomTrace + SchemeSwitch), 16 CMux T-table LUTs per block-round and
sample extract + key switch, every round a captured CUDA graph.  One step = one batch.
The FP64-FFT backend runs the blind rotation over groups of 2 LWE coefficients by default
(--multibit 2: the reference's CIRBTS_PBS_MULTIBIT=2 key grouping); --multibit 1 is the
one-coefficient GINX loop.

value: blocks/s with inputs resident in HBM, CUDA events on the launching stream, max over
ranks.  e2e: the same metric through the host-buffer C-ABI entry point of the whole
transciphering job (cbs_aes128_ctr_transcipher_ciphertext: counters and a public AES-CTR
ciphertext in host memory, LWE encryptions of the plaintext bits copied back).  Every output
block is decrypted and compared after the timed region: the keystream with AES-128 from
OpenSSL, the e2e output with the plaintext.

--impl reference: the CPU restatement of the same path (oracle/, all host threads) on a
bounded sample of the same workload; rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "gpu-circuitbootstrapping-aestransciphering_b200"
METRICS = {"fft64": "AES-128 CTR transciphering blocks/s (1 B200, FP64-FFT circuit bootstrapping)",
           "ntt": "AES-128 CTR transciphering blocks/s (1 B200, exact-NTT circuit bootstrapping)",
           "fft64-split": "AES-128 CTR transciphering blocks/s (1 B200, exact split-FFT circuit bootstrapping)"}


def backend_id(pkg, name: str) -> int:
    return {"fft64": pkg.BR_FFT64, "ntt": pkg.BR_NTT, "fft64-split": pkg.BR_FFT64_SPLIT}[name]
UNIT = "blocks/s"
ROUNDS = 10


def load_pkg():
    spec = importlib.util.spec_from_file_location("cbs_b200", PKG_DIR / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cbs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_replicas():
    """The package's multi-GPU plumbing (replicas.py: CTR-stream sharding, max over ranks)."""
    spec = importlib.util.spec_from_file_location("cbs_b200_replicas", PKG_DIR / "replicas.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> dict:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.proc, self.lines = gpu, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def counter_bits(ctrs: np.ndarray) -> np.ndarray:
    """[blocks][16] bytes -> [blocks*128] bits, bit t = byte*8 + b."""
    return np.unpackbits(ctrs, axis=1, bitorder="little").reshape(-1).astype(np.uint8)


def aes_ecb(key: bytes, blocks: np.ndarray) -> np.ndarray:
    """AES-128 of each 16-byte row (OpenSSL through `cryptography`)."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes
    enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    return np.frombuffer(enc.update(blocks.tobytes()), np.uint8).reshape(blocks.shape[0], 16)


def verify(pkg, ctx, key: bytes, ctrs: np.ndarray, ha: np.ndarray, hb: np.ndarray,
           plain: np.ndarray | None = None) -> int:
    """Blocks whose decrypted LWE bits equal AES_K(counter), or `plain` when given."""
    n = ctx.params.n
    blocks = ctrs.shape[0]
    dec = np.zeros(blocks * 128, np.uint8)
    pkg.call("cbs_lwe_decrypt_bits", ctx.handle, ha.ctypes.data, hb.ctypes.data, blocks * 128, n, dec.ctypes.data)
    got = np.packbits(dec.reshape(blocks, 128), axis=1, bitorder="little")
    want = aes_ecb(key, ctrs) if plain is None else plain
    return int((got == want).all(axis=1).sum())


def output_noise(pkg, ctx, key: bytes, ctrs: np.ndarray, ha: np.ndarray, hb: np.ndarray) -> dict:
    """Phase error of the transciphered keystream bits (secret key exported for the measurement
    only): e = b - <a, s> - m q/2 (mod q, centred) against the true AES bit m; its rms sigma and the
    Gaussian tail at the decision margin q/4 give the failure probability of one bit decision
    (every extraction of every round has this noise: 1280 decisions per block)."""
    p = ctx.params
    s = np.zeros(p.n, np.int32)
    pkg.call("cbs_export_keys", ctx.handle, s.ctypes.data, None, None, None, None, None, None, None, None)
    q = int(p.q_lwe)
    dot = (ha[:, : p.n].astype(np.int64) @ s.astype(np.int64)) % q
    m = np.unpackbits(aes_ecb(key, ctrs), axis=1, bitorder="little").reshape(-1).astype(np.int64)
    e = (hb.astype(np.int64) - dot - m * (q // 2) + q // 2) % q - q // 2
    sigma = float(np.sqrt(np.mean(e.astype(np.float64) ** 2)))
    lp = pkg.log2_pfail_gaussian(sigma, q / 4)
    return {"bits": int(e.size), "sigma": sigma, "max_abs": int(np.abs(e).max()), "margin": q // 4,
            "p_fail_log2_per_bit": lp, "p_fail_log2_per_block": lp + float(np.log2(128 * ROUNDS)),
            "target_log2": -40.0,
            "method": "sigma = rms of the measured output-bit phase errors (keystream bits of the last step); "
                      "p = erfc(margin / (sqrt(2) sigma)) per bit decision, x 1280 decisions per block"}


def split_fft64_pair(pkg, torch, ctx, count: int = 2368, steps: int = 2) -> dict:
    """The exact split-FFT blind rotation (CBS_BR_FFT64_SPLIT: FP64 products of 18-bit key limbs,
    bit-identical to the exact NTT kernel) beside the approximate FP64 kernel on the AES
    context's keys, grouped mb = 2, `count` seeded random LWE ciphertexts, CUDA events; the
    context is left on the split backend (called after the AES legs)."""
    p = ctx.params
    rng = np.random.default_rng(11)
    a = torch.from_numpy(rng.integers(0, p.q_lwe, size=(count, p.n), dtype=np.int64)).cuda()
    b = torch.from_numpy(rng.integers(0, p.q_lwe, size=count, dtype=np.int64)).cuda()
    mv = torch.empty((count, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    fn = lambda: pkg.call("cbs_blind_rotate_batch_device", ctx.handle, a.data_ptr(), b.data_ptr(), count,  # noqa: E731
                          p.n, mv.data_ptr(), stream.cuda_stream)
    res = {"batch": count, "br_multibit": 2}
    for name, backend in (("fp64_approximate", pkg.BR_FFT64), ("split_exact", pkg.BR_FFT64_SPLIT)):
        pkg.call("cbs_context_set_br_backend", ctx.handle, backend)
        ctx.set_br_multibit(2)
        res[name] = {"us_per_bootstrap": _timed(torch, stream, fn, 1, steps) * 1e3 / count}
    res["limbs"] = dict(zip(("limbs", "limb_bits", "bound_bits"), pkg.split_fft_plan(p, 2)))
    res["ratio_split_over_fp64_time"] = res["split_exact"]["us_per_bootstrap"] / res["fp64_approximate"]["us_per_bootstrap"]
    res["note"] = ("AES on the exact split backend: bench.py --backend fft64-split --multibit 2 "
                   "(every output word equal to the exact NTT path's)")
    return res


def gate_split_pair(pkg, torch, count: int = 1184, steps: int = 3) -> dict:
    """The split-FP32 external product where it is built (torus-32 gate path, n = 636, N = 1024):
    NAND gates/s with split FP32 (one-bit) beside FP64 (grouped mb = 2, the FP64 default), same
    inputs, timed with CUDA events; every output gate checked."""
    ctx = pkg.GateContext(max_batch=count)
    ctx.keygen(7)
    p = ctx.params
    rng = np.random.default_rng(7)
    x = rng.integers(0, 2, count).astype(np.uint8)
    y = rng.integers(0, 2, count).astype(np.uint8)
    a1, b1 = ctx.encrypt(x, seed=8)
    a2, b2 = ctx.encrypt(y, seed=9)
    d = [torch.from_numpy(np.ascontiguousarray(v).view(np.int32)).cuda() for v in (a1, b1, a2, b2)]
    oa = torch.zeros((count, p.n), dtype=torch.int32, device="cuda")
    ob = torch.zeros(count, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    res = {}
    for name, mb, mode in (("fp64_mb2", 2, "fp64"), ("split_fp32", 1, "fp32-split")):
        ctx.set_fft_mode("fp64")
        ctx.set_multibit(mb)
        ctx.set_fft_mode(mode)
        fn = lambda: pkg.call("cbs_gate_eval_batch_device", ctx.handle, pkg.GATE_NAND,  # noqa: E731
                              *(t.data_ptr() for t in d), count, oa.data_ptr(), ob.data_ptr(), stream.cuda_stream)
        ms = _timed(torch, stream, fn, 2, steps)
        ok = int((ctx.decrypt(oa.cpu().numpy().view(np.uint32), ob.cpu().numpy().view(np.uint32))
                  == 1 - (x & y)).sum())
        res[name] = {"gates_per_s": count / (ms * 1e-3), "correct": ok, "of": count}
    ctx.close()
    res["ratio_split_over_fp64"] = res["split_fp32"]["gates_per_s"] / res["fp64_mb2"]["gates_per_s"]
    return res


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch

    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    blocks = args.blocks
    ctx = pkg.Context(params=pkg.preset_params(args.params), max_batch=128 * min(blocks, 256))
    ctx.keygen(args.seed)
    pkg.call("cbs_context_set_br_backend", ctx.handle, backend_id(pkg, args.backend))
    tuned = None
    if args.backend == "fft64" and args.tune:
        # the product's autotuner picks the grouping and schedule (16 waves of 148 ciphertexts)
        tuned = ctx.autotune(min(16 * 148, 128 * min(blocks, 256)))
        args.multibit, args.schedule = tuned["mb"], tuned["schedule"]
    else:
        if args.multibit > 1:
            ctx.set_br_multibit(args.multibit)
        ctx.set_br_schedule(args.schedule)
    key = np.random.default_rng(args.seed).bytes(16)
    pkg.call("cbs_aes128_setup", ctx.handle, key, args.seed + 1)
    p = ctx.params
    rep = load_replicas()
    ctrs = rep.rank_counters(args.seed, rank, world, blocks)  # this rank's share of one CTR stream
    d_bits = torch.from_numpy(counter_bits(ctrs)).cuda()
    out_a = torch.empty((blocks * 128, p.n), dtype=torch.int64, device="cuda")
    out_b = torch.empty(blocks * 128, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()  # a real stream: the per-round graphs are captured on it
    sptr = stream.cuda_stream

    def step():
        pkg.call("cbs_aes128_ctr_transcipher_device", ctx.handle, d_bits.data_ptr(), blocks, out_a.data_ptr(),
                 out_b.data_ptr(), 1, sptr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    rep.barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    rep.barrier(world)
    ms_max = rep.max_over_ranks(ev0.elapsed_time(ev1), world, device="cuda")
    ms_per_step = ms_max / args.steps

    # correctness of the last step's output and its noise
    ha = out_a.cpu().numpy().view(np.uint64).copy()
    hb = out_b.cpu().numpy().view(np.uint64).copy()
    ok = verify(pkg, ctx, key, ctrs, ha, hb)
    noise = output_noise(pkg, ctx, key, ctrs, ha, hb)

    # dominant kernel: the fused blind rotation over the whole batch, timed alone
    T = min(blocks, 256) * 128
    lwe_a = torch.from_numpy(ha[:T].view(np.int64)).cuda()
    lwe_b = torch.from_numpy(hb[:T].view(np.int64)).cuda()
    mv = torch.empty((T, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")

    def br():
        pkg.call("cbs_blind_rotate_batch_device", ctx.handle, lwe_a.data_ptr(), lwe_b.data_ptr(), T, p.n,
                 mv.data_ptr(), sptr)

    br()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 2
    e0.record(stream)
    for _ in range(reps):
        br()
    e1.record(stream)
    torch.cuda.synchronize()
    br_ms = e0.elapsed_time(e1) / reps
    N, n, l2, L = p.N, p.n, 2 * p.digits_g, p.num_lut
    alg_bytes = br_key_bytes(p, args.multibit) + T * ((n + 1) * 8 + L * 2 * N * 8)  # key once + LWE in + MV out
    traffic = BR_TRAFFIC.get((args.backend, args.params, args.multibit, T))

    # e2e through the host-buffer C-ABI entry point of the whole job: a public AES-CTR
    # ciphertext of seeded random plaintext in, LWE encryptions of the plaintext bits out
    plain = np.random.default_rng(args.seed + 1 + rank).integers(0, 256, (blocks, 16), dtype=np.uint8)
    cipher = np.ascontiguousarray(plain ^ aes_ecb(key, ctrs))
    out_ha = np.empty((blocks * 128, p.n), np.uint64)
    out_hb = np.empty(blocks * 128, np.uint64)
    e2e_steps = max(1, min(args.steps, 2))

    def e2e_call():
        pkg.call("cbs_aes128_ctr_transcipher_ciphertext", ctx.handle, ctrs.ctypes.data, cipher.ctypes.data, blocks,
                 out_ha.ctypes.data, out_hb.ctypes.data)

    e2e_call()
    rep.barrier(world)
    t0 = time.perf_counter()  # the host API call is synchronous: copies and kernels inside
    for _ in range(e2e_steps):
        e2e_call()
    e2e_ms = rep.max_over_ranks((time.perf_counter() - t0) / e2e_steps * 1e3, world, device="cuda")
    e2e_ok = verify(pkg, ctx, key, ctrs, out_ha, out_hb, plain)

    chunks = -(-blocks // 256)
    # per round: blind rotation, HomTrace+SchemeSwitch, 8 CMux levels, word assembly and
    # extraction (+ one inverse NTT of the words on the NTT backend); + state init per chunk
    # (the split backend adds one forward NTT of the MV outputs after its blind rotation)
    launches_per_step = chunks * (1 + ROUNDS * {"fft64": 12, "ntt": 13, "fft64-split": 14}[args.backend])
    result = {
        "metric": METRICS[args.backend],
        "value": rep.whole_job_rate(world, blocks, ms_per_step),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (blind-rotation FFT products) + u64 (exact mod-Q NTT elsewhere)" if args.backend == "fft64"
                 else "f64 (exact blind-rotation key-limb products) + u64 (exact mod-Q NTT elsewhere)"
                 if args.backend == "fft64-split"
                 else "u64 (exact mod-Q NTT arithmetic)",
        "data": "synthetic (seeded AES key; counters: one seeded CTR stream, rank r takes blocks [r B, (r+1) B))",
        "config": {"workload": "aes128_ctr_transcipher", "blocks_per_gpu": blocks, "global_blocks": world * blocks,
                   "params": f"N=2048 Q=54-bit n=630 q=2^14 BR 2^{p.base_g.bit_length() - 1}x{p.digits_g} RGSW 2^6x4 "
                             f"HT 2^9x5 SS 2^9x5 KS 2^14/2^7",
                   "param_set": args.params,
                   "l2": "per-step working set (keys + RGSW + LUT buffers) >> 126 MB L2",
                   "br_multibit": args.multibit,
                   "br_schedule": args.schedule,
                   "br_tuned": tuned,
                   "parallelism": f"replicas x{world} (independent blocks per GPU)"},
        "us_per_bootstrap": ms_per_step * 1e3 / (blocks * 128 * ROUNDS),
        "correct_blocks": ok,
        "gpu_launches": launches_per_step * args.steps,
        "e2e": {"value": rep.whole_job_rate(world, blocks, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": blocks * (128 + 16),
                "d2h_bytes_per_step": blocks * 128 * (p.n + 1) * 8, "correct_blocks": e2e_ok},
        "roofline": br_roofline(args, p, T, br_ms, alg_bytes, traffic),
        "p_fail": noise,
        "clocks": clk.summary(),
    }
    if args.backend == "fft64":
        result["split_fp32"] = {
            "aes_path": "not built: an exact FP32 limb of the 54-bit-Q external product holds at most 3 bits "
                        "under 12-bit digits (6 under 9-bit) at N = 2048, i.e. 18+ limbs with an inverse "
                        "transform and key spectra each against one FP64 product, and a whole-key FP32 product "
                        "misses by ~2^-7 of Q (tests/test_fp32_split_analysis.py)",
            "gate_path_measured": gate_split_pair(pkg, torch)}
        result["split_fft64"] = split_fft64_pair(pkg, torch, ctx)
    if rank == 0 and args.cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(result), flush=True)
    ctx.close()


def _timed(torch, stream, fn, warmup: int, steps: int) -> float:
    """Average device milliseconds of fn over `steps` launches on `stream` after `warmup`."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_blind_rotate(args, rank: int, world: int, local_rank: int) -> None:
    """Blind rotation alone (the dominant kernel) over `--batch` random LWE ciphertexts: the
    profiling case for the fused blind-rotation kernel."""
    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    T = args.batch or 2368
    params = pkg.preset_params(args.params)
    lmk = args.method == "lmkcdey"
    if lmk:  # one test-vector slot (LMKCDEY's odd masks), the exact NTT form
        params.num_lut = 1
        args.backend, args.multibit = "ntt", 1
    ctx = pkg.Context(params=params, max_batch=T)
    ctx.keygen(args.seed)
    pkg.call("cbs_context_set_br_backend", ctx.handle, backend_id(pkg, args.backend))
    if args.multibit > 1:
        ctx.set_br_multibit(args.multibit)
    ctx.set_br_schedule(args.schedule)
    if lmk:
        ctx.set_br_method(pkg.BR_LMKCDEY, 10, 0)
    p = ctx.params
    rng = np.random.default_rng(args.seed + rank)
    a = torch.from_numpy(rng.integers(0, p.q_lwe, size=(T, p.n), dtype=np.int64)).cuda()
    b = torch.from_numpy(rng.integers(0, p.q_lwe, size=T, dtype=np.int64)).cuda()
    mv = torch.empty((T, p.num_lut, 2, p.N), dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    fn = lambda: pkg.call("cbs_blind_rotate_batch_device", ctx.handle, a.data_ptr(), b.data_ptr(), T, p.n,  # noqa: E731
                          mv.data_ptr(), stream.cuda_stream)
    with ClockSampler(local_rank) as clk:
        ms = _timed(torch, stream, fn, args.warmup, args.steps)
    N, n, l2, L = p.N, p.n, 2 * p.digits_g, p.num_lut
    alg_bytes = br_key_bytes(p, args.multibit) + T * ((n + 1) * 8 + L * 2 * N * 8)
    out = {"metric": f"blind rotations/s ({'lmkcdey, ' if lmk else ''}{args.backend}, N={N}, n={n})",
           "value": world * T / (ms * 1e-3),
           "unit": "bootstraps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "u64" if args.backend == "ntt" else "f64", "data": "synthetic (seeded random LWE)",
           "config": {"workload": "blind_rotate", "batch": T, "backend": args.backend, "br_multibit": args.multibit,
                      "br_schedule": args.schedule, "br_method": args.method,
                      "param_set": args.params, "br_gadget": f"2^{p.base_g.bit_length() - 1}x{p.digits_g}",
                      "l2": "BSK read once per launch (124 MB fft64 / 124 MB ntt); no flush between launches"},
           "us_per_bootstrap": ms * 1e3 / T, "gpu_launches": args.steps,
           "roofline": br_roofline(args, p, T, ms, alg_bytes, BR_TRAFFIC.get((args.backend, args.params,
                                                                              args.multibit, T))),
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()


def rns_chain(pkg, n: int, size_q: int, size_p: int, bits: int = 50):
    """Phantom-style chain: size_q + size_p NTT primes of `bits` bits (get_primes order)."""
    out = np.zeros(size_q + size_p, np.uint64)
    pkg.call("cbs_get_primes", n, bits, size_q + size_p, out.ctypes.data)
    return out[:size_q].copy(), out[size_q:].copy()


def run_aes_setup(args, rank: int, world: int, local_rank: int) -> None:
    """Encryption of the AES material (8 x 256 T-table words and 44 round-key words as RLWE,
    the 128 round-0 key bits as LWE): cbs_aes128_setup_device (ChaCha20, NTT and products on
    the GPU; the host copies stay on the device until exported) per step, beside the host encryption cbs_aes128_setup
    (the reference's shape: one sample at a time on one host thread).  Both end with the
    material resident and its coefficient-domain copies derived."""
    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    ctx = pkg.Context(max_batch=128)
    ctx.keygen(args.seed)
    key, rng_key = bytes(range(16)), bytes(range(32, 64))
    for _ in range(max(1, args.warmup)):
        pkg.call("cbs_aes128_setup_device", ctx.handle, key, rng_key)
    torch.cuda.synchronize()
    rep = load_replicas()
    with ClockSampler(local_rank) as clk:
        rep.barrier(world)
        t0 = time.perf_counter()  # each call is synchronous (it ends with the host copies)
        for _ in range(args.steps):
            pkg.call("cbs_aes128_setup_device", ctx.handle, key, rng_key)
        dev_ms = rep.max_over_ranks((time.perf_counter() - t0) / args.steps * 1e3, world, device="cuda")
    t0 = time.perf_counter()
    pkg.call("cbs_aes128_setup", ctx.handle, key, 7)
    host_ms = (time.perf_counter() - t0) * 1e3
    samples = 8 * 256 + 44
    out = {"metric": "AES material encryptions/s (2092 RLWE + 128 LWE samples each)",
           "value": world * 1e3 / dev_ms, "unit": "setups/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u32 (ChaCha20) + u64 (mod-Q NTT)", "data": "synthetic (seeded keys)",
           "config": {"workload": "aes_setup", "rlwe_samples": samples, "lwe_samples": 128, "N": ctx.params.N},
           "gpu_launches": args.steps * (2 * 3 + 1 + 2),
           "e2e": {"value": world * 1e3 / dev_ms, "unit": "setups/s", "h2d_bytes_per_step": samples * 4 + 128,
                   "d2h_bytes_per_step": 0},
           "roofline": None,
           "cpu_baseline": {"value": 1e3 / host_ms, "unit": "setups/s", "cores": 1, "kind": "port",
                            "sample": "one cbs_aes128_setup: the same samples encrypted on the host, "
                                      "one at a time (xoshiro + Box-Muller noise, host NTT)"},
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_keyswitch(args, rank: int, world: int, local_rank: int) -> None:
    """Phantom RNS core: hybrid key switching of `--batch` ciphertexts (N = 2^16, 24 primes of
    50 bits + alpha special primes) per step, inputs resident in HBM."""
    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    n, size_q, alpha = 1 << 16, 24, args.alpha
    count = args.batch or 32
    q, p = rns_chain(pkg, n, size_q, alpha)
    ctx = pkg.RnsContext(n, q, p)
    chain = np.concatenate([q, p])
    beta = ctx.beta(size_q)
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed + rank)

    def rand_limbs(lead, mods):
        t = torch.randint(0, 2 ** 62, lead + (len(mods), n), dtype=torch.int64, device="cuda", generator=g)
        m = torch.from_numpy(np.asarray(mods).view(np.int64)).cuda().view(*([1] * len(lead)), -1, 1)
        return torch.remainder(t, m).contiguous()

    c2 = rand_limbs((count,), q)
    ct = rand_limbs((count, 2), q)
    evk = [rand_limbs((2,), chain) for _ in range(beta)]
    ptrs = pkg.RnsContext.evk_array([e.data_ptr() for e in evk])
    pkg.call("cbs_rns_prepare_level", ctx.handle, size_q)
    stream = torch.cuda.Stream()

    def fn():
        pkg.call("cbs_rns_keyswitch_inplace", ctx.handle, ct.data_ptr(), c2.data_ptr(), ptrs, size_q, count,
                 stream.cuda_stream)

    with ClockSampler(local_rank) as clk:
        ms = _timed(torch, stream, fn, args.warmup, args.steps)
    # e2e: c2 from pinned host memory, the switched ciphertext back to the host
    h_c2 = c2.cpu().pin_memory()
    h_ct = torch.empty(ct.shape, dtype=torch.int64).pin_memory()

    def e2e():
        with torch.cuda.stream(stream):
            c2.copy_(h_c2, non_blocking=True)
            fn()
            h_ct.copy_(ct, non_blocking=True)

    e2e_ms = _timed(torch, stream, e2e, 1, max(1, args.steps))
    N8 = n * 8
    qlp = size_q + alpha
    alg = beta * 2 * qlp * N8 + count * (size_q * N8 + 4 * size_q * N8 + 2 * beta * qlp * N8)
    peaks = measured_peaks()
    gbs = alg / (ms * 1e-3) / 1e9
    out = {"metric": f"CKKS hybrid key switches/s (N=2^16, 24+{alpha} primes, dnum={beta})",
           "value": world * count / (ms * 1e-3), "unit": "keyswitches/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform residues and keys)",
           "config": {"workload": "keyswitch", "batch": count, "N": n, "size_q": size_q, "size_p": alpha,
                      "beta": beta, "l2": "working set (evk + t_mod_up) >> 126 MB L2"},
           "us_per_keyswitch": ms * 1e3 / count, "gpu_launches": args.steps * 11,
           "e2e": {"value": world * count / (e2e_ms * 1e-3), "unit": "keyswitches/s",
                   "h2d_bytes_per_step": count * size_q * N8, "d2h_bytes_per_step": count * 2 * size_q * N8},
           "roofline": {"kernel": "keyswitch_inplace (modup + inner product + moddown)", "bound": "hbm",
                        "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": gbs / peaks["hbm_gbs"],
                        "peak_src": peaks["src"], "traffic": None, "algorithmic_bytes_per_step": alg},
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()


def run_rns_ntt(args, rank: int, world: int, local_rank: int) -> None:
    """Forward + inverse multi-prime NTT over `--batch` ciphertexts x 2 polys x `--limbs`
    limbs at N = 2^`--ntt-logn` (default: the Phantom-core transform, N = 2^16, 24 limbs),
    in place, inputs resident in HBM.  (The reference's own 2-D kernels on the same data are
    timed beside it by tests/test_ref_timing_gpu.py.)"""
    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    logn, size_q = args.ntt_logn, args.limbs
    n = 1 << logn
    count = args.batch or 32
    q, p = rns_chain(pkg, n, size_q, 2)
    ctx = pkg.RnsContext(n, q, p)
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed + rank)
    t = torch.randint(0, 2 ** 62, (count * 2, size_q, n), dtype=torch.int64, device="cuda", generator=g)
    x = torch.remainder(t, torch.from_numpy(q.view(np.int64)).cuda().view(1, -1, 1)).contiguous()
    ref = x.clone()
    stream = torch.cuda.Stream()
    polys = count * 2

    def fn():
        pkg.call("cbs_rns_ntt_batched", ctx.handle, x.data_ptr(), polys, size_q * n, size_q, 0, 0, stream.cuda_stream)
        pkg.call("cbs_rns_ntt_batched", ctx.handle, x.data_ptr(), polys, size_q * n, size_q, 0, 1, stream.cuda_stream)

    with ClockSampler(local_rank) as clk:
        ms = _timed(torch, stream, fn, args.warmup, args.steps)
    ok = bool(torch.equal(x, ref))  # forward then inverse is the identity
    alg = 2 * 2 * polys * size_q * n * 8  # each transform reads and writes every limb once
    peaks = measured_peaks()
    gbs = alg / (ms * 1e-3) / 1e9
    out = {"metric": f"RNS NTT forward+inverse limb-polys/s (N=2^{logn})",
           "value": world * polys * size_q / (ms * 1e-3),
           "unit": "limb-polys/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
           "data": "synthetic (seeded uniform residues)",
           "config": {"workload": "rns_ntt", "ciphertexts": count, "polys": polys, "limbs": size_q, "N": n,
                      "l2": f"{polys * size_q * n * 8 / 1e9:.2f} GB per transform "
                            f"({'>' if polys * size_q * n * 8 > 126e6 else '<'} 126 MB L2)"},
           "roundtrip_identity": ok, "gpu_launches": args.steps * (4 if logn >= 13 else 2),
           "roofline": {"kernel": "k_rns_fwd/inv cols+rows" if logn >= 13 else "k_rns_small_fwd/inv", "bound": "hbm",
                        "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": gbs / peaks["hbm_gbs"],
                        "peak_src": peaks["src"], "traffic": None, "algorithmic_bytes_per_step": alg,
                        "note": "two HBM round trips per transform (2-D)" if logn >= 13 else "one round trip"},
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()


# external-product arithmetic of the torus-32 gate path (cbs_gate_set_fft_mode): key limbs
# per key polynomial, bytes per spectrum value, and how the JSON line names it
FFT_MODE_INFO = {
    "fp64": {"limbs": 1, "bytes": 16, "fp": "fp64", "name": "FP64 FFT", "kernel": "k_gate_blind_rotate",
             "dtype": "f64 (FFT products, exact after rounding) + u32 torus"},
    "fp32-split": {"limbs": 2, "bytes": 8, "fp": "fp32", "name": "split-FP32 FFT",
                   "kernel": "k_gate_blind_rotate_f32<LIMBS=2>",
                   "dtype": "f32 (FFT products; keys split into a 24/25-bit and an exact 8/7-bit limb) + u32 torus"},
    "fp32": {"limbs": 1, "bytes": 8, "fp": "fp32", "name": "FP32 FFT", "kernel": "k_gate_blind_rotate_f32<LIMBS=1>",
             "dtype": "f32 (FFT products on whole keys, approximate) + u32 torus"},
}


def run_gate(args, rank: int, world: int, local_rank: int) -> None:
    """Plain gate bootstrapping (torus-32, n=636, N=1024, base 2^7 x 3, FP64 FFT): `--batch`
    NAND gates per step (default 64, the configuration's batch), inputs resident in HBM."""
    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    count = args.batch or 64
    ctx = pkg.GateContext(max_batch=count)
    ctx.keygen(args.seed)
    ctx.set_multibit(args.multibit)
    ctx.set_fft_mode(args.fft_mode)
    p = ctx.params
    rng = np.random.default_rng(args.seed + rank)
    x = rng.integers(0, 2, count).astype(np.uint8)
    y = rng.integers(0, 2, count).astype(np.uint8)
    a1, b1 = ctx.encrypt(x, seed=args.seed + 1)
    a2, b2 = ctx.encrypt(y, seed=args.seed + 2)
    dev = lambda v: torch.from_numpy(np.ascontiguousarray(v).view(np.int32)).cuda()  # noqa: E731
    d = [dev(v) for v in (a1, b1, a2, b2)]
    oa = torch.zeros((count, p.n), dtype=torch.int32, device="cuda")
    ob = torch.zeros(count, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    fn = lambda: pkg.call("cbs_gate_eval_batch_device", ctx.handle, pkg.GATE_NAND,  # noqa: E731
                          *(t.data_ptr() for t in d), count, oa.data_ptr(), ob.data_ptr(), stream.cuda_stream)
    with ClockSampler(local_rank) as clk:
        ms = _timed(torch, stream, fn, args.warmup, args.steps)
    torch.cuda.synchronize()
    ok = int((ctx.decrypt(oa.cpu().numpy().view(np.uint32), ob.cpu().numpy().view(np.uint32)) == 1 - (x & y)).sum())
    # e2e: inputs from pinned host memory, outputs back to the host, every step
    h_in = [t.cpu().pin_memory() for t in d]
    h_oa = torch.empty(oa.shape, dtype=torch.int32).pin_memory()
    h_ob = torch.empty(ob.shape, dtype=torch.int32).pin_memory()

    def e2e():
        with torch.cuda.stream(stream):
            for t, h in zip(d, h_in):
                t.copy_(h, non_blocking=True)
            fn()
            h_oa.copy_(oa, non_blocking=True)
            h_ob.copy_(ob, non_blocking=True)

    e2e_ms = _timed(torch, stream, e2e, 1, max(1, args.steps))
    M = p.N // 2
    logm = M.bit_length() - 1
    fm = FFT_MODE_INFO[args.fft_mode]
    limbs, esize = fm["limbs"], fm["bytes"]
    flop = count * p.n * ((2 * p.levels + 2 * limbs) * 5 * M * logm + 2 * 2 * p.levels * limbs * M * 8)
    key_bytes = (p.n * 2 * p.levels * 2 * limbs * M * esize +
                 p.N * p.ks_levels * ((1 << p.ks_base_bits) - 1) * (p.n + 1) * 4)
    peaks = measured_peaks()
    gbs = key_bytes / (ms * 1e-3) / 1e9
    out = {"metric": f"NAND gate bootstraps/s (torus32, n={p.n}, N={p.N}, {fm['name']})",
           "value": world * count / (ms * 1e-3), "unit": "gates/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": fm["dtype"],
           "data": "synthetic (seeded uniform random input bits)",
           "config": {"workload": "gate_nand", "batch": count, "n": p.n, "N": p.N, "br_multibit": args.multibit,
                      "fft_mode": args.fft_mode,
                      "gadget": f"2^{p.bg_bits}x{p.levels}", "ks": f"2^{p.ks_base_bits}x{p.ks_levels}",
                      "l2": "keys (62 MB spectra + 62 MB KSK) stay L2/HBM resident; no flush"},
           "us_per_gate": ms * 1e3 / count, "correct_gates": ok, "gpu_launches": args.steps * 2,
           "e2e": {"value": world * count / (e2e_ms * 1e-3), "unit": "gates/s",
                   "h2d_bytes_per_step": 2 * count * (p.n + 1) * 4, "d2h_bytes_per_step": count * (p.n + 1) * 4},
           "roofline": {"kernel": f"{fm['kernel']} + k_gate_keyswitch", "bound": "hbm", "achieved": gbs,
                        "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": gbs / peaks["hbm_gbs"],
                        "peak_src": peaks["src"], "traffic": None,
                        "note": "key bytes once per step; the blind rotation is FP-pipe-bound, see compute_rate"},
           "compute_rate": {f"{fm['fp']}_flop_per_step": flop,
                            f"achieved_{fm['fp']}_tflops": flop / (ms * 1e-3) / 1e12},
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()


def run_ragged(args, rank: int, world: int, local_rank: int) -> None:
    """Ragged batching: a seeded mix of sign-bootstrap requests, sizes uniform in 1..2048
    ciphertexts, parameter set per request N=1024/n=636 or N=2048/n=630 with probability 1/2,
    until at least `--batch` (default 65536) bootstraps.  One step = every request once.
    Compared: one captured CUDA graph of one ragged launch pair per parameter set (the two on
    separate streams), against one launch pair per request (the plain FP64 path)."""
    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    total_min = args.batch or 65536
    pa = pkg.gate_default_params()
    pb = pkg.gate_default_params()
    pb.N, pb.n = 2048, 630
    ctxs = [pkg.GateContext(pa, max_batch=2048), pkg.GateContext(pb, max_batch=2048)]
    for i, c in enumerate(ctxs):
        c.keygen(args.seed + i)
        c.set_multibit(args.multibit)
        c.set_fft_mode(args.fft_mode)
    rng = np.random.default_rng(args.seed + 5 + rank)
    reqs, bufs, total = [[], []], [], 0
    while total < total_min:
        cnt = int(rng.integers(1, 2049))
        which = int(rng.integers(0, 2))
        c = ctxs[which]
        bits = rng.integers(0, 2, cnt).astype(np.uint8)
        a, b = c.encrypt(bits, seed=int(rng.integers(1 << 40)))
        dev = lambda v: torch.from_numpy(np.ascontiguousarray(v).view(np.int32)).cuda()  # noqa: E731
        da, db = dev(a), dev(b)
        oa = torch.zeros((cnt, c.params.n), dtype=torch.int32, device="cuda")
        ob = torch.zeros(cnt, dtype=torch.int32, device="cuda")
        bufs.append((which, bits, da, db, oa, ob))
        reqs[which].append((da.data_ptr(), db.data_ptr(), oa.data_ptr(), ob.data_ptr(), cnt))
        total += cnt
    s_main, s_side = torch.cuda.Stream(), torch.cuda.Stream()

    def per_request():
        for (which, _, da, db, oa, ob) in bufs:
            pkg.call("cbs_gate_bootstrap_batch_device", ctxs[which].handle, da.data_ptr(), db.data_ptr(), len(ob),
                     None, oa.data_ptr(), ob.data_ptr(), s_main.cuda_stream)

    def capture(grids):
        for i, c in enumerate(ctxs):
            c.ragged_plan(reqs[i], grid_ctas=grids[i])
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s_main):
            cur = torch.cuda.current_stream()
            s_side.wait_stream(cur)
            ctxs[0].ragged_launch(cur.cuda_stream)
            with torch.cuda.stream(s_side):
                ctxs[1].ragged_launch(s_side.cuda_stream)
            cur.wait_stream(s_side)
        return g

    # tile schedule: the product's autotuner picks each parameter set's persistent grid on its plan
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    tune = []
    best = []
    for i, c in enumerate(ctxs):
        c.ragged_plan(reqs[i], grid_ctas=0)
        grid, t_ms = c.ragged_autotune()
        best.append(grid)
        tune.append({"set": i, "grid_ctas": grid, "ctas_per_sm": grid / sms, "ms": t_ms})

    def replay_on(graph):
        def run():
            with torch.cuda.stream(s_main):  # replay on the stream the events are recorded on
                graph.replay()
        return run

    g = capture(best)
    with ClockSampler(local_rank) as clk:
        ms = _timed(torch, s_main, replay_on(g), args.warmup, args.steps)
    ok = 0
    for (which, bits, _, _, oa, ob) in bufs:
        got = ctxs[which].decrypt(oa.cpu().numpy().view(np.uint32), ob.cpu().numpy().view(np.uint32))
        ok += int((got == bits).sum())
    per_ms = _timed(torch, s_main, per_request, 1, max(1, min(args.steps, 2)))
    out = {"metric": "ragged sign-bootstrap throughput (bootstraps/s, mixed N=1024/n=636 and N=2048/n=630)",
           "value": world * total / (ms * 1e-3), "unit": "bootstraps/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": FFT_MODE_INFO[args.fft_mode]["dtype"],
           "data": "synthetic (seeded request sizes, parameter sets and bits)",
           "config": {"workload": "ragged_bootstrap", "requests": len(bufs), "bootstraps": total,
                      "br_multibit": args.multibit, "fft_mode": args.fft_mode,
                      "per_set": [sum(r[4] for r in reqs[0]), sum(r[4] for r in reqs[1])],
                      "l2": "keys of both sets (2 x ~125 MB) do not fit L2 together; no flush"},
           "correct": ok, "gpu_launches": args.steps * 4,
           "per_request_launches": {"ms_per_step": per_ms, "value": world * total / (per_ms * 1e-3),
                                    "launches_per_step": 2 * len(bufs), "ragged_speedup": per_ms / ms},
           "autotune": {"chosen_grid_ctas": list(best), "per_set": tune,
                        "note": "cbs_gate_ragged_autotune: one timed launch per candidate grid and set"},
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    del g
    for c in ctxs:
        c.close()


def run_tcb(args, rank: int, world: int, local_rank: int) -> None:
    """Circuit bootstrapping with PFKS (the configuration's parameters): `--batch` LWE bits
    (default 256, n=630, sigma 2^-15) to RGSW under the level-1 key per step; then the phase
    error of every produced RGSW row against its exact message and the failure probability
    of one CMux that uses these rows (Gaussian tail of the measured row error)."""
    import math

    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    sys.path.insert(0, str(ROOT / "tests"))
    from tcb_harness import rgsw_row_errors  # noqa: E402  (exact decryption of the rows)
    count = args.batch or 256
    ctx = pkg.TcbContext(max_batch=count)
    ctx.keygen(args.seed)
    ctx.set_multibit(args.multibit)
    p = ctx.params
    rng = np.random.default_rng(args.seed + rank)
    bits = rng.integers(0, 2, count).astype(np.uint8)
    a, b = ctx.encrypt(bits, seed=args.seed + 3)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    rgsw = torch.zeros((count, p.cb_levels, 2, 2, p.N1), dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()

    def fn():
        pkg.call("cbs_tcb_circuit_bootstrap_device", ctx.handle, da.data_ptr(), db.data_ptr(), count, None,
                 rgsw.data_ptr(), stream.cuda_stream)

    with ClockSampler(local_rank) as clk:
        ms = _timed(torch, stream, fn, args.warmup, args.steps)
    keys = ctx.export_keys(with_pfks=False)
    sample = min(count, 32)
    rg = rgsw[:sample].cpu().numpy().view(np.uint32)
    err = rgsw_row_errors(rg, bits[:sample], keys["z1"], p.cb_bits, p.cb_levels).astype(np.float64)
    sigma_row = float(np.std(err)) / 2 ** 32
    # one CMux with these rows: error = sum over 2*levels*N1 digit-row products, digits uniform
    # in [-2^(b-1), 2^(b-1)); a decision at distance 1/8 from the message
    sigma_digit = (2 ** p.cb_bits) / math.sqrt(12.0)
    sigma_cmux = math.sqrt(2 * p.cb_levels * p.N1) * sigma_digit * sigma_row
    z = 0.125 / sigma_cmux
    log2_pfail = (math.log2(math.erfc(z / math.sqrt(2))) if z < 37 else
                  -(z * z / 2) / math.log(2) - math.log2(z * math.sqrt(math.pi / 2)))
    pfks_bytes = 2 * (p.N2 + 1) * p.pfks_levels * ((1 << p.pfks_base_bits) - 1) * 2 * p.N1 * 4
    out = {"metric": "circuit bootstraps/s with PFKS (n=630 -> RGSW, N2=2048 2^9x3, PFKS 2^4x8, FP64 FFT)",
           "value": world * count / (ms * 1e-3), "unit": "bits/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64 (64-bit-torus FFT products) + u32/u64 torus",
           "data": "synthetic (seeded uniform random bits)",
           "config": {"workload": "tcb_pfks", "bits": count, "n": p.n, "N2": p.N2, "l2": p.l2, "bg2_bits": p.bg2_bits,
                      "br_multibit": args.multibit,
                      "N1": p.N1, "cb": f"2^{p.cb_bits}x{p.cb_levels}", "pfks": f"2^{p.pfks_base_bits}x{p.pfks_levels}",
                      "l2_cache": f"PFKS keys {pfks_bytes / 1e9:.1f} GB >> 126 MB L2"},
           "us_per_bit": ms * 1e3 / count, "gpu_launches": args.steps * 2,
           "phase_error": {"rows_sampled": int(err.size), "sigma_log2": math.log2(sigma_row),
                           "max_log2": math.log2(float(np.max(np.abs(err))) / 2 ** 32),
                           "cmux_sigma_log2": math.log2(sigma_cmux), "cmux_pfail_log2": log2_pfail,
                           "note": "row phases vs exact m*g_k (row 2k+1) and -m*g_k*z1 (row 2k); FP64 path"},
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()


def mb_keys(mb: int) -> int:
    """Grouped keys per group: 2^mb - 1 subsets, 8 for the staged mb = 4 (3 + 1)."""
    return 8 if mb == 4 else (1 << mb) - 1


def br_key_bytes(p, mb: int) -> int:
    """Blind-rotation key bytes one launch reads (once, shared through L2): n RGSWs, or
    ceil(n/mb) groups of mb_keys(mb) RGSWs; FFT spectra and NTT words are both 8 bytes per
    coefficient."""
    rgsw = 2 * p.digits_g * 2 * p.N * 8
    return (-(-p.n // mb)) * mb_keys(mb) * rgsw


# DRAM bytes (read + write) of one blind-rotation launch, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum, one pass) on the launch this bench times:
# (backend, parameter set, mb, ciphertexts per launch) -> bytes.  16384 = 128 blocks x 128 bits;
# the grouped key (186 MB at 3x12, 124 MB at 2x18) does not stay in the 126 MB L2 while the
# multi-value outputs stream through it, so each wave of 148 ciphertexts re-reads it.
BR_TRAFFIC = {("fft64", "3x12", 2, 16384): 20810.3e6 + 2151.6e6,
              ("fft64", "2x18", 2, 16384): 13797.989e6 + 2148.365e6}


def br_roofline(args, p, T: int, br_ms: float, alg_bytes: int, traffic) -> dict:
    """Roofline of the dominant kernel, the fused blind rotation: on the FFT backend its bound is
    the FP64 pipe (algorithmic flops per launch over the launch time against the recorded FP64
    peak); the exact-NTT backend is bounded by 64-bit integer multiplies and reports HBM."""
    method = "LMKCDEY" if getattr(args, "method", "ginx") == "lmkcdey" else "GINX"
    name = br_kernel_name(args, p) + f" (fused {method} blind rotation + finalize + MV split)"
    extra = {"algorithmic_bytes_per_launch": alg_bytes, "launch_ms": br_ms, "traffic": traffic,
             "traffic_over_algorithmic": (traffic / alg_bytes) if traffic else None,
             "traffic_src": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this launch (one pass), recorded"}
    if args.backend in ("fft64", "fft64-split"):
        flop = (fp64_flop_per_launch(p, T, args.multibit) if args.backend == "fft64"
                else split_fp64_flop_per_launch(p, T, args.multibit))
        achieved = flop / (br_ms * 1e-3) / 1e12
        return {"kernel": name, "bound": "fp64", "achieved": achieved, "peak": FP64_PEAK["tflops"],
                "unit": "TFLOP/s", "frac": achieved / FP64_PEAK["tflops"], "peak_src": FP64_PEAK["src"],
                "fp64_flop_per_launch": flop, **extra}
    peaks = measured_peaks()
    gbs = alg_bytes / (br_ms * 1e-3) / 1e9
    return {"kernel": name, "bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": gbs / peaks["hbm_gbs"], "peak_src": peaks["src"],
            "note": "integer-multiply bound; compute_rate gives the modular products per second",
            "compute_rate": None if method == "LMKCDEY" else compute_rate(args.backend, T, p, br_ms, args.multibit),
            **extra}


def br_kernel_name(args, p=None) -> str:
    if getattr(args, "method", "ginx") == "lmkcdey":
        return "k_lmkcdey"
    if args.backend == "fft64-split":
        return f"k_blind_rotate_fft_split<11,·,{p.digits_g if p is not None else '·'},{args.multibit}>"
    if args.backend != "fft64":
        return "k_blind_rotate"
    if args.multibit == 1:
        return "k_blind_rotate_fft"
    sched = getattr(args, "schedule", 0)
    if args.multibit == 2 and p is not None and p.digits_g == 2 and sched == 3 and p.N == 2048:
        return "k_blind_rotate_fft_mb2_x2<11> (two ciphertexts per CTA, digit transforms in lockstep)"
    if args.multibit == 2 and p is not None and p.digits_g == 2 and sched != 1:
        return "k_blind_rotate_fft_mb_d2<11,2> (two digit transforms in lockstep)"
    return f"k_blind_rotate_fft_mb<11,{args.multibit}>"


# FP64 peak of this pool's B200, measured once (not driver-written): cuBLAS DGEMM through
# torch.matmul, float64 4096^3 (2 n^3 flop), best of 5 after a warm-up, CUDA events; three runs
# on separate boxes gave 35.43, 35.36 and 35.40 TFLOP/s at 1965 MHz (profiles/fp64_peak_b200.md).
FP64_PEAK = {"tflops": 35.4, "src": "recorded: cuBLAS DGEMM 4096^3 (torch.matmul float64), best of 5, "
                                    "median of three B200 runs (profiles/fp64_peak_b200.md); not driver-written"}


def run_keygen(args, rank: int, world: int, local_rank: int) -> None:
    """Key generation of the headline parameter set: the seeded host generation (cbs_keygen, the
    role of the reference's OpenFHE CirBTKeyGen + gpu_init_cirbsk) against the device generation
    (cbs_keygen_device, ChaCha20 per coefficient), each followed by the FFT key spectra and the
    grouped (mb = 2) keys the AES path needs; wall time of the synchronous calls."""
    import torch
    torch.cuda.set_device(local_rank)
    pkg = load_pkg()
    p = pkg.preset_params(args.params)
    res = {}
    for name in ("host", "device"):
        ctx = pkg.Context(params=p, max_batch=128)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if name == "host":
            ctx.keygen(args.seed)
        else:
            ctx.keygen_device(bytes(range(32)))
        t1 = time.perf_counter()
        pkg.call("cbs_context_set_br_backend", ctx.handle, pkg.BR_FFT64)
        ctx.set_br_multibit(2)
        t2 = time.perf_counter()
        res[name] = {"keygen_s": t1 - t0, "fft_and_grouped_keys_s": t2 - t1, "total_s": t2 - t0}
        ctx.close()
    if rank == 0:
        print(json.dumps({"metric": f"key generation, {args.params} parameter set (seconds, lower is better)",
                          "value": res["device"]["keygen_s"], "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
                          "higher_is_better": False, "data": "synthetic (fixed ChaCha20 key / seed)",
                          "config": {"workload": "keygen", "param_set": args.params,
                                     "keys": "secrets, BSK, HomTrace, SchemeSwitch, extraction KSK; then FFT "
                                             "spectra and mb = 2 grouped keys"},
                          "host": res["host"], "device": res["device"],
                          "speedup_keygen": res["host"]["keygen_s"] / res["device"]["keygen_s"]}), flush=True)


def run_fp64_peak(args, rank: int, world: int, local_rank: int) -> None:
    """The FP64 peak the blind rotation's roofline is quoted against: cuBLAS DGEMM through
    torch.matmul, float64 n^3 (n = 4096, 2 n^3 flop), best of 5 after a warm-up, CUDA events."""
    import torch
    torch.cuda.set_device(local_rank)
    n = 4096
    a = torch.randn((n, n), dtype=torch.float64, device="cuda")
    b = torch.randn((n, n), dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = float("inf")
    with ClockSampler(local_rank) as clk:
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
    if rank == 0:
        print(json.dumps({"metric": "FP64 DGEMM TFLOP/s (cuBLAS through torch.matmul, 4096^3)",
                          "value": 2 * n ** 3 / (best * 1e-3) / 1e12, "unit": "TFLOP/s", "ms": best,
                          "clocks": clk.summary()}), flush=True)


def fp64_flop_per_launch(p, T: int, mb: int) -> int:
    """Algorithmic FP64 flops of one FFT blind-rotation launch over T ciphertexts: per step (mb = 1)
    or group, 2 digits_g forward and 2 inverse M-point complex transforms (5 M log2 M each), and
    per spectrum slot and key row 8 flops per complex multiply-add with the 2^mb - 1 combined keys
    plus the product with the digit spectrum (mb > 1).  The staged mb = 4 runs per group an mb = 3
    step and a one-bit step (the latter skipped for a group without a fourth coefficient)."""
    N, n, l2 = p.N, p.n, 2 * p.digits_g
    M = N // 2
    fft_flop = 5 * M * (M.bit_length() - 1)
    if mb == 4:
        return T * (
            (-(-n // 4)) * ((l2 + 2) * fft_flop + 2 * l2 * M * 8 * 8) + (n // 4) * ((l2 + 2) * fft_flop + 2 * l2 * M * 8))
    steps = -(-n // mb)
    keys = (1 << mb) - 1
    return T * steps * ((l2 + 2) * fft_flop + 2 * l2 * M * 8 * (keys + (1 if mb > 1 else 0)))


def split_fp64_flop_per_launch(p, T: int, mb: int) -> int:
    """Algorithmic FP64 flops of the exact split-FFT blind rotation: per step 2 digits forward
    and 2 limbs inverse M-point transforms, and per limb the digit x key-limb products of both
    columns (mb = 2: the combined key c0 (K0 + c1 K01) + c1 K1 adds three complex multiply-adds
    per product).  Limbs from the plan the backend uses (cbs_split_fft_plan)."""
    M, n, l2 = p.N // 2, p.n, 2 * p.digits_g
    limbs = 3  # both parameter sets, mb 1 and 2: 3 balanced limbs of 18 bits
    fft_flop = 5 * M * (M.bit_length() - 1)
    steps = -(-n // mb)
    return T * steps * ((l2 + 2 * limbs) * fft_flop + limbs * 2 * l2 * M * 8 * (1 if mb == 1 else 4))


def compute_rate(backend: str, T: int, p, br_ms: float, mb: int = 1) -> dict:
    """Algorithmic arithmetic rate of one blind-rotation launch over T ciphertexts."""
    N, n, l2 = p.N, p.n, 2 * p.digits_g
    logn = N.bit_length() - 1
    if backend == "fft64":
        flop = fp64_flop_per_launch(p, T, mb)
        achieved = flop / (br_ms * 1e-3) / 1e12
        return {"kernel": "k_blind_rotate_fft" if mb == 1 else f"k_blind_rotate_fft_mb (mb={mb})",
                "fp64_flop_per_launch": flop, "achieved_fp64_tflops": achieved,
                "fp64_peak_tflops": FP64_PEAK["tflops"], "frac": achieved / FP64_PEAK["tflops"],
                "peak_src": FP64_PEAK["src"],
                "note": "algorithmic flops (5 M log2 M per M-point complex transform, 8 per complex "
                        "multiply-add); ncu counts ~12 % more executed FP64 flops"}
    modmuls = T * n * (8 * (N // 2) * logn + 2 * l2 * N)
    return {"kernel": "k_blind_rotate", "modmul_per_launch": modmuls,
            "achieved_gmodmul_s": modmuls / (br_ms * 1e-3) / 1e9}


def cpu_sample(args) -> dict:
    """Time the CPU oracle on a bounded sample of the AES workload, with the bench's parameter
    set and blind-rotation grouping: two circuit bootstraps per host thread in parallel (blind
    rotation over groups of args.multibit coefficients + HomTrace + SchemeSwitch of its num_lut
    multi-value RLWEs), two 8->32 CMux LUTs per thread, 128 extract + key switches; blocks/s is
    composed as 10 rounds x (128 CBS + 16 LUT + 128 extractions) from the per-unit times.  Keys
    and parameters come from the oracle itself: nothing of the product library is loaded."""
    sys.path.insert(0, str(ROOT / "tests"))
    from cbs_harness import OracleCbs, lwe_encrypt_bits, oracle_keys, oracle_keys_mb, oracle_params  # noqa: E402
    from conftest import load_oracle  # noqa: E402
    from concurrent.futures import ThreadPoolExecutor

    o = load_oracle()
    threads = int(o.orc_num_threads())
    p = oracle_params(o, args.params)
    keys = oracle_keys(o, p, args.seed)
    mb = args.multibit
    mbk = oracle_keys_mb(o, p, keys, mb, args.seed) if mb > 1 else None
    oc = OracleCbs(o, p, keys)
    rng = np.random.default_rng(1)
    nb = 2 * threads  # two per thread: a few seconds of host work per sample
    a, b = lwe_encrypt_bits(rng, keys["s_lwe"], rng.integers(0, 2, nb), p.q_lwe)
    w0 = time.perf_counter()
    t0 = time.perf_counter()
    if mbk is None:
        oc.br_acc(a, b)
    else:
        oc.br_acc_mb(a, b, mbk, mb)
    t_br = (time.perf_counter() - t0) / nb
    mv = rng.integers(0, p.Q, size=(nb * p.num_lut, 2, p.N), dtype=np.uint64)
    t0 = time.perf_counter()
    rg = oc.trace_ss(mv)
    t_trace = (time.perf_counter() - t0) / nb
    t_cbs = t_br + t_trace
    rg = rg.reshape(nb, -1)[:, : p.num_lut * 4 * p.N]
    table = rng.integers(0, p.Q, size=(256, 2, p.N), dtype=np.uint64)
    ctrls = [np.ascontiguousarray(rg[k % nb]) for k in range(8)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda _: oc.lut(table, ctrls), range(2 * threads)))
    t_lut = (time.perf_counter() - t0) / (2 * threads)
    words = rng.integers(0, p.Q, size=(4, 2, p.N), dtype=np.uint64)
    info = np.array([((t // 32) << 16) | (t % 32) for t in range(128)], np.uint32)
    t0 = time.perf_counter()
    oc.extract(words, info)
    t_ext = (time.perf_counter() - t0) / 128
    wall = time.perf_counter() - w0
    per_block = ROUNDS * (128 * t_cbs + 16 * t_lut + 128 * t_ext)
    return {"value": 1.0 / per_block, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{nb} circuit bootstraps (blind rotation n={p.n}, mb={mb}, gadget 2^{p.base_g.bit_length() - 1}"
                      f"x{p.digits_g}; HomTrace + SchemeSwitch of {p.num_lut} RLWEs each) on {threads} threads, "
                      f"{2 * threads} 8->32 CMux LUTs, 128 extract+KS; blocks/s composed as 10 rounds x (128 CBS + 16 LUT + "
                      f"128 extract) from the per-unit times",
            "sample_wall_s": wall, "params": args.params,
            "per_unit_s": {"cbs": t_cbs, "blind_rotation": t_br, "trace": t_trace, "lut": t_lut, "extract": t_ext},
            "mulmod": "exact 128/64-bit hardware division (measured on the build host: 8.1 ns per dependent "
                      "modular product against 10.5 ns for a Barrett reduction, so kept)"}


def cpu_baseline(args) -> dict:
    return cpu_sample(args)


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    vals, walls = [], []
    last = None
    for i in range(args.warmup + args.steps):
        r = cpu_sample(args)
        if i >= args.warmup:
            vals.append(r["value"])
            walls.append(r["sample_wall_s"])
            last = r
    value = statistics.median(vals)
    last["value"] = value
    out = {
        "impl": "reference", "metric": METRICS[args.backend], "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (exact mod-Q arithmetic, CPU)",
        "data": "synthetic (seeded)",
        "config": {"workload": "aes128_ctr_transcipher", "blocks_per_gpu": args.blocks, "param_set": args.params,
                   "br_multibit": args.multibit,
                   "note": "the reference's CPU path (OpenFHE fork) is absent; CPU restatement of the same "
                           "algorithm (oracle/) on all host threads; each step is one bounded sample (its wall "
                           "time is ms_per_step) from which blocks/s is composed"},
        "cpu_baseline": last,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--blocks", type=int, default=128)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--backend", choices=["fft64", "ntt", "fft64-split"], default="fft64",
                    help="blind-rotation arithmetic: FP64 FFT (approximate, the headline), exact 64-bit NTT, or "
                         "the exact split FFT (FP64 products of key limbs, bit-identical to ntt)")
    ap.add_argument("--multibit", type=int, choices=[1, 2, 3, 4], default=None,
                    help="blind rotation over groups of 1, 2, 3 or 4 (staged 3 + 1) LWE coefficients "
                         "(fft64 backend; fft64-split takes 1 or 2; default 2 for fft64 and fft64-split, 1 for ntt)")
    ap.add_argument("--fft-mode", dest="fft_mode", choices=["fp64", "fp32-split", "fp32"], default="fp64",
                    help="external-product arithmetic of --workload gate / ragged (torus-32): exact FP64, "
                         "split FP32 (24/25-bit + exact top key limb), or FP32 on whole keys; FP32 modes use "
                         "--multibit 1")
    ap.add_argument("--params", choices=["3x12", "2x18"], default="2x18",
                    help="parameter set of the aes128 / blind_rotate workloads: blind-rotation gadget 2^12 x 3 "
                         "(cbs_params_default) or 2^18 x 2")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="aes128 on fft64: use --multibit instead of the product's autotuned grouping")
    ap.add_argument("--schedule", choices=["auto", "digitwise", "lockstep", "paired"], default="auto",
                    help="two-digit grouped blind-rotation schedule (aes128 with --no-tune / --multibit, "
                         "blind_rotate); auto = the context's tuned choice")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--workload", choices=["aes128", "blind_rotate", "keyswitch", "rns_ntt", "gate", "ragged", "tcb",
                                           "aes_setup", "fp64_peak", "keygen"],
                    default="aes128",
                    help="aes128 is the headline; the others time one kernel family")
    ap.add_argument("--batch", type=int, default=0, help="units per step for the kernel workloads")
    ap.add_argument("--method", choices=["ginx", "lmkcdey"], default="ginx",
                    help="blind-rotation method of --workload blind_rotate (lmkcdey: exact NTT form, one LUT slot, "
                         "10 automorphism keys; needs --params 2x18)")
    ap.add_argument("--alpha", type=int, default=2, help="special primes (digit width) for --workload keyswitch")
    ap.add_argument("--ntt-logn", dest="ntt_logn", type=int, default=16, help="log2 N for --workload rns_ntt")
    ap.add_argument("--limbs", type=int, default=24, help="limbs per polynomial for --workload rns_ntt")
    args = ap.parse_args()
    if args.fft_mode != "fp64":
        if args.workload not in ("gate", "ragged"):
            ap.error("--fft-mode applies to --workload gate / ragged")
        if args.multibit not in (None, 1):
            ap.error("--fft-mode fp32* runs one coefficient per step (--multibit 1)")
        args.multibit = 1
    args.schedule = {"auto": 0, "digitwise": 1, "lockstep": 2, "paired": 3}[args.schedule]
    if args.multibit is not None or args.schedule:
        args.tune = False  # an explicit grouping or schedule is measured as given
    if args.multibit is None:
        args.multibit = 2 if args.backend in ("fft64", "fft64-split") else 1
    if args.multibit > 1 and args.backend != "fft64" and not (args.backend == "fft64-split" and args.multibit == 2):
        ap.error("--multibit > 1 needs --backend fft64 (or 2 with fft64-split)")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        # short timeout: a rank that dies or hangs ends the others' next collective with an error
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    runner = {"aes128": run_ours, "blind_rotate": run_blind_rotate, "keyswitch": run_keyswitch,
              "rns_ntt": run_rns_ntt, "gate": run_gate,
              "ragged": run_ragged, "tcb": run_tcb, "aes_setup": run_aes_setup,
              "fp64_peak": run_fp64_peak, "keygen": run_keygen}[args.workload]
    try:
        runner(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
