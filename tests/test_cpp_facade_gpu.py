"""A C++ program written against the reference-shaped facade (include/cbs_b200.hpp), compiled
and linked against libcbs_b200.so, run on the GPU (tests/cpp/facade_main.cpp):
* keyswitch_inplace(PhantomContext, PhantomCiphertext, c2, PhantomRelinKey, is_relin, stream)
  (src/eval_key_switch.cu:94) on a level-2 ciphertext, bit-exact against the oracle;
* GPUCirBTSContext::gpu_CircuitBootstrappingBatch / gpu_CircuitBootstrapping /
  gpu_CircuitBootstrappingBatchToDevice on host LWE ciphertexts (cirbts.cuh:454-462), the RGSW
  rows bit-exact against the oracle's circuit bootstrap;
* GPUBinFHEContext::BatchGPUEvalBinGate(NAND, ...) (binfhecontext.cuh:53-57), every gate
  decrypting to the truth table, and its functional evaluators (EvalFunc / Floor / Sign / Decomp,
  :60-118), every result decrypting right;
* GPUCirBTSContext with the LMKCDEY method (SetMethod, LMKCDEY_EvalAcc, cirbts.cuh:491), CBS rows
  and EvalAcc bit-exact against the oracle;
* the CKKS evaluator (include/evaluate.cuh): multiply_and_relin_inplace + rescale_to_next_inplace
  and rotate_inplace, bit-exact against the oracle's keyswitch with the restated tensor
  product, rescale and Galois permutation."""
from __future__ import annotations

import ctypes
import shutil
import subprocess

import numpy as np
import pytest

from cbs_harness import OracleCbs, lwe_encrypt_bits
from conftest import PKG_DIR, ROOT
from rns_harness import declare_rns, rns_primes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def facade_bin(tmp_path_factory, lib):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("facade") / "facade_main"
    cmd = [gxx, "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-I", "/usr/local/cuda/include",
           str(ROOT / "tests" / "cpp" / "facade_main.cpp"), "-o", str(out), "-L", str(PKG_DIR), "-lcbs_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{PKG_DIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def _run(binary, mode, d):
    r = subprocess.run([str(binary), mode, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, f"{mode}: exit {r.returncode}: {r.stderr}"


def test_facade_keyswitch_inplace(facade_bin, tmp_path, oracle):
    o = declare_rns(oracle)
    n, logn, size_q, size_p, chain_index = 1 << 12, 12, 6, 2, 2
    size_ql = size_q - (chain_index - 1)
    q, p = rns_primes(o, n, size_q, size_p)
    chain = np.concatenate([q, p]).astype(np.uint64)
    beta = -(-size_q // size_p)
    rng = np.random.default_rng(404)
    ql = q[:size_ql]
    c2 = np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in ql])
    ct = np.stack([np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in ql]) for _ in range(2)])
    evk = np.stack([np.stack([np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in chain])
                              for _ in range(2)]) for _ in range(beta)])
    np.array([n, size_q, size_p, chain_index, beta], np.uint64).tofile(tmp_path / "ks_dims")
    chain.tofile(tmp_path / "ks_chain")
    c2.tofile(tmp_path / "ks_c2")
    ct.tofile(tmp_path / "ks_ct")
    evk.tofile(tmp_path / "ks_evk")
    _run(facade_bin, "ks", tmp_path)
    got = np.fromfile(tmp_path / "ks_out", np.uint64).reshape(ct.shape)
    want = np.ascontiguousarray(ct).copy()
    o.orc_keyswitch(want, np.ascontiguousarray(c2), np.ascontiguousarray(evk), logn, q, size_ql, size_q, p, size_p)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("backend", ["ntt", "split"])
def test_facade_circuit_bootstrap_host_lwe(facade_bin, tmp_path, pkg, oracle, backend):
    """The exact backends through the facade (SetBackend): NTT and the split FFT (the
    reference's CIRBTS_BACKEND=split_fft), both bit-identical to the oracle's CBS."""
    p = pkg.default_params()
    seed, batch = 21, 3
    keys = pkg.generate_keys_host(p, seed)
    rng = np.random.default_rng(5)
    a, b = lwe_encrypt_bits(rng, keys["s_lwe"], [1, 0, 1], p.q_lwe)
    be = pkg.BR_NTT if backend == "ntt" else pkg.BR_FFT64_SPLIT
    np.array([seed, batch, be], np.uint64).tofile(tmp_path / "cbs_dims")
    a.astype(np.uint64).tofile(tmp_path / "cbs_a")
    b.astype(np.uint64).tofile(tmp_path / "cbs_b")
    _run(facade_bin, "cbs", tmp_path)
    got = np.fromfile(tmp_path / "cbs_out", np.uint64).reshape(batch, p.num_lut, 2, 2, p.N)
    oc = OracleCbs(oracle, p, keys)
    want = np.zeros((batch, p.num_lut, 2, 2, p.N), np.uint64)
    oracle.orc_circuit_bootstrap(ctypes.byref(oc.op), ctypes.byref(oc.ok), a.ctypes.data, b.ctypes.data, batch, p.n,
                                 want.ctypes.data)
    assert np.array_equal(got, want)


def test_facade_lmkcdey(facade_bin, tmp_path, pkg, oracle):
    """SetMethod(LMKCDEY) and LMKCDEY_EvalAcc through the facade: the CBS rows equal the oracle's
    HomTrace + SchemeSwitch of its LMKCDEY accumulator, and EvalAcc the oracle's, word for word."""
    from cbs_harness import oracle_lmkcdey_keys
    p = pkg.preset_params("2x18")
    p.num_lut = 1
    seed, batch, num_auto = 23, 2, 10
    keys = pkg.generate_keys_host(p, seed)
    rng = np.random.default_rng(6)
    a, b = lwe_encrypt_bits(rng, keys["s_lwe"], [1, 0], p.q_lwe)
    acc = rng.integers(0, p.Q, size=(2, p.N), dtype=np.uint64)
    masks = rng.integers(0, 2 * p.N, size=p.n, dtype=np.uint32)
    np.array([seed, batch, num_auto], np.uint64).tofile(tmp_path / "lmk_dims")
    a.astype(np.uint64).tofile(tmp_path / "lmk_a")
    b.astype(np.uint64).tofile(tmp_path / "lmk_b")
    acc.tofile(tmp_path / "lmk_acc")
    masks.tofile(tmp_path / "lmk_masks")
    _run(facade_bin, "lmk", tmp_path)
    oc = OracleCbs(oracle, p, keys)
    lmk = oracle_lmkcdey_keys(oracle, p, keys, num_auto, seed)
    got = np.fromfile(tmp_path / "lmk_cbs_out", np.uint64).reshape(batch, 2, 2, p.N)
    assert np.array_equal(got, oc.trace_ss(oc.br_acc_lmkcdey(a, b, lmk)))
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    oracle.orc_lmkcdey_eval_acc.argtypes = [vp, vp, vp, vp, u32, u32, vp, u32, vp]
    want = acc.copy()
    oracle.orc_lmkcdey_eval_acc(ctypes.byref(oc.op), lmk["eval"].ctypes.data, lmk["auto"].ctypes.data,
                                lmk["maps"].ctypes.data, num_auto, 0, masks.ctypes.data, p.n, want.ctypes.data)
    assert np.array_equal(np.fromfile(tmp_path / "lmk_acc_out", np.uint64).reshape(2, p.N), want)


def test_facade_batch_gate(facade_bin, tmp_path):
    _run(facade_bin, "gate", tmp_path)


def test_facade_functional_evaluators(facade_bin, tmp_path):
    """GPUBinFHEContext::BatchGPUEvalFunc / GPUEvalFunc / BatchGPUEvalSign / BatchGPUEvalFloor /
    BatchGPUEvalDecomp (binfhecontext.cuh:60-118) at the default gate parameters: every result
    decrypts to what it computes."""
    _run(facade_bin, "gfunc", tmp_path)


def test_facade_ckks_evaluator(facade_bin, tmp_path, oracle):
    from rns_harness import addmod, mulmod, ntt
    from test_ckks_gpu import galois_perm, rescale_oracle
    o = declare_rns(oracle)
    n, logn, size_q, size_p, chain_index = 1 << 12, 12, 5, 2, 1
    size_ql = size_q - (chain_index - 1)
    q, p = rns_primes(o, n, size_q, size_p)
    chain = np.concatenate([q, p]).astype(np.uint64)
    beta = -(-size_q // size_p)
    rng = np.random.default_rng(606)
    ql = q[:size_ql]
    colq = ql.reshape(-1, 1)

    def rnd(shape_lead):
        return np.stack([np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in ql])
                         for _ in range(shape_lead)])

    ct1, ct2 = rnd(2), rnd(2)
    rk = np.stack([np.stack([np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in chain])
                             for _ in range(2)]) for _ in range(beta)])
    gk = np.stack([np.stack([np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in chain])
                             for _ in range(2)]) for _ in range(beta)])
    elt = 5  # rotation by one step
    np.array([n, size_q, size_p, chain_index, beta, elt], np.uint64).tofile(tmp_path / "ck_dims")
    chain.tofile(tmp_path / "ck_chain")
    ct1.tofile(tmp_path / "ck_ct1")
    ct2.tofile(tmp_path / "ck_ct2")
    rk.tofile(tmp_path / "ck_rk")
    gk.tofile(tmp_path / "ck_gk")
    _run(facade_bin, "ckks", tmp_path)
    # multiply + relinearize + rescale
    d0 = mulmod(ct1[0], ct2[0], colq)
    d1 = addmod(mulmod(ct1[0], ct2[1], colq), mulmod(ct1[1], ct2[0], colq), colq)
    d2 = mulmod(ct1[1], ct2[1], colq)
    want = np.ascontiguousarray(np.stack([d0, d1]))
    o.orc_keyswitch(want, np.ascontiguousarray(d2), np.ascontiguousarray(rk), logn, q, size_ql, size_q, p, size_p)
    want = rescale_oracle(o, want, ql)
    got = np.fromfile(tmp_path / "ck_mr", np.uint64).reshape(want.shape)
    assert np.array_equal(got, want)
    # rotate by one step
    perm = galois_perm(elt, logn)
    want = np.ascontiguousarray(np.stack([ct1[0][:, perm], np.zeros_like(ct1[1])]))
    o.orc_keyswitch(want, np.ascontiguousarray(ct1[1][:, perm]), np.ascontiguousarray(gk), logn, q, size_ql, size_q,
                    p, size_p)
    got = np.fromfile(tmp_path / "ck_rot", np.uint64).reshape(want.shape)
    assert np.array_equal(got, want)
