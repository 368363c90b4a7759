"""GPU parity of the RNS path (multi-prime NTT, modup, key inner product, moddown,
keyswitch_inplace) against the CPU oracle: bit-exact on seeded inputs, through the C ABI."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_pkg, load_oracle
from rns_harness import (addmod, crt_centered, declare_rns, make_switch_key, mulmod, ntt, rns_primes, small_to_rns,
                         submod)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available()
    return load_pkg(), declare_rns(load_oracle()), torch


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint64)


def rand_limbs(rng, mods, n, lead=()):
    return np.stack([rng.integers(0, int(m), lead + (n,), dtype=np.uint64) for m in mods], axis=len(lead))


@pytest.mark.parametrize("logn,bits", [(10, 50), (11, 50), (12, 50), (13, 50), (14, 50), (15, 50), (16, 50),
                                       (17, 50), (13, 59), (16, 59)])
def test_rns_ntt_bit_exact(env, logn, bits):
    """50-bit primes take the FP64-pipe 2-D transforms (N >= 2^13), 59-bit primes the integer
    ones; both bit-exact."""
    pkg, o, torch = env
    n = 1 << logn
    q, p = rns_primes(o, n, 3, 2, bits)
    chain = np.concatenate([q, p])
    ctx = pkg.RnsContext(n, q, p)
    rng = np.random.default_rng(logn)
    # batched: 2 polys of limbs 1..3 of the chain, poly stride with a gap
    x = rand_limbs(rng, chain[1:4], n, (2,))  # [2][3][n]
    stride = 4 * n
    buf = np.zeros((2, 4, n), np.uint64)
    buf[:, :3] = x
    d = dev(torch, buf)
    pkg.call("cbs_rns_ntt_batched", ctx.handle, d.data_ptr(), 2, stride, 3, 1, 0, None)
    torch.cuda.synchronize()
    got = host(d).reshape(2, 4, n)
    want = ntt(o, x, chain[1:4])
    assert np.array_equal(got[:, :3], want)
    assert np.array_equal(got[:, 3], np.zeros((2, n), np.uint64))  # the gap is untouched
    assert ctx.device_fault() == 0
    pkg.call("cbs_rns_ntt_batched", ctx.handle, d.data_ptr(), 2, stride, 3, 1, 1, None)
    torch.cuda.synchronize()
    assert np.array_equal(host(d).reshape(2, 4, n)[:, :3], x)
    # Phantom-form single polynomial over the whole chain, start index 0 and 2
    y = rand_limbs(rng, chain, n)
    dy = dev(torch, y)
    pkg.call("cbs_nwt_2d_radix8_forward_inplace", ctx.handle, dy.data_ptr(), 3, 2, None)
    torch.cuda.synchronize()
    got = host(dy).reshape(5, n)
    assert np.array_equal(got[:2], y[:2])
    assert np.array_equal(got[2:], ntt(o, y[2:], chain[2:]))
    pkg.call("cbs_nwt_2d_radix8_backward_inplace", ctx.handle, dy.data_ptr(), 3, 2, None)
    torch.cuda.synchronize()
    assert np.array_equal(host(dy).reshape(5, n), y)
    ctx.close()


KS_CASES = [  # (logn, size_q, size_p, size_ql, count)
    (13, 5, 2, 5, 3),   # last digit partial
    (13, 5, 2, 4, 1),
    (13, 3, 1, 3, 2),   # alpha = 1
    (14, 6, 3, 5, 2),   # alpha = 3, partial digit
    (13, 4, 2, 1, 5),   # level 1: one digit of one limb
    (12, 3, 2, 3, 2),   # N = 4096: the one-CTA-per-limb transforms
    (10, 4, 1, 4, 3),
]


def _ks_inputs(o, rng, n, q, p, size_ql, count):
    chain = np.concatenate([q, p])
    beta_full = -(-len(q) // len(p))
    ql = q[:size_ql]
    c2 = rand_limbs(rng, ql, n, (count,))  # [count][ql][n]
    ct = rand_limbs(rng, ql, n, (count, 2))  # [count][2][ql][n]
    evk = np.stack([rand_limbs(rng, chain, n, (2,)) for _ in range(beta_full)])  # [beta][2][QP][n]
    return c2, ct, evk


@pytest.mark.parametrize("logn,size_q,size_p,size_ql,count", KS_CASES)
def test_modup_inner_moddown_bit_exact(env, logn, size_q, size_p, size_ql, count):
    pkg, o, torch = env
    n = 1 << logn
    q, p = rns_primes(o, n, size_q, size_p)
    rng = np.random.default_rng(logn * 1000 + size_q * 100 + size_p * 10 + size_ql)
    ctx = pkg.RnsContext(n, q, p)
    c2, ct, evk = _ks_inputs(o, rng, n, q, p, size_ql, count)
    beta = ctx.beta(size_ql)
    qlp = size_ql + size_p
    # modup
    d_c2 = dev(torch, c2)
    d_t = torch.empty((count, beta, qlp, n), dtype=torch.int64, device="cuda")
    pkg.call("cbs_rns_modup", ctx.handle, d_t.data_ptr(), d_c2.data_ptr(), size_ql, count, None)
    torch.cuda.synchronize()
    t_gpu = host(d_t).reshape(count, beta, qlp, n)
    t_ref = np.zeros_like(t_gpu)
    for k in range(count):
        one = np.zeros((beta, qlp, n), np.uint64)
        o.orc_modup(np.ascontiguousarray(c2[k]), one, logn, q, size_ql, p, size_p)
        t_ref[k] = one
    assert np.array_equal(t_gpu, t_ref)
    assert np.array_equal(host(d_c2).reshape(c2.shape), c2)  # input untouched
    # inner product
    d_evk = [dev(torch, evk[b]) for b in range(evk.shape[0])]
    ptrs = pkg.RnsContext.evk_array([t.data_ptr() for t in d_evk])
    d_cx = torch.empty((count, 2, qlp, n), dtype=torch.int64, device="cuda")
    pkg.call("cbs_rns_key_switch_inner_prod", ctx.handle, d_cx.data_ptr(), d_t.data_ptr(), ptrs, size_ql, count,
             None)
    torch.cuda.synchronize()
    cx_gpu = host(d_cx).reshape(count, 2, qlp, n)
    cx_ref = np.zeros_like(cx_gpu)
    for k in range(count):
        one = np.zeros((2, qlp, n), np.uint64)
        o.orc_ks_inner(np.ascontiguousarray(t_ref[k]), np.ascontiguousarray(evk), one, n, q, size_ql, size_q, p,
                       size_p)
        cx_ref[k] = one
    assert np.array_equal(cx_gpu, cx_ref)
    # moddown (overwrite form) over all 2 * count polys
    d_out = torch.zeros((count, 2, size_ql, n), dtype=torch.int64, device="cuda")
    pkg.call("cbs_rns_moddown_from_ntt", ctx.handle, d_out.data_ptr(), d_cx.data_ptr(), size_ql, 2 * count, 0, None)
    torch.cuda.synchronize()
    out_gpu = host(d_out).reshape(count, 2, size_ql, n)
    for k in range(count):
        for j in range(2):
            one = np.zeros((size_ql, n), np.uint64)
            o.orc_moddown(np.ascontiguousarray(cx_ref[k, j]), one, logn, q, size_ql, p, size_p)
            assert np.array_equal(out_gpu[k, j], one)
    # whole keyswitch_inplace, accumulating into ct
    d_ct = dev(torch, ct)
    pkg.call("cbs_rns_keyswitch_inplace", ctx.handle, d_ct.data_ptr(), d_c2.data_ptr(), ptrs, size_ql, count, None)
    torch.cuda.synchronize()
    ct_gpu = host(d_ct).reshape(ct.shape)
    for k in range(count):
        one = np.ascontiguousarray(ct[k]).copy()
        o.orc_keyswitch(one, np.ascontiguousarray(c2[k]), np.ascontiguousarray(evk), logn, q, size_ql, size_q, p,
                        size_p)
        assert np.array_equal(ct_gpu[k], one)
    ctx.close()


def test_keyswitch_decrypts(env):
    """Semantics with a real switching key: ct' = ks(c2) decrypts under s to c2 * s'."""
    pkg, o, torch = env
    n, logn, size_q, size_p, size_ql, count = 1 << 13, 13, 6, 2, 5, 2
    rng = np.random.default_rng(77)
    q, p = rns_primes(o, n, size_q, size_p)
    chain = np.concatenate([q, p])
    s = rng.integers(-1, 2, n)
    sp = rng.integers(-1, 2, n)
    s_ntt = ntt(o, small_to_rns(s, chain), chain)
    sp_ntt = ntt(o, small_to_rns(sp, q), q)
    evk = make_switch_key(o, rng, n, q, p, s_ntt, sp_ntt)
    ctx = pkg.RnsContext(n, q, p)
    ql = q[:size_ql]
    c2 = rand_limbs(rng, ql, n, (count,))
    d_c2 = dev(torch, c2)
    d_ct = torch.zeros((count, 2, size_ql, n), dtype=torch.int64, device="cuda")
    d_evk = [dev(torch, evk[b]) for b in range(evk.shape[0])]
    ptrs = pkg.RnsContext.evk_array([t.data_ptr() for t in d_evk])
    pkg.call("cbs_rns_keyswitch_inplace", ctx.handle, d_ct.data_ptr(), d_c2.data_ptr(), ptrs, size_ql, count, None)
    torch.cuda.synchronize()
    ct = host(d_ct).reshape(count, 2, size_ql, n)
    colq = ql.reshape(-1, 1)
    for k in range(count):
        dec = addmod(ct[k, 0], mulmod(ct[k, 1], s_ntt[:size_ql], colq), colq)
        err = submod(dec, mulmod(c2[k], sp_ntt[:size_ql], colq), colq)
        e = crt_centered(ntt(o, err, ql, inverse=True), ql, 64)
        assert max(abs(v) for v in e) < 2 ** 30
    ctx.close()


@pytest.mark.parametrize("alpha", [2, 8])
def test_keyswitch_phantom_core_size(env, alpha):
    """The Phantom-core configuration: N = 2^16, 24 primes of 50 bits + alpha special primes
    (alpha = 2: beta = 12; alpha = 8: beta = 3), two ciphertexts, bit-exact vs the oracle."""
    pkg, o, torch = env
    n, logn, size_q, count = 1 << 16, 16, 24, 2
    q, p = rns_primes(o, n, size_q, alpha)
    rng = np.random.default_rng(2024 + alpha)
    ctx = pkg.RnsContext(n, q, p)
    c2, ct, evk = _ks_inputs(o, rng, n, q, p, size_q, count)
    d_c2, d_ct = dev(torch, c2), dev(torch, ct)
    d_evk = [dev(torch, evk[b]) for b in range(evk.shape[0])]
    ptrs = pkg.RnsContext.evk_array([t.data_ptr() for t in d_evk])
    pkg.call("cbs_rns_keyswitch_inplace", ctx.handle, d_ct.data_ptr(), d_c2.data_ptr(), ptrs, size_q, count, None)
    torch.cuda.synchronize()
    ct_gpu = host(d_ct).reshape(ct.shape)
    for k in range(count):
        one = np.ascontiguousarray(ct[k]).copy()
        o.orc_keyswitch(one, np.ascontiguousarray(c2[k]), np.ascontiguousarray(evk), logn, q, size_q, size_q, p,
                        alpha)
        assert np.array_equal(ct_gpu[k], one)
    ctx.close()


def test_keyswitch_phantom_core_batch32(env):
    """Config 2 at its full batch: 32 ciphertexts of N = 2^16 over 24 primes of 50 bits + 2
    special primes (beta = 12) key-switched in one call, every one bit-exact against the
    oracle (the oracle's per-ciphertext cost, a few seconds on the host, sets the time of this
    test)."""
    pkg, o, torch = env
    n, logn, size_q, alpha, count = 1 << 16, 16, 24, 2, 32
    q, p = rns_primes(o, n, size_q, alpha)
    rng = np.random.default_rng(3232)
    ctx = pkg.RnsContext(n, q, p)
    c2, ct, evk = _ks_inputs(o, rng, n, q, p, size_q, count)
    d_c2, d_ct = dev(torch, c2), dev(torch, ct)
    d_evk = [dev(torch, evk[b]) for b in range(evk.shape[0])]
    ptrs = pkg.RnsContext.evk_array([t.data_ptr() for t in d_evk])
    pkg.call("cbs_rns_keyswitch_inplace", ctx.handle, d_ct.data_ptr(), d_c2.data_ptr(), ptrs, size_q, count, None)
    torch.cuda.synchronize()
    ct_gpu = host(d_ct).reshape(ct.shape)
    del d_c2, d_ct, d_evk
    evk = np.ascontiguousarray(evk)
    for k in range(count):
        one = np.ascontiguousarray(ct[k]).copy()
        o.orc_keyswitch(one, np.ascontiguousarray(c2[k]), evk, logn, q, size_q, size_q, p, alpha)
        assert np.array_equal(ct_gpu[k], one), k
    ctx.close()
