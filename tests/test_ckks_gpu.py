"""CKKS evaluator operations on the RNS context (csrc/ckks.cu) against the CPU oracle: the
element-wise operations and the tensor product bit-exact against numpy on the same residues,
rescale_to_next bit-exact against a restatement of DRNSTool::divide_and_round_q_last_ntt
(src/rns.cu:1183-1208) built on the oracle's NTT, the Galois slot permutation against a
restatement of PhantomGaloisTool's table (include/galois.cuh:78-91) and apply_galois against the
oracle's keyswitch, and multiply + relinearize + rescale decrypting to the product of the
messages.  50-bit chains run the FP64-pipe products, 59-bit chains the 128-bit integer ones."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle, load_pkg
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


def host(t, shape):
    return t.cpu().numpy().view(np.uint64).reshape(shape)


def rand_limbs(rng, mods, n, lead=()):
    return np.stack([rng.integers(0, int(m), lead + (n,), dtype=np.uint64) for m in mods], axis=len(lead))


@pytest.mark.parametrize("logn,bits", [(12, 50), (13, 50), (13, 59)])
def test_elementwise_and_tensor_bit_exact(env, logn, bits):
    pkg, o, torch = env
    n, size_q, size_ql = 1 << logn, 5, 4
    q, p = rns_primes(o, n, size_q, 2, bits)
    ctx = pkg.RnsContext(n, q, p)
    rng = np.random.default_rng(logn * 7 + bits)
    ql = q[:size_ql]
    col = ql.reshape(1, -1, 1)
    a = rand_limbs(rng, ql, n, (2,))
    b = rand_limbs(rng, ql, n, (2,))
    plain = rand_limbs(rng, ql, n)
    try:
        for name, args, want in [
            ("cbs_ckks_add_inplace", (2, size_ql), addmod(a, b, col)),
            ("cbs_ckks_sub_inplace", (2, size_ql, 0), submod(a, b, col)),
            ("cbs_ckks_sub_inplace", (2, size_ql, 1), submod(b, a, col)),
        ]:
            da, db = dev(torch, a), dev(torch, b)
            pkg.call(name, ctx.handle, da.data_ptr(), db.data_ptr(), *args, None)
            assert np.array_equal(host(da, a.shape), want), name
        da = dev(torch, a)
        pkg.call("cbs_ckks_negate_inplace", ctx.handle, da.data_ptr(), 2, size_ql, None)
        assert np.array_equal(host(da, a.shape), submod(np.zeros_like(a), a, col))
        da, dp = dev(torch, a), dev(torch, plain)
        pkg.call("cbs_ckks_multiply_plain_inplace", ctx.handle, da.data_ptr(), dp.data_ptr(), 2, size_ql, None)
        assert np.array_equal(host(da, a.shape), mulmod(a, plain[None], col))
        # tensor product and square
        c = np.zeros((3, size_ql, n), np.uint64)
        c[:2] = a
        dc, db = dev(torch, c), dev(torch, b)
        pkg.call("cbs_ckks_multiply_inplace", ctx.handle, dc.data_ptr(), db.data_ptr(), size_ql, None)
        colq = ql.reshape(-1, 1)
        want = np.stack([mulmod(a[0], b[0], colq), addmod(mulmod(a[0], b[1], colq), mulmod(a[1], b[0], colq), colq),
                         mulmod(a[1], b[1], colq)])
        assert np.array_equal(host(dc, c.shape), want)
        dc = dev(torch, c)
        pkg.call("cbs_ckks_multiply_inplace", ctx.handle, dc.data_ptr(), dc.data_ptr(), size_ql, None)
        want = np.stack([mulmod(a[0], a[0], colq), addmod(mulmod(a[0], a[1], colq), mulmod(a[1], a[0], colq), colq),
                         mulmod(a[1], a[1], colq)])
        assert np.array_equal(host(dc, c.shape), want)
        # overlapping operands (other than the same pointer) are rejected
        assert pkg.load().cbs_ckks_multiply_inplace(ctx.handle, dc.data_ptr(), dc.data_ptr() + 8 * n, size_ql,
                                                    None) == 1
    finally:
        ctx.close()


def rescale_oracle(o, src, ql):
    """DRNSTool::divide_and_round_q_last_ntt restated on the oracle's NTT: the last limb to the
    coefficient domain, its residues mod the other primes back to the NTT domain, then
    (c_j - that) * q_last^-1 mod q_j."""
    size, limbs, n = src.shape
    qlast = int(ql[-1])
    rest = ql[:-1]
    out = np.zeros((size, limbs - 1, n), np.uint64)
    for k in range(size):
        last = ntt(o, src[k, -1:].copy(), ql[-1:], inverse=True)[0]
        red = np.stack([(last % np.uint64(m)).astype(np.uint64) for m in rest])
        v = ntt(o, red, rest)
        inv = np.array([pow(qlast % int(m), -1, int(m)) for m in rest], dtype=object).reshape(-1, 1)
        out[k] = ((submod(src[k, :-1], v, rest.reshape(-1, 1)).astype(object) * inv) %
                  rest.reshape(-1, 1).astype(object)).astype(np.uint64)
    return out


@pytest.mark.parametrize("logn,bits", [(12, 50), (13, 50), (14, 59)])
def test_rescale_and_mod_switch_bit_exact(env, logn, bits):
    pkg, o, torch = env
    n, size_q, size_ql, size = 1 << logn, 5, 5, 2
    q, p = rns_primes(o, n, size_q, 2, bits)
    ctx = pkg.RnsContext(n, q, p)
    rng = np.random.default_rng(300 + logn)
    ql = q[:size_ql]
    src = rand_limbs(rng, ql, n, (size,))
    try:
        ds = dev(torch, src)
        dd = torch.zeros((size, size_ql - 1, n), dtype=torch.int64, device="cuda")
        pkg.call("cbs_ckks_rescale_to_next", ctx.handle, dd.data_ptr(), ds.data_ptr(), size, size_ql, None)
        assert np.array_equal(host(dd, (size, size_ql - 1, n)), rescale_oracle(o, src, ql))
        assert np.array_equal(host(ds, src.shape), src)  # the source is left as it was
        pkg.call("cbs_ckks_mod_switch_to_next", ctx.handle, dd.data_ptr(), ds.data_ptr(), size, size_ql, None)
        assert np.array_equal(host(dd, (size, size_ql - 1, n)), src[:, :-1])
        assert ctx.device_fault() == 0
    finally:
        ctx.close()


def galois_perm(elt: int, logn: int):
    """PhantomGaloisTool::insert_permutation_table restated: NTT slot j of sigma_elt(p) is slot
    perm[j] of p (bit-reversed evaluation order)."""
    n = 1 << logn

    def rev(x, bits):
        return int(format(x, f"0{bits}b")[::-1], 2)

    out = np.zeros(n, np.int64)
    for i in range(n, 2 * n):
        raw = ((elt * rev(i, logn + 1)) >> 1) & (n - 1)
        out[i - n] = rev(raw, logn)
    return out


def test_galois_element_from_step(env):
    pkg, _, _ = env
    n = 1 << 13
    m = 2 * n
    for step, want in [(0, m - 1), (1, 5), (2, 25), (-1, pow(5, n // 2 - 1, m))]:
        assert pkg.load().cbs_ckks_galois_elt_from_step(step, n) == want
    assert pkg.load().cbs_ckks_galois_elt_from_step(n // 2, n) == 0


@pytest.mark.parametrize("step", [1, -3])
def test_apply_galois_matches_oracle_and_decrypts(env, step):
    pkg, o, torch = env
    n, logn, size_q, size_p, size_ql = 1 << 13, 13, 6, 2, 5
    q, p = rns_primes(o, n, size_q, size_p)
    chain = np.concatenate([q, p])
    rng = np.random.default_rng(500 + step)
    ctx = pkg.RnsContext(n, q, p)
    elt = pkg.load().cbs_ckks_galois_elt_from_step(step, n)
    perm = galois_perm(elt, logn)
    s = rng.integers(-1, 2, n)
    s_ntt = ntt(o, small_to_rns(s, chain), chain)
    sigma_s = s_ntt[:size_q][:, perm]  # sigma(s) in the NTT domain over Q
    gk = make_switch_key(o, rng, n, q, p, s_ntt, sigma_s)
    ql = q[:size_ql]
    colq = ql.reshape(-1, 1)
    # an encryption of a small message m under s
    msg = rng.integers(-1000, 1001, n)
    a = rand_limbs(rng, ql, n)
    e = ntt(o, small_to_rns(rng.integers(-4, 5, n), ql), ql)
    m_ntt = ntt(o, small_to_rns(msg, ql), ql)
    c0 = addmod(submod(e, mulmod(a, s_ntt[:size_ql], colq), colq), m_ntt, colq)
    ct = np.stack([c0, a])
    try:
        dct = dev(torch, ct)
        d_gk = [dev(torch, gk[b]) for b in range(gk.shape[0])]
        ptrs = pkg.RnsContext.evk_array([t.data_ptr() for t in d_gk])
        pkg.call("cbs_ckks_rotate_inplace", ctx.handle, dct.data_ptr(), step, ptrs, size_ql, None)
        got = host(dct, ct.shape)
        # oracle: (sigma(c0), 0) += keyswitch(sigma(c1)) with the same key
        want = np.stack([ct[0][:, perm], np.zeros_like(ct[1])])
        o.orc_keyswitch(want, np.ascontiguousarray(ct[1][:, perm]), np.ascontiguousarray(gk), logn, q, size_ql,
                        size_q, p, size_p)
        assert np.array_equal(got, want)
        # and it decrypts under s to sigma(m): coefficient j of m(X^elt)
        dec = ntt(o, addmod(got[0], mulmod(got[1], s_ntt[:size_ql], colq), colq), ql, inverse=True)
        vals = crt_centered(dec, ql, 64)
        sig = np.zeros(n, dtype=object)
        for i in range(n):
            k = (i * elt) % (2 * n)
            sig[k % n] += msg[i] if k < n else -msg[i]
        assert max(abs(int(vals[j]) - int(sig[j])) for j in range(64)) < 2 ** 24
    finally:
        ctx.close()


def test_multiply_relinearize_rescale_decrypts(env):
    """(Delta u1) (Delta u2) relinearised and rescaled by q_last decrypts to Delta^2 / q_last
    times the negacyclic product u1 u2, within the noise."""
    pkg, o, torch = env
    n, logn, size_q, size_p, size_ql = 1 << 13, 13, 6, 2, 6
    q, p = rns_primes(o, n, size_q, size_p)
    chain = np.concatenate([q, p])
    rng = np.random.default_rng(909)
    ctx = pkg.RnsContext(n, q, p)
    s = rng.integers(-1, 2, n)
    s_ntt = ntt(o, small_to_rns(s, chain), chain)
    s2 = mulmod(s_ntt[:size_q], s_ntt[:size_q], q.reshape(-1, 1))
    rk = make_switch_key(o, rng, n, q, p, s_ntt, s2)
    ql = q[:size_ql]
    colq = ql.reshape(-1, 1)
    delta = 1 << 40
    u1 = rng.integers(-8, 9, n)
    u2 = rng.integers(-8, 9, n)

    def encrypt(u):
        a = rand_limbs(rng, ql, n)
        e = ntt(o, small_to_rns(rng.integers(-4, 5, n), ql), ql)
        m = ntt(o, small_to_rns(u.astype(object) * delta, ql), ql)
        return np.stack([addmod(submod(e, mulmod(a, s_ntt[:size_ql], colq), colq), m, colq), a])

    c = np.zeros((3, size_ql, n), np.uint64)
    c[:2] = encrypt(u1)
    c2 = encrypt(u2)
    try:
        dc, dc2 = dev(torch, c), dev(torch, c2)
        d_rk = [dev(torch, rk[b]) for b in range(rk.shape[0])]
        ptrs = pkg.RnsContext.evk_array([t.data_ptr() for t in d_rk])
        pkg.call("cbs_ckks_multiply_and_relin_inplace", ctx.handle, dc.data_ptr(), dc2.data_ptr(), ptrs, size_ql, None)
        dr = torch.zeros((2, size_ql - 1, n), dtype=torch.int64, device="cuda")
        pkg.call("cbs_ckks_rescale_to_next", ctx.handle, dr.data_ptr(), dc.data_ptr(), 2, size_ql, None)
        res = host(dr, (2, size_ql - 1, n))
        qn = q[:size_ql - 1]
        dec = ntt(o, addmod(res[0], mulmod(res[1], s_ntt[:size_ql - 1], qn.reshape(-1, 1)), qn.reshape(-1, 1)), qn,
                  inverse=True)
        vals = crt_centered(dec, qn, 64)
        scale = delta * delta / int(q[size_ql - 1])
        # the first 64 coefficients of the negacyclic product u1 u2
        exact = [sum((int(u1[i]) * int(u2[(k - i) % n]) * (1 if i <= k else -1)) for i in range(n)) for k in range(64)]
        err = max(abs(vals[k] - scale * exact[k]) for k in range(64))
        assert err < 2 ** 22, err
    finally:
        ctx.close()
