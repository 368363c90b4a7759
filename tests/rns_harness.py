"""Test helpers for the RNS (Phantom) NTT and hybrid key-switching path.

The oracle functions (oracle/oracle.c: orc_rns_ntt, orc_modup, orc_ks_inner, orc_moddown,
orc_keyswitch) are the CPU restatement of src/ntt/fntt_2d.cu, src/rns_bconv.cu:530-828 and
src/eval_key_switch.cu:13-181.  Key generation here is test data only: a switching key for
s' under s in Phantom's hybrid form (evk_b = (-a s + e + P [i in digit b] s', a) over Q+P).
"""
from __future__ import annotations

import ctypes

import numpy as np

from conftest import _U64P

RNS_BITS = 50


def declare_rns(o):
    u32, sz = ctypes.c_uint32, ctypes.c_size_t
    o.orc_rns_ntt.argtypes = [_U64P, sz, u32, u32, _U64P, ctypes.c_int]
    o.orc_modup.argtypes = [_U64P, _U64P, u32, _U64P, u32, _U64P, u32]
    o.orc_ks_inner.argtypes = [_U64P, _U64P, _U64P, u32, _U64P, u32, u32, _U64P, u32]
    o.orc_moddown.argtypes = [_U64P, _U64P, u32, _U64P, u32, _U64P, u32]
    o.orc_keyswitch.argtypes = [_U64P, _U64P, _U64P, u32, _U64P, u32, u32, _U64P, u32]
    return o


def rns_primes(o, n: int, size_q: int, size_p: int, bits: int = RNS_BITS):
    """size_q + size_p distinct NTT primes of `bits` bits (Phantom's get_primes order)."""
    out = np.zeros(size_q + size_p, np.uint64)
    assert o.orc_get_primes(n, bits, size_q + size_p, out) == 0
    return out[:size_q].copy(), out[size_q:].copy()


def mulmod(a, b, q):
    """Elementwise a * b mod q for uint64 arrays (q broadcast per limb)."""
    return ((a.astype(object) * b.astype(object)) % q.astype(object)).astype(np.uint64)


def addmod(a, b, q):
    return ((a.astype(object) + b.astype(object)) % q.astype(object)).astype(np.uint64)


def submod(a, b, q):
    return ((a.astype(object) - b.astype(object)) % q.astype(object)).astype(np.uint64)


def small_to_rns(v, mods):
    """Signed small integer polynomial -> [limbs][N] residues."""
    return np.stack([(v.astype(object) % int(m)).astype(np.uint64) for m in mods])


def ntt(o, x, mods, inverse=False):
    x = np.ascontiguousarray(x, dtype=np.uint64).copy()
    limbs, n = x.shape[-2], x.shape[-1]
    polys = x.size // (limbs * n)
    o.orc_rns_ntt(x, polys, limbs, n.bit_length() - 1, np.ascontiguousarray(mods, dtype=np.uint64),
                  1 if inverse else 0)
    return x


def make_switch_key(o, rng, n, q, p, s_ntt_chain, sp_ntt_q):
    """Hybrid switching key from s' to s: evk [beta_full][2][Q+P][N], NTT domain.
    s_ntt_chain: s in NTT form over the whole chain; sp_ntt_q: s' over the Q primes."""
    size_q, alpha = len(q), len(p)
    chain = np.concatenate([q, p])
    beta = -(-size_q // alpha)
    P = 1
    for pj in p:
        P *= int(pj)
    evk = np.zeros((beta, 2, len(chain), n), np.uint64)
    colq = chain.reshape(-1, 1)
    for b in range(beta):
        a = np.stack([rng.integers(0, int(m), n, dtype=np.uint64) for m in chain])
        e = ntt(o, small_to_rns(rng.integers(-8, 9, n), chain), chain)
        k0 = submod(e, mulmod(a, s_ntt_chain, colq), colq)
        for i in range(alpha * b, min(alpha * (b + 1), size_q)):
            gi = np.uint64(P % int(q[i]))
            k0[i] = addmod(k0[i], mulmod(sp_ntt_q[i], np.full(n, gi, np.uint64), np.full(n, q[i])), np.full(n, q[i]))
        evk[b, 0] = k0
        evk[b, 1] = a
    return evk


def crt_centered(res, mods, count):
    """First `count` coefficients of [limbs][N] residues as centered integers mod prod(mods)."""
    M = 1
    for m in mods:
        M *= int(m)
    out = []
    for c in range(count):
        x = 0
        for i, m in enumerate(mods):
            mi = M // int(m)
            x += int(res[i, c]) * mi * pow(mi, -1, int(m))
        x %= M
        out.append(x - M if x > M // 2 else x)
    return out
