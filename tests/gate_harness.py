"""Test helpers for the torus-32 gate bootstrap: oracle declarations, numpy encryption and
decryption, and a thread pool around the (single-ciphertext) oracle calls."""
from __future__ import annotations

import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from conftest import _U32P

TRUTH = {0: lambda x, y: x | y, 1: lambda x, y: x & y, 2: lambda x, y: 1 - (x | y), 3: lambda x, y: 1 - (x & y),
         4: lambda x, y: x ^ y, 5: lambda x, y: 1 - (x ^ y)}


class OrcGateParams(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("N", ctypes.c_uint32), ("bg_bits", ctypes.c_uint32),
                ("levels", ctypes.c_uint32), ("ks_base_bits", ctypes.c_uint32), ("ks_levels", ctypes.c_uint32)]


def declare_gate(o):
    u32 = ctypes.c_uint32
    o.orc_gate_combine.argtypes = [ctypes.c_int, _U32P, u32, _U32P, u32, u32, _U32P, ctypes.POINTER(u32)]
    o.orc_gate_blind_rotate.argtypes = [ctypes.POINTER(OrcGateParams), _U32P, _U32P, u32, _U32P]
    o.orc_gate_blind_rotate_tv_mb.argtypes = [ctypes.POINTER(OrcGateParams), _U32P, u32, _U32P, u32, u32, u32, _U32P]
    o.orc_gate_keyswitch.argtypes = [ctypes.POINTER(OrcGateParams), _U32P, _U32P, _U32P]
    return o


def orc_params(p) -> OrcGateParams:
    return OrcGateParams(p.n, p.N, p.bg_bits, p.levels, p.ks_base_bits, p.ks_levels)


def encrypt(rng, s, bits, sigma):
    n = len(s)
    a = rng.integers(0, 2 ** 32, size=(len(bits), n), dtype=np.uint64).astype(np.uint32)
    e = np.round(rng.normal(0, sigma * 2 ** 32, len(bits))).astype(np.int64)
    mu = np.where(np.asarray(bits) == 1, 1 << 29, (1 << 32) - (1 << 29)).astype(np.int64)
    b = (a.astype(np.int64) @ s.astype(np.int64) + e + mu) % (1 << 32)
    return a, b.astype(np.uint32)


def phase(s, a, b):
    ph = (b.astype(np.int64) - a.astype(np.int64) @ s.astype(np.int64)) % (1 << 32)
    return np.where(ph >= 1 << 31, ph - (1 << 32), ph)


def decrypt(s, a, b):
    return (phase(s, a, b) > 0).astype(np.uint8)


class OracleGate:
    def __init__(self, o, p, keys, threads: int = 16):
        self.o, self.p, self.k = o, p, keys
        self.op = orc_params(p)
        self.threads = threads

    def combine(self, gate, a1, b1, a2, b2):
        n = self.p.n
        a = np.zeros((len(b1), n), np.uint32)
        b = np.zeros(len(b1), np.uint32)
        for i in range(len(b1)):
            out_b = ctypes.c_uint32()
            ai = np.zeros(n, np.uint32)
            self.o.orc_gate_combine(gate, np.ascontiguousarray(a1[i]), int(b1[i]), np.ascontiguousarray(a2[i]),
                                    int(b2[i]), n, ai, ctypes.byref(out_b))
            a[i], b[i] = ai, out_b.value
        return a, b

    def blind_rotate(self, a, b):
        N = self.p.N
        bsk = np.ascontiguousarray(self.k["bsk"])

        def one(i):
            ext = np.zeros(N + 1, np.uint32)
            self.o.orc_gate_blind_rotate(ctypes.byref(self.op), bsk, np.ascontiguousarray(a[i]), int(b[i]), ext)
            return ext

        with ThreadPoolExecutor(self.threads) as ex:
            return np.stack(list(ex.map(one, range(len(b)))))

    def blind_rotate_mb(self, a, b, mbk, mb):
        """Grouped (multi-bit) blind rotation with keys mbk, test vector 1/8."""
        N = self.p.N
        mbk = np.ascontiguousarray(mbk, np.uint32)

        def one(i):
            ext = np.zeros(N + 1, np.uint32)
            self.o.orc_gate_blind_rotate_tv_mb(ctypes.byref(self.op), mbk, mb, np.ascontiguousarray(a[i]), int(b[i]),
                                               1 << 29, 0, ext)
            return ext

        with ThreadPoolExecutor(self.threads) as ex:
            return np.stack(list(ex.map(one, range(len(b)))))

    def keyswitch(self, ext):
        n = self.p.n
        ksk = np.ascontiguousarray(self.k["ksk"])
        out = np.zeros((ext.shape[0], n + 1), np.uint32)
        for i in range(ext.shape[0]):
            self.o.orc_gate_keyswitch(ctypes.byref(self.op), ksk, np.ascontiguousarray(ext[i]), out[i])
        return out[:, :n].copy(), out[:, n].copy()


# ---- functional bootstrapping (binfhe-base-scheme-batch.cu:215-712), restated on the oracle ----
# Ciphertexts are (a [count][n], b [count]) of integers mod a power of two, as the reference's
# LWECiphertext carries its modulus; every helper takes and returns the modulus in bits.

def lwe_encrypt_mod(rng, s, phases, bits, sigma_units=1.0):
    """LWE_s of the given phases mod 2^bits (noise sigma_units, in units of the modulus)."""
    Q = 1 << bits
    n = len(s)
    a = rng.integers(0, Q, size=(len(phases), n), dtype=np.uint64)
    e = np.round(rng.normal(0, sigma_units, len(phases))).astype(np.int64)
    b = (a.astype(np.int64) @ s.astype(np.int64) + np.asarray(phases, np.int64) + e) % Q
    return a.astype(np.uint32), b.astype(np.uint32)


def phase_mod(s, a, b, bits):
    return (b.astype(np.int64) - a.astype(np.int64) @ s.astype(np.int64)) % (1 << bits)


def lut_via_function(f, p, q):
    """OpenFHE's GenerateLUTviaFunction: LUT[x] = (q/p) f(floor(x p / q)) mod q."""
    return np.array([(q // p) * (f((x * p) // q, p) % p) % q for x in range(q)], np.uint32)


class OracleGateFunc:
    """The reference's functional evaluators over the oracle's programmable bootstrap."""

    def __init__(self, o, p, keys, threads: int = 16):
        u32 = ctypes.c_uint32
        o.orc_gate_bootstrap_func.argtypes = [ctypes.POINTER(OrcGateParams), _U32P, _U32P, _U32P, u32, u32,
                                              ctypes.c_void_p, u32, _U32P]
        self.o, self.p, self.k, self.threads = o, p, keys, threads
        self.op = orc_params(p)

    def bootstrap(self, a, b, in_bits, lut, f_bits):
        n = self.p.n
        bsk, ksk = np.ascontiguousarray(self.k["bsk"]), np.ascontiguousarray(self.k["ksk"])
        lut = np.ascontiguousarray(np.asarray(lut, np.uint64))

        def one(i):
            out = np.zeros(n + 1, np.uint32)
            self.o.orc_gate_bootstrap_func(ctypes.byref(self.op), bsk, ksk, np.ascontiguousarray(a[i]), int(b[i]),
                                           in_bits, lut.ctypes.data, f_bits, out)
            return out

        with ThreadPoolExecutor(self.threads) as ex:
            outs = np.stack(list(ex.map(one, range(len(b)))))
        return outs[:, :n].copy(), outs[:, n].copy()

    @staticmethod
    def _mask(x, bits):
        return (np.asarray(x, np.uint64) & np.uint64((1 << bits) - 1)).astype(np.uint32)

    def _add(self, a, b, bits, c):
        return self._mask(a, bits), self._mask(b.astype(np.uint64) + np.uint64(c % (1 << 32)), bits)

    def _sub(self, x, y, bits):
        return (self._mask(x[0].astype(np.int64) - y[0].astype(np.int64) + (1 << 32), bits),
                self._mask(x[1].astype(np.int64) - y[1].astype(np.int64) + (1 << 32), bits))

    @staticmethod
    def _round(a, b, from_bits, to_bits):
        sh = from_bits - to_bits

        def r(x):
            x = np.asarray(x, np.uint64)
            y = (x + np.uint64(1 << (sh - 1))) >> np.uint64(sh) if sh else x
            return (y & np.uint64((1 << to_bits) - 1)).astype(np.uint32)

        return r(a), r(b)

    def eval_func(self, a, b, q, lut, beta):
        """EvalFunc (:366-479)."""
        qb = q.bit_length() - 1
        mid = q // 2
        lut = [int(x) for x in lut]
        if lut[0] == q - lut[mid]:
            prop = 0 if all(lut[i] == q - lut[mid + i] for i in range(1, mid)) else 2
        elif lut[0] == lut[mid]:
            prop = 1 if all(lut[i] == lut[mid + i] for i in range(1, mid)) else 2
        else:
            prop = 2
        if prop == 0:
            a1, b1 = self._add(a, b, qb, beta)
            return self.bootstrap(a1, b1, qb, lut[:mid], qb)
        if prop == 2:
            db, dq = qb + 1, 2 * q
            a2, b2 = self._add(a, b, db, beta)
            c3 = self.bootstrap(a2, b2, db, [dq - dq // 4] * (dq // 2), db)
            c3 = self._sub((self._mask(a, db), self._mask(b, db)), c3, db)
            a3, b3 = self._add(c3[0], c3[1], db, beta - (q >> 1))
            a4, b4 = self.bootstrap(a3, b3, db, lut[:q], db)
            return self._mask(a4, qb), self._mask(b4, qb)
        a1, b1 = self._add(a, b, qb, beta)
        c2 = self.bootstrap(a1, b1, qb, [q - q // 4] * mid, qb)
        c2 = self._sub((self._mask(a, qb), self._mask(b, qb)), c2, qb)
        a2, b2 = self._add(c2[0], c2[1], qb, beta - (q >> 2))
        return self.bootstrap(a2, b2, qb, lut[:mid], qb)

    def eval_floor(self, a, b, mod_bits, q_bits, beta):
        """EvalFloor (:481-543)."""
        q, Q = 1 << q_bits, 1 << mod_bits
        c1 = self._add(a, b, mod_bits, beta)
        low = (self._mask(c1[0], q_bits), self._mask(c1[1], q_bits))
        c2 = self.bootstrap(low[0], low[1], q_bits, [Q - (q >> 2)] * (q // 2), mod_bits)
        c1 = self._sub(c1, c2, mod_bits)
        f2 = [(Q - (q >> 1) - v) % Q if v < (q >> 2) else v for v in range(q // 2)]
        low = (self._mask(c1[0], q_bits), self._mask(c1[1], q_bits))
        c3 = self.bootstrap(low[0], low[1], q_bits, f2, mod_bits)
        return self._sub(c1, c3, mod_bits)

    def eval_sign(self, a, b, mod_bits, q_bits, beta, scheme_switch=False):
        """EvalSign (:545-631), one bootstrapping key."""
        beta_bits = beta.bit_length() - 1
        x = (self._mask(a, mod_bits), self._mask(b, mod_bits))
        while mod_bits > q_bits:
            x = self.eval_floor(x[0], x[1], mod_bits, q_bits, beta)
            nxt = mod_bits + 1 + beta_bits - q_bits
            x = self._round(x[0], x[1], mod_bits, nxt)
            mod_bits = nxt
        x = self._add(x[0], x[1], mod_bits, beta)
        q = 1 << q_bits
        f3 = [q - q // 4 if scheme_switch else q // 4] * (1 << (mod_bits - 1))
        out = self.bootstrap(x[0], x[1], mod_bits, f3, q_bits)
        return out if scheme_switch else self._add(out[0], out[1], q_bits, -(q >> 2))

    def eval_decomp(self, a, b, mod_bits, q_bits, beta):
        """EvalDecomp (:633-712): the digits, least significant first, and their moduli (bits)."""
        beta_bits = beta.bit_length() - 1
        x = (self._mask(a, mod_bits), self._mask(b, mod_bits))
        digits = []
        while mod_bits > q_bits:
            digits.append(((self._mask(x[0], q_bits), self._mask(x[1], q_bits)), q_bits))
            x = self.eval_floor(x[0], x[1], mod_bits, q_bits, beta)
            nxt = mod_bits - q_bits + 1 + beta_bits
            x = self._round(x[0], x[1], mod_bits, nxt)
            mod_bits = nxt
        digits.append((x, mod_bits))
        return digits
