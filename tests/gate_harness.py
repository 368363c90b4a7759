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
