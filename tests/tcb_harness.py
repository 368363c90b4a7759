"""Helpers for the torus circuit bootstrap with PFKS: oracle declarations, exact RLWE phases
and the RGSW-row error measure used by the tests and the bench."""
from __future__ import annotations

import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from conftest import _U32P, _U64P
from gate_harness import OrcGateParams


def declare_tcb(o):
    u32 = ctypes.c_uint32
    u64 = ctypes.c_uint64
    o.orc_tcb_blind_rotate64.argtypes = [ctypes.POINTER(OrcGateParams), _U64P, _U32P, u32, u64, u64, _U64P]
    o.orc_tcb_pfks.argtypes = [u32, u32, u32, u32, _U32P, _U64P, _U32P]
    o.orc_tcb_blind_rotate64_mb.argtypes = [ctypes.POINTER(OrcGateParams), _U64P, u32, _U32P, u32, u64, u64, _U64P]
    return o


def negacyclic_binary(a, z):
    """a * z mod (X^N + 1) over Z (a int64 vector, z binary), exact."""
    N = len(a)
    out = np.zeros(N, np.int64)
    for j in np.nonzero(z)[0]:
        out[j:] += a[:N - j]
        out[:j] -= a[N - j:]
    return out


def centered(x):
    x = np.asarray(x, np.int64) % (1 << 32)
    return np.where(x >= 1 << 31, x - (1 << 32), x)


def rlwe_phase(row, z):
    """b - a*z of an RLWE [2][N] torus32 row, centred."""
    a = centered(row[0])
    return centered(centered(row[1]) - negacyclic_binary(a, z))


def lwe64_phase_top(ext, z):
    """Phase of a torus64 LWE ext [N+1] under binary z, as a centred value in units of 2^-32."""
    a = ext[:-1].astype(object)
    ph = (int(ext[-1]) - sum(int(x) for x, zz in zip(a, z) if zz)) % (1 << 64)
    ph = ph - (1 << 64) if ph >= 1 << 63 else ph
    return ph / 2 ** 32


def rgsw_row_errors(rgsw, bits, z1, cb_bits, cb_levels):
    """Phase errors of every RGSW row: row 2k+1 should have phase m g_k, row 2k phase -m g_k z1.
    rgsw: [count][levels][2][2][N1]. Returns the errors as one flat int64 array."""
    errs = []
    for i, m in enumerate(int(x) for x in bits):
        for k in range(cb_levels):
            g = 1 << (32 - (k + 1) * cb_bits)
            ph1 = rlwe_phase(rgsw[i, k, 1], z1)
            ph1[0] -= m * g
            ph0 = rlwe_phase(rgsw[i, k, 0], z1) + centered(m * g * z1.astype(np.int64))
            errs.append(centered(ph1))
            errs.append(centered(ph0))
    return np.concatenate(errs)


class OracleTcb:
    def __init__(self, o, p, keys, threads: int = 16):
        self.o, self.p, self.k = o, p, keys
        self.op = OrcGateParams(p.n, p.N2, p.bg2_bits, p.l2, 4, 8)
        self.threads = threads

    def blind_rotate(self, a, b):
        """[count][levels][N2+1] level-2 (torus64) LWEs of m g_k."""
        p = self.p
        bsk = np.ascontiguousarray(self.k["bsk2"])
        jobs = [(i, k) for i in range(len(b)) for k in range(p.cb_levels)]

        def one(job):
            i, k = job
            half = 1 << (64 - (k + 1) * p.cb_bits - 1)
            ext = np.zeros(p.N2 + 1, np.uint64)
            self.o.orc_tcb_blind_rotate64(ctypes.byref(self.op), bsk, np.ascontiguousarray(a[i]), int(b[i]), half,
                                          half, ext)
            return ext

        with ThreadPoolExecutor(self.threads) as ex:
            out = list(ex.map(one, jobs))
        return np.stack(out).reshape(len(b), p.cb_levels, p.N2 + 1)

    def blind_rotate_mb(self, a, b, mbk, mb):
        """Grouped (multi-bit) level-2 blind rotation with keys mbk: [count][levels][N2+1]."""
        p = self.p
        mbk = np.ascontiguousarray(mbk, np.uint64)
        jobs = [(i, k) for i in range(len(b)) for k in range(p.cb_levels)]

        def one(job):
            i, k = job
            half = 1 << (64 - (k + 1) * p.cb_bits - 1)
            ext = np.zeros(p.N2 + 1, np.uint64)
            self.o.orc_tcb_blind_rotate64_mb(ctypes.byref(self.op), mbk, mb, np.ascontiguousarray(a[i]), int(b[i]),
                                             half, half, ext)
            return ext

        with ThreadPoolExecutor(self.threads) as ex:
            out = list(ex.map(one, jobs))
        return np.stack(out).reshape(len(b), p.cb_levels, p.N2 + 1)

    def pfks(self, ext):
        """ext [count][levels][N2+1] -> rgsw [count][levels][2][2][N1]."""
        p = self.p
        key = self.k["pfks"]
        cnt, L = ext.shape[0], ext.shape[1]
        out = np.zeros((cnt, L, 2, 2, p.N1), np.uint32)
        for i in range(cnt):
            for k in range(L):
                for c in range(2):
                    row = np.zeros(2 * p.N1, np.uint32)
                    self.o.orc_tcb_pfks(p.N2, p.N1, p.pfks_base_bits, p.pfks_levels, np.ascontiguousarray(key[c]),
                                        np.ascontiguousarray(ext[i, k]), row)
                    out[i, k, c] = row.reshape(2, p.N1)
        return out
