"""Test-side helpers: oracle structs, encryption/decryption in numpy (test-only, uses the
secret keys exported by the product) and small utilities shared by the CBS tests."""
from __future__ import annotations

import ctypes
from types import SimpleNamespace

import numpy as np

from conftest import _U16P, _U32P, _U64P, oracle_primes, oracle_tables


def mb_keys(mb: int) -> int:
    """Grouped keys per group: every non-empty subset (mb = 2, 3), 8 for the staged mb = 4."""
    return 8 if mb == 4 else (1 << mb) - 1


class OrcParams(ctypes.Structure):
    _fields_ = [("N", ctypes.c_uint32), ("log_n", ctypes.c_uint32), ("Q", ctypes.c_uint64), ("n", ctypes.c_uint32),
                ("q_lwe", ctypes.c_uint64), ("base_g", ctypes.c_uint32), ("digits_g", ctypes.c_uint32),
                ("num_lut", ctypes.c_uint32), ("base_cc", ctypes.c_uint32), ("base_ht", ctypes.c_uint32),
                ("digits_ht", ctypes.c_uint32), ("base_ss", ctypes.c_uint32), ("digits_ss", ctypes.c_uint32),
                ("trace_rounds", ctypes.c_uint32)]


class OrcKeys(ctypes.Structure):
    _fields_ = [("rp", ctypes.c_void_p), ("irp", ctypes.c_void_p), ("n_inv", ctypes.c_uint64),
                ("auto_maps", ctypes.c_void_p), ("tv", ctypes.c_void_p), ("gpow", ctypes.c_void_p),
                ("bsk", ctypes.c_void_p), ("ht_key", ctypes.c_void_p), ("ss_key", ctypes.c_void_p)]


def declare_cbs(oracle) -> None:
    vp = ctypes.c_void_p
    u32 = ctypes.c_uint32
    oracle.orc_blind_rotate.argtypes = [vp, vp, vp, vp, u32, u32, vp, ctypes.c_int]
    oracle.orc_blind_rotate_mv.argtypes = [vp, vp, vp, vp, u32, u32, vp]
    oracle.orc_blind_rotate_mb.argtypes = [vp, vp, vp, u32, vp, vp, u32, u32, vp, ctypes.c_int]
    oracle.orc_circuit_bootstrap.argtypes = [vp, vp, vp, vp, u32, u32, vp]
    oracle.orc_trace_schemeswitch.argtypes = [vp, vp, vp, u32, vp]
    oracle.orc_external_product.argtypes = [vp, vp, vp, u32, ctypes.c_uint64, vp, vp, ctypes.c_uint64, u32, u32]
    oracle.orc_lut8x32.argtypes = [vp, vp, vp, u32, ctypes.c_uint64, vp, vp, ctypes.c_uint64, u32, u32]


class OracleCbs:
    """Oracle view of one key set (keeps the numpy buffers alive)."""

    def __init__(self, oracle, p, keys: dict):
        declare_cbs(oracle)
        self.o, self.p, self.k = oracle, p, keys
        N = p.N
        self.rp, self.rps, self.irp, self.irps, self.ninv = oracle_tables(oracle, N, p.Q)
        self.op = OrcParams(N=N, log_n=N.bit_length() - 1, Q=p.Q, n=p.n, q_lwe=p.q_lwe, base_g=p.base_g,
                            digits_g=p.digits_g, num_lut=p.num_lut, base_cc=p.base_cc, base_ht=p.base_ht,
                            digits_ht=p.digits_ht, base_ss=p.base_ss, digits_ss=p.digits_ss,
                            trace_rounds=N.bit_length() - 1 - p.trace_shift)
        self.ok = OrcKeys(rp=self.rp.ctypes.data, irp=self.irp.ctypes.data, n_inv=int(self.ninv[0]),
                          auto_maps=keys["maps"].ctypes.data, tv=keys["tv"].ctypes.data,
                          gpow=keys["gpow"].ctypes.data, bsk=keys["bsk"].ctypes.data, ht_key=keys["ht"].ctypes.data,
                          ss_key=keys["ss"].ctypes.data)

    def br_acc(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        """Finalized one-bit blind rotation [batch][2][N] (NTT domain)."""
        batch, stride = a.shape
        out = np.zeros((batch, 2, self.p.N), np.uint64)
        self.o.orc_blind_rotate(ctypes.byref(self.op), ctypes.byref(self.ok), a.ctypes.data, b.ctypes.data, batch,
                                stride, out.ctypes.data, 1)
        return out

    def br_acc_mb(self, a: np.ndarray, b: np.ndarray, mbk: np.ndarray, mb: int) -> np.ndarray:
        """Finalized multi-bit blind rotation with grouped keys mbk [batch][2][N] (NTT domain)."""
        batch, stride = a.shape
        out = np.zeros((batch, 2, self.p.N), np.uint64)
        mbk = np.ascontiguousarray(mbk, np.uint64)
        self.o.orc_blind_rotate_mb(ctypes.byref(self.op), ctypes.byref(self.ok), mbk.ctypes.data, mb, a.ctypes.data,
                                   b.ctypes.data, batch, stride, out.ctypes.data, 1)
        return out

    def br_acc_lmkcdey(self, a: np.ndarray, b: np.ndarray, lmk: dict, finalize: bool = True) -> np.ndarray:
        """LMKCDEY blind rotation [batch][2][N] (NTT domain) with the keys and maps of
        oracle_lmkcdey_keys."""
        vp, u32 = ctypes.c_void_p, ctypes.c_uint32
        self.o.orc_blind_rotate_lmkcdey.argtypes = [vp, vp, vp, vp, vp, u32, u32, vp, vp, u32, u32, vp, ctypes.c_int]
        batch, stride = a.shape
        a = np.ascontiguousarray(a, np.uint64)
        b = np.ascontiguousarray(b, np.uint64)
        out = np.zeros((batch, 2, self.p.N), np.uint64)
        self.o.orc_blind_rotate_lmkcdey(ctypes.byref(self.op), ctypes.byref(self.ok), lmk["eval"].ctypes.data,
                                        lmk["auto"].ctypes.data, lmk["maps"].ctypes.data, lmk["num_auto_keys"],
                                        lmk.get("window", 0), a.ctypes.data, b.ctypes.data, batch, stride,
                                        out.ctypes.data, int(finalize))
        return out

    def br_mv(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        batch, stride = a.shape
        out = np.zeros((batch, self.p.num_lut, 2, self.p.N), np.uint64)
        self.o.orc_blind_rotate_mv(ctypes.byref(self.op), ctypes.byref(self.ok), a.ctypes.data, b.ctypes.data, batch,
                                   stride, out.ctypes.data)
        return out

    def trace_ss(self, mv: np.ndarray) -> np.ndarray:
        mv = np.ascontiguousarray(mv.reshape(-1, 2, self.p.N))
        out = np.zeros((mv.shape[0], 2, 2, self.p.N), np.uint64)
        self.o.orc_trace_schemeswitch(ctypes.byref(self.op), ctypes.byref(self.ok), mv.ctypes.data, mv.shape[0],
                                      out.ctypes.data)
        return out

    def lut(self, table: np.ndarray, ctrls: list[np.ndarray]) -> np.ndarray:
        out = np.zeros((2, self.p.N), np.uint64)
        ptrs = (ctypes.c_void_p * 8)(*[c.ctypes.data for c in ctrls])
        self.o.orc_lut8x32(table.ctypes.data, ptrs, out.ctypes.data, self.p.N, self.p.Q, self.rp.ctypes.data,
                           self.irp.ctypes.data, int(self.ninv[0]), self.p.base_cc, self.p.num_lut)
        return out

    def extract(self, words_coef: np.ndarray, info: np.ndarray):
        p = self.p
        T = len(info)
        out_a = np.zeros((T, p.n), np.uint64)
        out_b = np.zeros(T, np.uint64)
        self.o.orc_extract_keyswitch(np.ascontiguousarray(words_coef, np.uint64), info.astype(np.uint32), T, p.N, p.Q,
                                     np.ascontiguousarray(self.k["ksk"]), p.n, int(p.base_ks).bit_length() - 1, p.qks,
                                     p.q_lwe, out_a, out_b, p.n)
        return out_a, out_b

    # ---- test-only decryption helpers (secret key) ----
    def phase_coef(self, ct: np.ndarray) -> np.ndarray:
        """b - a*s of RLWE ct [2][N] (NTT domain) in the coefficient domain, centered."""
        p = self.p
        N, Q = p.N, p.Q
        s = self.k["s_rlwe"].astype(np.int64) % Q
        s_ntt = s.astype(np.uint64).copy()
        self.o.orc_ntt_forward(s_ntt, 1, N, Q, self.rp)
        a = [int(x) for x in ct[0]]
        b = [int(x) for x in ct[1]]
        sn = [int(x) for x in s_ntt]
        ph = np.array([(bb - aa * ss) % Q for aa, bb, ss in zip(a, b, sn)], dtype=np.uint64)
        self.o.orc_ntt_inverse(ph, 1, N, Q, self.irp, int(self.ninv[0]))
        v = ph.astype(object)
        return np.array([int(x) - Q if int(x) > Q // 2 else int(x) for x in v], dtype=object)

    def to_coef(self, poly_ntt: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(poly_ntt, np.uint64).copy()
        self.o.orc_ntt_inverse(x, 1, self.p.N, self.p.Q, self.irp, int(self.ninv[0]))
        return x


def lwe_encrypt_bits(rng: np.random.Generator, s_lwe: np.ndarray, bits, q: int, sigma: float = 0.5):
    bits = np.asarray(bits)
    n = len(s_lwe)
    a = rng.integers(0, q, size=(len(bits), n), dtype=np.uint64)
    e = np.rint(rng.normal(0, sigma, size=len(bits))).astype(np.int64)
    dot = (a.astype(object) * s_lwe.astype(object)).sum(axis=1)
    b = np.array([(int(d) + int(m) * (q // 2) + int(ee)) % q for d, m, ee in zip(dot, bits, e)], dtype=np.uint64)
    return a, b


def lwe_decrypt_bits(s_lwe: np.ndarray, a: np.ndarray, b: np.ndarray, q: int):
    dot = (a.astype(object) * s_lwe.astype(object)).sum(axis=1)
    ph = [(int(bb) - int(d)) % q for bb, d in zip(b, dot)]
    bits = np.array([((2 * x + q // 2) // q) & 1 for x in ph], dtype=np.uint8)
    err = [min(abs(x - (q // 2) * int(bt)), q - abs(x - (q // 2) * int(bt))) for x, bt in zip(ph, bits)]
    return bits, err


def orc_params(p) -> OrcParams:
    """The oracle's parameter record of a parameter set (any object with the cbs_params fields)."""
    N = p.N
    return OrcParams(N=N, log_n=N.bit_length() - 1, Q=p.Q, n=p.n, q_lwe=p.q_lwe, base_g=p.base_g,
                     digits_g=p.digits_g, num_lut=p.num_lut, base_cc=p.base_cc, base_ht=p.base_ht,
                     digits_ht=p.digits_ht, base_ss=p.base_ss, digits_ss=p.digits_ss,
                     trace_rounds=N.bit_length() - 1 - p.trace_shift)


def oracle_keys(oracle, p, seed: int) -> dict:
    """The key set of seed from the oracle's key generation (same layouts as the product's
    export_keys)."""
    vp = ctypes.c_void_p
    oracle.orc_cbs_keygen.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_uint64] + [vp] * 9
    oracle.orc_cbs_keygen.restype = ctypes.c_int
    N, n, rounds = p.N, p.n, p.N.bit_length() - 1 - p.trace_shift
    k = {"s_lwe": np.zeros(n, np.int32), "s_rlwe": np.zeros(N, np.int32),
         "bsk": np.zeros((n, 2 * p.digits_g, 2, N), np.uint64),
         "ht": np.zeros((rounds, p.digits_ht, 2, N), np.uint64), "ss": np.zeros((p.digits_ss, 2, N), np.uint64),
         "ksk": np.zeros((2, N, p.base_ks, n + 1), np.uint16), "tv": np.zeros(N, np.uint64),
         "gpow": np.zeros(p.num_lut, np.uint64), "maps": np.zeros((rounds, N), np.uint32)}
    op = orc_params(p)
    st = oracle.orc_cbs_keygen(ctypes.byref(op), p.sigma_lwe, p.sigma_rlwe, p.qks, p.base_ks, seed,
                               *(k[f].ctypes.data for f in ("s_lwe", "s_rlwe", "bsk", "ht", "ss", "ksk", "tv", "gpow",
                                                            "maps")))
    assert st == 0
    return k


def oracle_params(oracle, preset: str = "3x12") -> SimpleNamespace:
    """The parameter sets of cbs_params_preset restated for the CPU legs, which load nothing from
    the product library (test_oracle_keygen.py pins the values to the product's)."""
    base_g, digits_g = {"3x12": (1 << 12, 3), "2x18": (1 << 18, 2)}[preset]
    return SimpleNamespace(N=2048, Q=oracle_primes(oracle, 2048, 54, 1)[0], n=630, q_lwe=1 << 14, base_g=base_g,
                           digits_g=digits_g, num_lut=4, base_cc=1 << 6, base_ht=1 << 9, digits_ht=5,
                           base_ss=1 << 9, digits_ss=5, trace_shift=0, qks=1 << 14, base_ks=1 << 7, sigma_lwe=0.5,
                           sigma_rlwe=3.19)


# the product seeds a context's grouped keys with the key seed xor this tweak
MB_SEED_TWEAK = 0x6d756c7469626974


def oracle_keys_mb(oracle, p, keys: dict, mb: int, seed: int) -> np.ndarray:
    """Grouped keys [ceil(n/mb)][keys][2 digits_g][2][N] of a key set from the oracle (keys = 3, 7, 8
    for mb = 2, 3, 4), seeded as a context keyed with `seed` seeds them."""
    vp = ctypes.c_void_p
    oracle.orc_cbs_keygen_mb.argtypes = [vp, ctypes.c_double, vp, vp, ctypes.c_uint32, ctypes.c_uint64, vp]
    groups = -(-p.n // mb)
    out = np.zeros((groups, mb_keys(mb), 2 * p.digits_g, 2, p.N), np.uint64)
    op = orc_params(p)
    s_lwe = np.ascontiguousarray(keys["s_lwe"], np.int32)
    s_rlwe = np.ascontiguousarray(keys["s_rlwe"], np.int32)
    oracle.orc_cbs_keygen_mb(ctypes.byref(op), p.sigma_rlwe, s_lwe.ctypes.data, s_rlwe.ctypes.data, mb,
                             seed ^ MB_SEED_TWEAK, out.ctypes.data)
    return out


LMK_SEED_TWEAK = 0x6C6D6B6365797331  # the LMKCDEY keys' generator seed is the key seed xor this


def oracle_lmkcdey_keys(oracle, p, keys: dict, num_auto_keys: int, seed: int, window: int = 0) -> dict:
    """LMKCDEY keys of a key set from the oracle, seeded as a context keyed with `seed` seeds
    them: eval [n][2 digits_g][2][N], auto [keys][digits_g][2][N] (NTT domain), and the NTT-domain
    automorphism maps [keys][N] (keys: 1 + num_auto_keys, or the windowed set)."""
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    oracle.orc_lmkcdey_keygen.argtypes = [vp, ctypes.c_double, vp, vp, u32, u32, ctypes.c_uint64, vp, vp]
    oracle.orc_lmkcdey_auto_maps.argtypes = [u32, u32, u32, vp]
    oracle.orc_lmkcdey_auto_pows.argtypes = [u32, u32, u32, vp]
    oracle.orc_lmkcdey_auto_pows.restype = u32
    count = oracle.orc_lmkcdey_auto_pows(p.N, num_auto_keys, window, None)
    ev = np.zeros((p.n, 2 * p.digits_g, 2, p.N), np.uint64)
    au = np.zeros((count, p.digits_g, 2, p.N), np.uint64)
    maps = np.zeros((count, p.N), np.uint32)
    op = orc_params(p)
    s_lwe = np.ascontiguousarray(keys["s_lwe"], np.int32)
    s_rlwe = np.ascontiguousarray(keys["s_rlwe"], np.int32)
    oracle.orc_lmkcdey_keygen(ctypes.byref(op), p.sigma_rlwe, s_lwe.ctypes.data, s_rlwe.ctypes.data, num_auto_keys,
                              window, seed ^ LMK_SEED_TWEAK, ev.ctypes.data, au.ctypes.data)
    oracle.orc_lmkcdey_auto_maps(p.N, num_auto_keys, window, maps.ctypes.data)
    return {"eval": ev, "auto": au, "maps": maps, "num_auto_keys": num_auto_keys, "window": window}


# a fixed ChaCha20 key for reproducible key-generation tests
RNG_KEY = bytes(range(100, 132))


def oracle_chacha_keys(oracle, p, key: bytes) -> dict:
    """The key set the device key generation draws under the ChaCha20 key `key`, restated by
    the oracle (orc_cbs_keygen_chacha)."""
    vp = ctypes.c_void_p
    oracle.orc_cbs_keygen_chacha.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_uint32, ctypes.c_uint32,
                                             vp, vp, vp, vp, vp, vp, vp]
    oracle.orc_cbs_keygen_chacha.restype = ctypes.c_int
    N, n, rounds = p.N, p.n, p.N.bit_length() - 1 - p.trace_shift
    k = {"s_lwe": np.zeros(n, np.int32), "s_rlwe": np.zeros(N, np.int32),
         "bsk": np.zeros((n, 2 * p.digits_g, 2, N), np.uint64),
         "ht": np.zeros((rounds, p.digits_ht, 2, N), np.uint64), "ss": np.zeros((p.digits_ss, 2, N), np.uint64),
         "ksk": np.zeros((2, N, p.base_ks, n + 1), np.uint16)}
    kw = np.frombuffer(key, np.uint32).copy()
    op = orc_params(p)
    st = oracle.orc_cbs_keygen_chacha(ctypes.byref(op), p.sigma_lwe, p.sigma_rlwe, p.qks, p.base_ks, kw.ctypes.data,
                                      *(k[f].ctypes.data for f in ("s_lwe", "s_rlwe", "bsk", "ht", "ss", "ksk")))
    assert st == 0
    return k
