"""Generate the golden fixtures that pin the CPU oracle to the reference's own code.

Runs the reference's host routines compiled from its sources in place (oracle/Makefile,
target ``ref`` -> oracle/_ref/libref_host.so): Phantom's get_primes and NTT tables
(src/host/numth.cu, src/host/ntt.cu) and the example's plaintext AES-128
(bitwise/examples/aes_transcipher/aes128.cuh).  Output: tests/golden/reference_host.json
(digests of the large tables plus their leading entries, full small vectors).

Usage:  make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import hashlib
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF_SO = ROOT / "oracle" / "_ref" / "libref_host.so"

PRIME_CASES = [(1024, 30, 2), (2048, 54, 3), (4096, 50, 3), (4096, 60, 2), (65536, 50, 26)]
AES_SEED = 20241203
AES_CASES = 32


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    lib = ctypes.CDLL(str(REF_SO))
    u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    lib.ref_get_primes.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32, u64p]
    lib.ref_ntt_tables.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u64p, u64p, u64p, u64p, u64p]
    lib.ref_modulus_ratio.argtypes = [ctypes.c_uint64, u64p]
    lib.ref_aes_enc_tables.argtypes = [u32p]

    out: dict = {"source": "reference host code (oracle/_ref/libref_host.so)", "primes": [], "ntt_tables": [],
                 "aes": {}}
    for n, bits, count in PRIME_CASES:
        p = np.zeros(count, np.uint64)
        assert lib.ref_get_primes(n, bits, count, p) == 0
        out["primes"].append({"ntt_size": n, "bits": bits, "count": count, "values": [int(x) for x in p]})

    table_cases = [(1024, out["primes"][0]["values"][0]), (2048, out["primes"][1]["values"][0])]
    table_cases += [(4096, q) for q in out["primes"][2]["values"]]
    table_cases += [(65536, q) for q in out["primes"][4]["values"][:2]]
    for n, q in table_cases:
        arrs = [np.zeros(n, np.uint64) for _ in range(4)]
        ninv = np.zeros(2, np.uint64)
        assert lib.ref_ntt_tables(n.bit_length() - 1, q, *arrs, ninv) == 0
        ratio = np.zeros(2, np.uint64)
        lib.ref_modulus_ratio(q, ratio)
        out["ntt_tables"].append({
            "n": n, "q": int(q),
            "sha256": {k: sha(a) for k, a in zip(("rp", "rp_shoup", "irp", "irp_shoup"), arrs)},
            "head": {k: [int(x) for x in a[:8]] for k, a in zip(("rp", "rp_shoup", "irp", "irp_shoup"), arrs)},
            "n_inv": [int(ninv[0]), int(ninv[1])],
            "const_ratio": [int(ratio[0]), int(ratio[1])],
        })

    te = np.zeros(8 * 256, np.uint32)
    lib.ref_aes_enc_tables(te)
    rng = np.random.default_rng(AES_SEED)
    cases = []
    fips_key = bytes(range(16))
    fips_pt = bytes.fromhex("00112233445566778899aabbccddeeff")
    pairs = [(fips_key, fips_pt)] + [(rng.bytes(16), rng.bytes(16)) for _ in range(AES_CASES)]
    for key, pt in pairs:
        ct = ctypes.create_string_buffer(16)
        lib.ref_aes128_encrypt(key, pt, ct)
        rk = ctypes.create_string_buffer(176)
        lib.ref_aes128_key_expand(key, rk)
        cases.append({"key": key.hex(), "pt": pt.hex(), "ct": ct.raw.hex(), "round_keys": rk.raw.hex()})
    out["aes"] = {"enc_tables": [int(x) for x in te], "cases": cases}

    (HERE / "reference_host.json").write_text(json.dumps(out, indent=1))
    print("wrote", HERE / "reference_host.json")


if __name__ == "__main__":
    main()
