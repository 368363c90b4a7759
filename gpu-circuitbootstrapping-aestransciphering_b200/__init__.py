"""B200-native bootstrapping / AES-128 transciphering hot path: Python host glue.

The compute lives in ``libcbs_b200.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/cbs_b200.h``).  This module only locates and loads that library with ctypes
and declares argument types; there is no CPU fallback.  If the library is missing the
loader raises, so a missing build can never silently degrade to another path.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT_DIR = PKG_DIR.parent
LIB_PATH = PKG_DIR / "libcbs_b200.so"
HEADER_PATH = ROOT_DIR / "include" / "cbs_b200.h"

_lib: ctypes.CDLL | None = None

c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_vp = ctypes.c_void_p

BR_NTT, BR_FFT64, BR_FFT64_SPLIT = 0, 1, 2
BR_GINX, BR_LMKCDEY = 0, 1

CBS_STATUS = {
    0: "CBS_OK", 1: "CBS_ERR_INVALID_ARG", 2: "CBS_ERR_SHAPE_MISMATCH", 3: "CBS_ERR_OOM",
    4: "CBS_ERR_CUDA", 5: "CBS_ERR_DEVICE_TIMEOUT", 6: "CBS_ERR_UNSUPPORTED", 7: "CBS_ERR_NOT_READY",
}


class CbsError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {CBS_STATUS.get(status, status)}: {msg}")
        self.status = status


class DModulus(ctypes.Structure):
    _fields_ = [("value", ctypes.c_uint64), ("const_ratio", ctypes.c_uint64 * 2)]


class CbsParams(ctypes.Structure):
    """Mirror of cbs_params (include/cbs_b200.h)."""
    _fields_ = [("N", ctypes.c_uint32), ("Q", ctypes.c_uint64), ("n", ctypes.c_uint32), ("q_lwe", ctypes.c_uint64),
                ("base_g", ctypes.c_uint32), ("digits_g", ctypes.c_uint32), ("num_lut", ctypes.c_uint32),
                ("base_cc", ctypes.c_uint32), ("base_ht", ctypes.c_uint32), ("digits_ht", ctypes.c_uint32),
                ("base_ss", ctypes.c_uint32), ("digits_ss", ctypes.c_uint32), ("trace_shift", ctypes.c_uint32),
                ("qks", ctypes.c_uint32), ("base_ks", ctypes.c_uint32), ("sigma_lwe", ctypes.c_double),
                ("sigma_rlwe", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def declared_symbols() -> list[str]:
    """Function names declared in include/cbs_b200.h (the C ABI)."""
    text = HEADER_PATH.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cbs_[a-z0-9_]+)\s*\(", text)))


def _declare(lib: ctypes.CDLL) -> None:
    st = ctypes.c_int
    sz = ctypes.c_size_t
    u32 = ctypes.c_uint32
    u64 = ctypes.c_uint64
    sigs = {
        "cbs_last_error": (ctypes.c_char_p, []),
        "cbs_abi_version": (ctypes.c_int, []),
        "cbs_fnwt_1d_opt_batched": (st, [c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_fnwt_1d_opt_outofplace_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_inwt_1d_opt_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_inwt_1d_opt_outofplace_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_inwt_1d_opt_permute_batched": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, sz, sz, c_vp]),
        "cbs_ntt_tables_host": (st, [u32, u64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_get_primes": (st, [u32, ctypes.c_int, u32, c_vp]),
        "cbs_params_default": (st, [c_vp]),
        "cbs_params_preset": (st, [ctypes.c_int, c_vp]),
        "cbs_context_create": (st, [c_vp, u32, c_vp]),
        "cbs_context_destroy": (st, [c_vp]),
        "cbs_context_stream": (st, [c_vp, c_vp]),
        "cbs_keygen": (st, [c_vp, u64]),
        "cbs_context_set_br_backend": (st, [c_vp, ctypes.c_int]),
        "cbs_context_set_br_multibit": (st, [c_vp, u32]),
        "cbs_context_set_br_method": (st, [c_vp, ctypes.c_int, u32, u32]),
        "cbs_export_lmkcdey_keys": (st, [c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_import_lmkcdey_keys": (st, [c_vp, u32, u32, c_vp, sz, c_vp, sz]),
        "cbs_generate_lmkcdey_keys_host": (st, [c_vp, u64, u32, u32, c_vp, c_vp, c_vp, c_vp]),
        "cbs_lmkcdey_auto_maps_host": (st, [u32, u32, u32, c_vp, c_vp]),
        "cbs_lmkcdey_eval_acc_batch_device": (st, [c_vp, c_vp, u32, c_vp, u32, c_vp]),
        "cbs_export_mb_bsk": (st, [c_vp, c_vp, c_vp]),
        "cbs_generate_mb_bsk_host": (st, [c_vp, u64, u32, c_vp, c_vp]),
        "cbs_split_fft_plan": (st, [c_vp, u32, c_vp, c_vp, c_vp]),
        "cbs_export_keys": (st, [c_vp] + [c_vp] * 9),
        "cbs_import_keys": (st, [c_vp] + [c_vp] * 6),
        "cbs_import_mb_bsk": (st, [c_vp, u32, c_vp, sz]),
        "cbs_generate_keys_host": (st, [c_vp, u64] + [c_vp] * 9),
        "cbs_context_tables": (st, [c_vp] + [c_vp] * 7),
        "cbs_blind_rotate_batch_device": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp, c_vp]),
        "cbs_trace_schemeswitch_device": (st, [c_vp, c_vp, u32, c_vp, c_vp]),
        "cbs_circuit_bootstrap_batch_device": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp, c_vp]),
        "cbs_lut8x32_batch_device": (st, [c_vp, c_vp, u32, c_vp, c_vp, u32, u64, c_vp, u32, c_vp, c_vp]),
        "cbs_cmux_batch_device": (st, [c_vp, c_vp, c_vp, c_vp, u64, u32, c_vp, c_vp]),
        "cbs_circuit_bootstrap_batch": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_context_set_br_schedule": (st, [c_vp, u32]),
        "cbs_keygen_device": (st, [c_vp, c_vp]),
        "cbs_gate_ragged_autotune": (st, [c_vp, c_vp, c_vp]),
        "cbs_autotune_blind_rotation": (st, [c_vp, u32, ctypes.c_char_p, c_vp]),
        "cbs_context_tuned": (st, [c_vp, c_vp]),
        "cbs_extract_keyswitch_device": (st, [c_vp, c_vp, u32, c_vp, u32, c_vp, c_vp, u32, c_vp]),
        "cbs_aes128_setup": (st, [c_vp, c_vp, u64]),
        "cbs_aes128_setup_device": (st, [c_vp, c_vp, c_vp]),
        "cbs_cdt_table_host": (st, [ctypes.c_double, c_vp, u32, c_vp]),
        "cbs_aes128_export_material": (st, [c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_aes128_import_material": (st, [c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_aes128_ctr_transcipher_device": (st, [c_vp, c_vp, u32, c_vp, c_vp, ctypes.c_int, c_vp]),
        "cbs_aes128_ctr_transcipher": (st, [c_vp, c_vp, u32, c_vp, c_vp]),
        "cbs_aes128_ctr_add_ciphertext_device": (st, [c_vp, c_vp, u32, c_vp, c_vp]),
        "cbs_aes128_ctr_transcipher_ciphertext": (st, [c_vp, c_vp, c_vp, u32, c_vp, c_vp]),
        "cbs_lwe_decrypt_bits": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_circuit_bootstrap_noalloc_capacity_words": (sz, []),
        "cbs_circuit_bootstrap_batch_device_noalloc": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp, c_vp]),
        "cbs_gate_params_default": (st, [c_vp]),
        "cbs_gate_context_create": (st, [c_vp, u32, c_vp]),
        "cbs_gate_context_destroy": (st, [c_vp]),
        "cbs_gate_keygen": (st, [c_vp, u64]),
        "cbs_gate_set_multibit": (st, [c_vp, u32]),
        "cbs_gate_set_fft_mode": (st, [c_vp, u32]),
        "cbs_gate_export_mb_bsk": (st, [c_vp, c_vp, c_vp]),
        "cbs_gate_generate_keys_host": (st, [c_vp, u64, c_vp, c_vp, c_vp, c_vp]),
        "cbs_gate_export_keys": (st, [c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_gate_encrypt_bits": (st, [c_vp, c_vp, u32, u64, c_vp, c_vp]),
        "cbs_gate_decrypt_bits": (st, [c_vp, c_vp, c_vp, u32, c_vp]),
        "cbs_gate_eval_batch_device": (st, [c_vp, ctypes.c_int, c_vp, c_vp, c_vp, c_vp, u32, c_vp, c_vp, c_vp]),
        "cbs_gate_bootstrap_batch_device": (st, [c_vp, c_vp, c_vp, u32, c_vp, c_vp, c_vp, c_vp]),
        "cbs_gate_bootstrap_func_batch_device": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp, u64, c_vp, c_vp, c_vp]),
        "cbs_gate_eval_func_batch_device": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp, u32, c_vp, c_vp, c_vp]),
        "cbs_gate_eval_floor_batch_device": (st, [c_vp, c_vp, c_vp, u32, u64, u32, u32, u32, c_vp, c_vp, c_vp]),
        "cbs_gate_eval_sign_batch_device": (st, [c_vp, c_vp, c_vp, u32, u64, u32, u32, ctypes.c_int, c_vp, c_vp,
                                                 c_vp]),
        "cbs_gate_eval_decomp_batch_device": (st, [c_vp, c_vp, c_vp, u32, u64, u32, u32, c_vp, c_vp, c_vp, c_vp]),
        "cbs_tcb_params_default": (st, [c_vp]),
        "cbs_tcb_context_create": (st, [c_vp, u32, c_vp]),
        "cbs_tcb_context_destroy": (st, [c_vp]),
        "cbs_tcb_keygen": (st, [c_vp, u64]),
        "cbs_tcb_set_multibit": (st, [c_vp, u32]),
        "cbs_tcb_export_mb_bsk": (st, [c_vp, c_vp, c_vp]),
        "cbs_tcb_generate_keys_host": (st, [c_vp, u64, c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_tcb_export_keys": (st, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
        "cbs_tcb_encrypt_bits": (st, [c_vp, c_vp, u32, u64, c_vp, c_vp]),
        "cbs_tcb_circuit_bootstrap_device": (st, [c_vp, c_vp, c_vp, u32, c_vp, c_vp, c_vp]),
        "cbs_gate_ragged_plan": (st, [c_vp, c_vp, u32, u32]),
        "cbs_gate_ragged_launch": (st, [c_vp, c_vp]),
        "cbs_rns_context_create": (st, [u32, c_vp, u32, c_vp, u32, c_vp]),
        "cbs_rns_context_destroy": (st, [c_vp]),
        "cbs_rns_device_fault": (st, [c_vp, c_vp, ctypes.c_int]),
        "cbs_ckks_add_inplace": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_ckks_sub_inplace": (st, [c_vp, c_vp, c_vp, u32, u32, ctypes.c_int, c_vp]),
        "cbs_ckks_negate_inplace": (st, [c_vp, c_vp, u32, u32, c_vp]),
        "cbs_ckks_multiply_plain_inplace": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_ckks_multiply_inplace": (st, [c_vp, c_vp, c_vp, u32, c_vp]),
        "cbs_ckks_relinearize_inplace": (st, [c_vp, c_vp, c_vp, u32, c_vp]),
        "cbs_ckks_multiply_and_relin_inplace": (st, [c_vp, c_vp, c_vp, c_vp, u32, c_vp]),
        "cbs_ckks_rescale_to_next": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_ckks_mod_switch_to_next": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_ckks_galois_elt_from_step": (u32, [ctypes.c_int, u32]),
        "cbs_ckks_apply_galois_inplace": (st, [c_vp, c_vp, u32, c_vp, u32, c_vp]),
        "cbs_ckks_rotate_inplace": (st, [c_vp, c_vp, ctypes.c_int, c_vp, u32, c_vp]),
        "cbs_rns_context_tables": (st, [c_vp, c_vp]),
        "cbs_rns_prepare_level": (st, [c_vp, u32]),
        "cbs_nwt_2d_radix8_forward_inplace": (st, [c_vp, c_vp, u32, u32, c_vp]),
        "cbs_nwt_2d_radix8_backward_inplace": (st, [c_vp, c_vp, u32, u32, c_vp]),
        "cbs_rns_ntt_batched": (st, [c_vp, c_vp, u32, u64, u32, u32, ctypes.c_int, c_vp]),
        "cbs_rns_modup": (st, [c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_rns_key_switch_inner_prod": (st, [c_vp, c_vp, c_vp, c_vp, u32, u32, c_vp]),
        "cbs_rns_moddown_from_ntt": (st, [c_vp, c_vp, c_vp, u32, u32, ctypes.c_int, c_vp]),
        "cbs_rns_keyswitch_inplace": (st, [c_vp, c_vp, c_vp, c_vp, u32, u32, c_vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args


def load() -> ctypes.CDLL:
    """Load libcbs_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with build_lib.py (no CPU fallback exists)")
        _lib = ctypes.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def check(status: int, where: str) -> None:
    """Raise CbsError for a non-zero cbs_status."""
    if status != 0:
        lib = load()
        raise CbsError(status, where, lib.cbs_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    """Call a C-ABI entry point and raise on a non-OK status."""
    check(getattr(load(), name)(*args), name)


def default_params() -> CbsParams:
    p = CbsParams()
    call("cbs_params_default", ctypes.byref(p))
    return p


def log2_pfail_gaussian(sigma: float, margin: float) -> float:
    """log2 P(|X| >= margin) for X ~ N(0, sigma^2), i.e. log2 erfc(margin / (sqrt(2) sigma));
    past erfc's underflow, the leading term of its asymptotic expansion."""
    import math
    if sigma <= 0:
        return float("-inf")
    z = margin / sigma
    if z < 37:
        return math.log2(math.erfc(z / math.sqrt(2)))
    return -(z * z / 2) / math.log(2) - math.log2(z * math.sqrt(math.pi / 2))


class TuneChoice(ctypes.Structure):
    """cbs_tune_choice: the blind rotation's tuned grouping and schedule."""
    _fields_ = [("mb", ctypes.c_uint32), ("schedule", ctypes.c_uint32), ("us_per_bootstrap", ctypes.c_double),
                ("batch", ctypes.c_uint32), ("candidates", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


BR_SCHEDULE_AUTO, BR_SCHEDULE_DIGITWISE, BR_SCHEDULE_LOCKSTEP, BR_SCHEDULE_PAIRED = 0, 1, 2, 3

PARAMS_AES_3X12, PARAMS_AES_2X18 = 0, 1
PRESETS = {"3x12": PARAMS_AES_3X12, "2x18": PARAMS_AES_2X18}


def preset_params(name: str) -> CbsParams:
    """A named parameter set: "3x12" (cbs_params_default) or "2x18" (blind-rotation gadget
    2^18 x 2)."""
    p = CbsParams()
    call("cbs_params_preset", PRESETS[name], ctypes.byref(p))
    return p


def generate_lmkcdey_keys_host(params: CbsParams, seed: int, num_auto_keys: int, window: int = 0):
    """LMKCDEY keys (eval [n][2*digits_g][2][N], auto [keys][digits_g][2][N], NTT domain) of the key set
    cbs_keygen(seed) makes, generated on the host."""
    import numpy as np
    ew, aw = ctypes.c_size_t(), ctypes.c_size_t()
    call("cbs_generate_lmkcdey_keys_host", ctypes.byref(params), seed, num_auto_keys, window, None, None,
         ctypes.byref(ew), ctypes.byref(aw))
    ev, au = np.zeros(ew.value, np.uint64), np.zeros(aw.value, np.uint64)
    call("cbs_generate_lmkcdey_keys_host", ctypes.byref(params), seed, num_auto_keys, window, ev.ctypes.data,
         au.ctypes.data, ctypes.byref(ew), ctypes.byref(aw))
    return ev.reshape(params.n, 2 * params.digits_g, 2, params.N), au.reshape(-1, params.digits_g, 2, params.N)


def lmkcdey_auto_maps_host(N: int, num_auto_keys: int, window: int = 0):
    """NTT-domain automorphism maps [keys][N] of the LMKCDEY key set."""
    import numpy as np
    count = ctypes.c_uint32()
    call("cbs_lmkcdey_auto_maps_host", N, num_auto_keys, window, None, ctypes.byref(count))
    out = np.zeros((count.value, N), np.uint32)
    call("cbs_lmkcdey_auto_maps_host", N, num_auto_keys, window, out.ctypes.data, None)
    return out


def split_fft_plan(params: CbsParams, mb: int = 1):
    """(limbs, limb_bits, bound_bits) of the exact split-FFT blind rotation (BR_FFT64_SPLIT) for
    grouping mb (1 or 2)."""
    limbs, lb, bound = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    call("cbs_split_fft_plan", ctypes.byref(params), mb, ctypes.byref(limbs), ctypes.byref(lb), ctypes.byref(bound))
    return limbs.value, lb.value, bound.value


def generate_mb_bsk_host(params: CbsParams, seed: int, mb: int):
    """Grouped blind-rotation keys [ceil(n/mb)][keys][2*digits_g][2][N] (NTT domain; keys = 3, 7, 8
    for mb = 2, 3, 4) of the
    key set cbs_keygen(seed) makes, generated on the host."""
    import numpy as np
    words = ctypes.c_size_t()
    call("cbs_generate_mb_bsk_host", ctypes.byref(params), seed, mb, None, ctypes.byref(words))
    out = np.zeros(words.value, np.uint64)
    call("cbs_generate_mb_bsk_host", ctypes.byref(params), seed, mb, out.ctypes.data, ctypes.byref(words))
    return out


class Context:
    """Owning handle of a cbs_context (the GPUCirBTSContext counterpart)."""

    def __init__(self, params: CbsParams | None = None, max_batch: int = 128):
        self.params = params if params is not None else default_params()
        self.max_batch = max_batch
        self._h = ctypes.c_void_p()
        call("cbs_context_create", ctypes.byref(self.params), max_batch, ctypes.byref(self._h))

    @property
    def handle(self) -> int:
        return self._h.value

    def keygen_device(self, rng_key: bytes | None = None) -> None:
        """Generate every key on the device from ChaCha20 under rng_key (32 bytes; None draws one
        from the operating system)."""
        call("cbs_keygen_device", self._h, rng_key)

    def keygen(self, seed: int) -> None:
        call("cbs_keygen", self._h, seed)

    def close(self) -> None:
        if self._h.value:
            load().cbs_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export_keys(self):
        """Host copies (numpy) of secrets and key material in the reference layouts."""
        out = key_buffers(self.params)
        call("cbs_export_keys", self._h, *(out[k].ctypes.data for k in KEY_FIELDS))
        return out

    def import_keys(self, keys: dict, with_secrets: bool = True) -> None:
        """Load evaluation keys (the dict of export_keys / generate_keys_host) instead of
        keygen; with_secrets=False leaves the context without s_lwe / s_rlwe."""
        import numpy as np
        arr = {k: np.ascontiguousarray(keys[k]) for k in ("bsk", "ht", "ss", "ksk")}
        sec = [None, None]
        if with_secrets:
            sec = [np.ascontiguousarray(keys["s_lwe"], np.int32), np.ascontiguousarray(keys["s_rlwe"], np.int32)]
        call("cbs_import_keys", self._h, *(None if v is None else v.ctypes.data for v in sec),
             *(arr[k].ctypes.data for k in ("bsk", "ht", "ss", "ksk")))

    def import_mb_bsk(self, mb: int, keys) -> None:
        """Grouped keys in the layout of export_mb_bsk (selects mb)."""
        import numpy as np
        keys = np.ascontiguousarray(keys, np.uint64)
        call("cbs_import_mb_bsk", self._h, mb, keys.ctypes.data, keys.size)

    def aes_export_material(self) -> dict:
        """Encrypted AES material of cbs_aes128_setup: tables, rk_words, rk0_a, rk0_b."""
        import numpy as np
        p = self.params
        out = {"tables": np.zeros(8 * 256 * 2 * p.N, np.uint64), "rk_words": np.zeros(11 * 4 * 2 * p.N, np.uint64),
               "rk0_a": np.zeros(128 * p.n, np.uint64), "rk0_b": np.zeros(128, np.uint64)}
        call("cbs_aes128_export_material", self._h, *(out[k].ctypes.data for k in ("tables", "rk_words", "rk0_a",
                                                                                   "rk0_b")))
        return out

    def aes_import_material(self, m: dict) -> None:
        import numpy as np
        arr = [np.ascontiguousarray(m[k], np.uint64) for k in ("tables", "rk_words", "rk0_a", "rk0_b")]
        call("cbs_aes128_import_material", self._h, *(a.ctypes.data for a in arr))

    def set_br_backend(self, backend: int) -> None:
        call("cbs_context_set_br_backend", self._h, backend)

    def autotune(self, batch: int, cache_path: str | None = None) -> dict:
        """Time the blind rotation's groupings / schedules at `batch`, apply and cache the fastest."""
        c = TuneChoice()
        call("cbs_autotune_blind_rotation", self._h, batch, cache_path.encode() if cache_path else None,
             ctypes.byref(c))
        return c.as_dict()

    def tuned(self) -> dict | None:
        """The tuned choice this context holds (from the cache or the last autotune), or None."""
        c = TuneChoice()
        return c.as_dict() if load().cbs_context_tuned(self._h, ctypes.byref(c)) == 0 else None

    def set_br_multibit(self, mb: int) -> None:
        """Blind rotation over groups of mb = 1, 2, 3 or 4 LWE coefficients (FFT backend; mb = 4 is
        the staged grouping: an mb = 3 step, then a one-bit step)."""
        call("cbs_context_set_br_multibit", self._h, mb)

    def set_br_schedule(self, schedule: int) -> None:
        """Two-digit grouped blind-rotation schedule (BR_SCHEDULE_*; AUTO = the tuned one)."""
        call("cbs_context_set_br_schedule", self._h, schedule)

    def set_br_method(self, method: int, num_auto_keys: int = 10, window: int = 0) -> None:
        """Blind-rotation method: BR_GINX (default) or BR_LMKCDEY with automorphism keys for 2N - 5
        and 5^1 .. 5^num_auto_keys, or with window > 1 the windowed key set (NTT backend,
        num_lut = 1, g (digits_g + 1) >= log2 Q)."""
        call("cbs_context_set_br_method", self._h, method, num_auto_keys, window)

    def export_lmkcdey_keys(self):
        """LMKCDEY keys (NTT domain): eval [n][2*digits_g][2][N], auto [1 + num_auto_keys][digits_g][2][N]."""
        import numpy as np
        ew, aw = ctypes.c_size_t(), ctypes.c_size_t()
        call("cbs_export_lmkcdey_keys", self._h, None, None, ctypes.byref(ew), ctypes.byref(aw))
        ev, au = np.zeros(ew.value, np.uint64), np.zeros(aw.value, np.uint64)
        call("cbs_export_lmkcdey_keys", self._h, ev.ctypes.data, au.ctypes.data, ctypes.byref(ew), ctypes.byref(aw))
        p = self.params
        return ev.reshape(p.n, 2 * p.digits_g, 2, p.N), au.reshape(-1, p.digits_g, 2, p.N)

    def import_lmkcdey_keys(self, num_auto_keys: int, eval_keys, auto_keys, window: int = 0) -> None:
        """LMKCDEY keys in the layout of export_lmkcdey_keys (selects the method)."""
        import numpy as np
        ev = np.ascontiguousarray(eval_keys, np.uint64).reshape(-1)
        au = np.ascontiguousarray(auto_keys, np.uint64).reshape(-1)
        call("cbs_import_lmkcdey_keys", self._h, num_auto_keys, window, ev.ctypes.data, ev.size, au.ctypes.data,
             au.size)

    def export_mb_bsk(self):
        """Grouped blind-rotation keys [ceil(n/mb)][keys][2*digits_g][2][N] (NTT domain; keys = 3, 7,
        8 for mb = 2, 3, 4)."""
        import numpy as np
        words = ctypes.c_size_t()
        call("cbs_export_mb_bsk", self._h, None, ctypes.byref(words))
        out = np.zeros(words.value, np.uint64)
        call("cbs_export_mb_bsk", self._h, out.ctypes.data, ctypes.byref(words))
        return out


GATE_OR, GATE_AND, GATE_NOR, GATE_NAND, GATE_XOR, GATE_XNOR = range(6)


class GateParams(ctypes.Structure):
    """Mirror of cbs_gate_params (include/cbs_b200.h)."""
    _fields_ = [("n", ctypes.c_uint32), ("N", ctypes.c_uint32), ("bg_bits", ctypes.c_uint32),
                ("levels", ctypes.c_uint32), ("ks_base_bits", ctypes.c_uint32), ("ks_levels", ctypes.c_uint32),
                ("sigma_lwe", ctypes.c_double), ("sigma_rlwe", ctypes.c_double)]


class GateRequest(ctypes.Structure):
    """Mirror of cbs_gate_request: one request of a ragged batch (device pointers)."""
    _fields_ = [("d_a", ctypes.c_void_p), ("d_b", ctypes.c_void_p), ("d_out_a", ctypes.c_void_p),
                ("d_out_b", ctypes.c_void_p), ("count", ctypes.c_uint32)]


def gate_default_params() -> GateParams:
    p = GateParams()
    call("cbs_gate_params_default", ctypes.byref(p))
    return p


def gate_key_buffers(p: GateParams) -> dict:
    import numpy as np
    base = 1 << p.ks_base_bits
    return dict(s_lwe=np.zeros(p.n, np.int32), z_rlwe=np.zeros(p.N, np.int32),
                bsk=np.zeros((p.n, 2 * p.levels, 2, p.N), np.uint32),
                ksk=np.zeros((p.N, p.ks_levels, base - 1, p.n + 1), np.uint32))


def gate_generate_keys_host(p: GateParams, seed: int) -> dict:
    """Gate-bootstrapping keys on the host only; same keys as GateContext.keygen(seed)."""
    k = gate_key_buffers(p)
    call("cbs_gate_generate_keys_host", ctypes.byref(p), seed, k["s_lwe"].ctypes.data, k["z_rlwe"].ctypes.data,
         k["bsk"].ctypes.data, k["ksk"].ctypes.data)
    return k


class GateContext:
    """Owning handle of a cbs_gate_context (the GPUBinFHEContext counterpart)."""

    def __init__(self, params: GateParams | None = None, max_batch: int = 64):
        self.params = params if params is not None else gate_default_params()
        self.max_batch = max_batch
        self._h = ctypes.c_void_p()
        call("cbs_gate_context_create", ctypes.byref(self.params), max_batch, ctypes.byref(self._h))

    @property
    def handle(self) -> int:
        return self._h.value

    def keygen(self, seed: int) -> None:
        call("cbs_gate_keygen", self._h, seed)

    def set_multibit(self, mb: int) -> None:
        """Blind rotation over groups of mb = 1, 2 or 3 LWE coefficients."""
        call("cbs_gate_set_multibit", self._h, mb)

    FFT_MODES = {"fp64": 0, "fp32-split": 1, "fp32": 2}

    def set_fft_mode(self, mode: str) -> None:
        """External-product arithmetic: "fp64" (exact, default), "fp32-split" (FP32 transforms,
        keys split into a 24-bit and an exact 8-bit limb) or "fp32" (FP32, whole keys)."""
        call("cbs_gate_set_fft_mode", self._h, self.FFT_MODES[mode])

    def export_mb_bsk(self):
        """Grouped keys [ceil(n/mb)][2^mb - 1][2*levels][2][N] (uint32 torus)."""
        import numpy as np
        words = ctypes.c_size_t()
        call("cbs_gate_export_mb_bsk", self._h, None, ctypes.byref(words))
        out = np.zeros(words.value, np.uint32)
        call("cbs_gate_export_mb_bsk", self._h, out.ctypes.data, ctypes.byref(words))
        return out

    def encrypt(self, bits, seed: int):
        import numpy as np
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        a = np.zeros((len(bits), self.params.n), np.uint32)
        b = np.zeros(len(bits), np.uint32)
        call("cbs_gate_encrypt_bits", self._h, bits.ctypes.data, len(bits), seed, a.ctypes.data, b.ctypes.data)
        return a, b

    def decrypt(self, a, b):
        import numpy as np
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        out = np.zeros(len(b), np.uint8)
        call("cbs_gate_decrypt_bits", self._h, a.ctypes.data, b.ctypes.data, len(b), out.ctypes.data)
        return out

    def ragged_plan(self, requests, grid_ctas: int = 0) -> None:
        """requests: sequence of (d_a, d_b, d_out_a, d_out_b, count) device pointers."""
        arr = (GateRequest * max(1, len(requests)))(*[GateRequest(*r) for r in requests])
        call("cbs_gate_ragged_plan", self._h, arr, len(requests), grid_ctas)

    def ragged_autotune(self) -> tuple[int, float]:
        """Time the current plan at each candidate persistent grid, keep the fastest; returns
        (grid CTAs, ms)."""
        g, ms = ctypes.c_uint32(), ctypes.c_double()
        call("cbs_gate_ragged_autotune", self._h, ctypes.byref(g), ctypes.byref(ms))
        return g.value, ms.value

    def ragged_launch(self, stream: int | None = None) -> None:
        call("cbs_gate_ragged_launch", self._h, stream)

    def export_keys(self) -> dict:
        k = gate_key_buffers(self.params)
        call("cbs_gate_export_keys", self._h, k["s_lwe"].ctypes.data, k["z_rlwe"].ctypes.data, k["bsk"].ctypes.data,
             k["ksk"].ctypes.data)
        return k

    def close(self) -> None:
        if self._h.value:
            load().cbs_gate_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TcbParams(ctypes.Structure):
    """Mirror of cbs_tcb_params (include/cbs_b200.h)."""
    _fields_ = [("n", ctypes.c_uint32), ("N2", ctypes.c_uint32), ("bg2_bits", ctypes.c_uint32),
                ("l2", ctypes.c_uint32), ("N1", ctypes.c_uint32), ("cb_bits", ctypes.c_uint32),
                ("cb_levels", ctypes.c_uint32), ("pfks_base_bits", ctypes.c_uint32),
                ("pfks_levels", ctypes.c_uint32), ("sigma_lwe", ctypes.c_double), ("sigma_lvl2", ctypes.c_double),
                ("sigma_lvl1", ctypes.c_double)]


def tcb_default_params() -> TcbParams:
    p = TcbParams()
    call("cbs_tcb_params_default", ctypes.byref(p))
    return p


def tcb_key_buffers(p: TcbParams, with_pfks: bool = True) -> dict:
    import numpy as np
    base = 1 << p.pfks_base_bits
    k = dict(s0=np.zeros(p.n, np.int32), z2=np.zeros(p.N2, np.int32), z1=np.zeros(p.N1, np.int32),
             bsk2=np.zeros((p.n, 2 * p.l2, 2, p.N2), np.uint64))
    k["pfks"] = np.zeros((2, p.N2 + 1, p.pfks_levels, base - 1, 2, p.N1), np.uint32) if with_pfks else None
    return k


def _ptr(a):
    return None if a is None else a.ctypes.data


def tcb_generate_keys_host(p: TcbParams, seed: int, with_pfks: bool = True) -> dict:
    """Torus circuit-bootstrapping keys on the host only; same keys as TcbContext.keygen(seed)."""
    k = tcb_key_buffers(p, with_pfks)
    call("cbs_tcb_generate_keys_host", ctypes.byref(p), seed, *(_ptr(k[x]) for x in ("s0", "z2", "z1", "bsk2", "pfks")))
    return k


class TcbContext:
    """Owning handle of a cbs_tcb_context (torus circuit bootstrapping with PFKS)."""

    def __init__(self, params: TcbParams | None = None, max_batch: int = 64):
        self.params = params if params is not None else tcb_default_params()
        self.max_batch = max_batch
        self._h = ctypes.c_void_p()
        call("cbs_tcb_context_create", ctypes.byref(self.params), max_batch, ctypes.byref(self._h))

    @property
    def handle(self) -> int:
        return self._h.value

    def keygen(self, seed: int) -> None:
        call("cbs_tcb_keygen", self._h, seed)

    def set_multibit(self, mb: int) -> None:
        """Level-2 blind rotation over groups of mb = 1, 2 or 3 LWE coefficients."""
        call("cbs_tcb_set_multibit", self._h, mb)

    def export_mb_bsk(self):
        """Grouped level-2 keys [ceil(n/mb)][2^mb - 1][2*l2][2][N2] (uint64 torus)."""
        import numpy as np
        words = ctypes.c_size_t()
        call("cbs_tcb_export_mb_bsk", self._h, None, ctypes.byref(words))
        out = np.zeros(words.value, np.uint64)
        call("cbs_tcb_export_mb_bsk", self._h, out.ctypes.data, ctypes.byref(words))
        return out

    def encrypt(self, bits, seed: int):
        import numpy as np
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        a = np.zeros((len(bits), self.params.n), np.uint32)
        b = np.zeros(len(bits), np.uint32)
        call("cbs_tcb_encrypt_bits", self._h, bits.ctypes.data, len(bits), seed, a.ctypes.data, b.ctypes.data)
        return a, b

    def export_keys(self, with_pfks: bool = False) -> dict:
        k = tcb_key_buffers(self.params, with_pfks)
        call("cbs_tcb_export_keys", self._h, *(_ptr(k[x]) for x in ("s0", "z2", "z1", "bsk2", "pfks")))
        return k

    def close(self) -> None:
        if self._h.value:
            load().cbs_tcb_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RnsContext:
    """Owning handle of a cbs_rns_context (the PhantomContext counterpart for the NTT and
    key-switching path).  q / p are the Q-chain and special primes."""

    def __init__(self, poly_degree: int, q, p):
        import numpy as np
        self.n = int(poly_degree)
        self.q = np.ascontiguousarray(q, dtype=np.uint64)
        self.p = np.ascontiguousarray(p, dtype=np.uint64)
        self.size_q, self.size_p = len(self.q), len(self.p)
        self._h = ctypes.c_void_p()
        call("cbs_rns_context_create", self.n, self.q.ctypes.data, self.size_q, self.p.ctypes.data, self.size_p,
             ctypes.byref(self._h))

    @property
    def handle(self) -> int:
        return self._h.value

    def device_fault(self, clear: bool = False) -> int:
        """The RNS context's device fault word (0 after correct runs)."""
        v = ctypes.c_uint32()
        call("cbs_rns_device_fault", self._h, ctypes.byref(v), int(clear))
        return v.value

    def beta(self, size_ql: int) -> int:
        return -(-size_ql // self.size_p)

    @staticmethod
    def evk_array(ptrs):
        """Host array of device key pointers (one per digit) for the key-switching calls."""
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        return arr

    def close(self) -> None:
        if self._h.value:
            load().cbs_rns_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KEY_FIELDS = ("s_lwe", "s_rlwe", "bsk", "ht", "ss", "ksk", "tv", "gpow", "maps")


def key_buffers(p: CbsParams) -> dict:
    import numpy as np
    N, n, L = p.N, p.n, p.num_lut
    rounds = N.bit_length() - 1 - p.trace_shift
    return dict(
        s_lwe=np.zeros(n, np.int32), s_rlwe=np.zeros(N, np.int32),
        bsk=np.zeros((n, 2 * p.digits_g, 2, N), np.uint64),
        ht=np.zeros((rounds, p.digits_ht, 2, N), np.uint64), ss=np.zeros((p.digits_ss, 2, N), np.uint64),
        ksk=np.zeros((2, N, p.base_ks, n + 1), np.uint16), tv=np.zeros(N, np.uint64),
        gpow=np.zeros(L, np.uint64), maps=np.zeros((rounds, N), np.uint32))


def generate_keys_host(p: CbsParams, seed: int) -> dict:
    """Key generation on the host only (no device needed); same keys as Context.keygen(seed)."""
    out = key_buffers(p)
    call("cbs_generate_keys_host", ctypes.byref(p), seed, *(out[k].ctypes.data for k in KEY_FIELDS))
    return out
