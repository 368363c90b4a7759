"""The allocation-free circuit bootstrapping entry point, for callers that cannot call
cudaMalloc while they bootstrap (inside a stream capture, in latency-bound serving loops,
or under another allocator's memory budget).  Its output must equal the allocating entry
point's on the same inputs, on two calls in a row (the shared scratch keeps the previous
call's contents).  Kept in a file that pytest collects last."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cbs_harness import lwe_encrypt_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _copy_view(view: int, words: int):
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    out = torch.empty(words, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    assert cudart.cudaMemcpy(out.data_ptr(), view, words * 8, 3) == 0
    return out


@pytest.mark.parametrize("backend", ["ntt", "fft64", "fft64_split"])
def test_noalloc_matches_allocating_entry_point(pkg, backend):
    """Every blind-rotation backend: the exact NTT one hands NTT-domain RLWEs to the trace; the
    FFT one hands coefficient-domain RLWEs to the FFT trace, whose row spectra are written into
    the caller's output buffer and converted there to the NTT-domain rows; the exact split-FFT
    one hands NTT-domain RLWEs to the exact trace."""
    lib = pkg.load()
    ctx = pkg.Context(max_batch=32)
    ctx.keygen(5)
    if backend != "ntt":
        ctx.set_br_backend(pkg.BR_FFT64 if backend == "fft64" else pkg.BR_FFT64_SPLIT)
    p = ctx.params
    keys = ctx.export_keys()
    per = p.num_lut * 4 * p.N
    cap = lib.cbs_circuit_bootstrap_noalloc_capacity_words()
    max_batch = cap // (p.num_lut * 2 * p.N)
    assert max_batch >= 8
    rng = np.random.default_rng(12)
    for call, batch in enumerate((8, 5)):  # two calls in a row, the second smaller than the first
        a, b = lwe_encrypt_bits(rng, keys["s_lwe"], rng.integers(0, 2, batch), p.q_lwe)
        da, db = _dev(a), _dev(b)
        view = ctypes.c_void_p()
        pkg.call("cbs_circuit_bootstrap_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), batch, p.n,
                 ctypes.byref(view), None)
        want = _copy_view(view.value, batch * per)
        out = torch.full((batch * per,), -1, dtype=torch.int64, device="cuda")
        pkg.call("cbs_circuit_bootstrap_batch_device_noalloc", ctx.handle, da.data_ptr(), db.data_ptr(), batch, p.n,
                 out.data_ptr(), None)
        torch.cuda.synchronize()
        assert torch.equal(out, want), f"call {call}"
    # beyond the fixed scratch: rejected with a clear error, nothing launched
    too_big = max_batch + 1
    x = torch.zeros(too_big * p.n, dtype=torch.int64, device="cuda")
    st = lib.cbs_circuit_bootstrap_batch_device_noalloc(ctx.handle, x.data_ptr(), x.data_ptr(), too_big, p.n,
                                                        x.data_ptr(), None)
    assert st == 2
    assert b"exceeds the fixed scratch" in lib.cbs_last_error()
    ctx.close()
