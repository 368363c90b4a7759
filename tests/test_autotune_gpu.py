"""The blind-rotation autotuner: it times every grouping (mb = 1, 2, 3, staged 4) and the three schedules of
the two-digit gadget at mb = 2, applies the fastest, writes it to the tuning cache, and a context created
afterwards reads the cache and takes the cached grouping when the FFT64 backend is selected
(unless the caller sets mb)."""
from __future__ import annotations

import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_caches_and_applies(pkg, tmp_path, monkeypatch):
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("CBS_TUNE_CACHE", str(cache))
    p = pkg.preset_params("2x18")
    c = pkg.Context(params=p, max_batch=296)
    try:
        assert c.tuned() is None
        c.keygen(3)
        c.set_br_backend(pkg.BR_FFT64)
        choice = c.autotune(296)
        assert choice["mb"] in (1, 2, 3, 4) and choice["candidates"] == 6 and choice["us_per_bootstrap"] > 0
        assert choice["schedule"] in (pkg.BR_SCHEDULE_DIGITWISE, pkg.BR_SCHEDULE_LOCKSTEP, pkg.BR_SCHEDULE_PAIRED)
        print(f"tuned: {choice}")
        entries = json.loads(cache.read_text())
        assert len(entries) == 1 and entries[0]["mb"] == choice["mb"] and entries[0]["bucket"] == 512
        assert c.tuned()["mb"] == choice["mb"]
    finally:
        c.close()

    c2 = pkg.Context(params=p, max_batch=296)
    try:
        got = c2.tuned()
        assert got is not None and (got["mb"], got["schedule"]) == (choice["mb"], choice["schedule"])
        c2.keygen(3)
        c2.set_br_backend(pkg.BR_FFT64)
        if choice["mb"] > 1:  # the cached grouping is in effect: its grouped keys exist
            mbk = c2.export_mb_bsk()
            groups = -(-p.n // choice["mb"])
            keys = 8 if choice["mb"] == 4 else (1 << choice["mb"]) - 1
            assert np.asarray(mbk).size == groups * keys * 2 * p.digits_g * 2 * p.N
        c2.set_br_multibit(1)  # an explicit choice overrides the cache
        assert pkg.load().cbs_export_mb_bsk(c2.handle, None, pkg.ctypes.byref(pkg.ctypes.c_size_t())) == 7
    finally:
        c2.close()


def test_autotune_needs_fft_backend(pkg, tmp_path):
    c = pkg.Context(params=pkg.preset_params("2x18"), max_batch=8)
    try:
        c.keygen(1)
        st = pkg.load().cbs_autotune_blind_rotation(c.handle, 8, str(tmp_path / "t.json").encode(), None)
        assert st == 6
        c.set_br_backend(pkg.BR_FFT64)
        assert pkg.load().cbs_autotune_blind_rotation(c.handle, 9, None, None) == 1  # above max_batch
    finally:
        c.close()
