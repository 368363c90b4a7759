"""The multi-GPU plumbing of the transcipher (replicas.py) on CPU: counter blocks of the
shared CTR stream, each rank's share, and a world_size-2 gloo run in which the ranks' shares
are disjoint and together form the one-rank stream, the max over ranks is the slowest
rank's time, and the whole-job rate counts every rank's blocks."""
from __future__ import annotations

import datetime
import importlib.util
import os
import socket
from pathlib import Path

import numpy as np
import pytest

REPLICAS = Path(__file__).resolve().parents[1] / "gpu-circuitbootstrapping-aestransciphering_b200" / "replicas.py"


def _load():
    spec = importlib.util.spec_from_file_location("cbs_b200_replicas", REPLICAS)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_ctr_blocks_layout():
    rep = _load()
    nonce = bytes(range(12))
    b = rep.ctr_blocks(nonce, 0xfffffffe, 2)
    assert b.shape == (2, 16) and b.dtype == np.uint8
    assert bytes(b[0]) == nonce + bytes([0xff, 0xff, 0xff, 0xfe])
    assert bytes(b[1]) == nonce + bytes([0xff, 0xff, 0xff, 0xff])
    with pytest.raises(ValueError):
        rep.ctr_blocks(nonce, 0xffffffff, 2)  # past the 32-bit counter
    with pytest.raises(ValueError):
        rep.ctr_blocks(nonce[:8], 0, 1)


def test_rank_shares_partition_the_stream():
    rep = _load()
    world, blocks = 4, 5
    parts = [rep.rank_counters(7, r, world, blocks) for r in range(world)]
    whole = rep.ctr_blocks(rep.stream_nonce(7), 0, world * blocks)
    assert np.array_equal(np.concatenate(parts), whole)
    with pytest.raises(ValueError):
        rep.rank_counters(7, world, world, blocks)
    assert rep.max_over_ranks(3.5, 1) == 3.5
    assert rep.whole_job_rate(4, 128, 500.0) == pytest.approx(4 * 128 / 0.5)


def _worker(rank: int, world: int, port: int, outdir: str) -> None:
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rep = _load()
        mine = rep.rank_counters(11, rank, world, 6)
        shares = [None] * world
        dist.all_gather_object(shares, mine.tobytes())
        rep.barrier(world)
        ms = rep.max_over_ranks(100.0 + 10.0 * rank, world)  # rank 1 is the slower one
        if rank == 0:
            np.save(os.path.join(outdir, "shares.npy"), np.frombuffer(b"".join(shares), np.uint8).reshape(-1, 16))
            np.save(os.path.join(outdir, "ms.npy"), np.array([ms]))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    if not torch.distributed.is_available():
        pytest.skip("torch.distributed unavailable")
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    rep = _load()
    shares = np.load(tmp_path / "shares.npy")
    assert np.array_equal(shares, rep.ctr_blocks(rep.stream_nonce(11), 0, world * 6))
    assert len({bytes(r) for r in shares}) == world * 6  # disjoint
    ms = float(np.load(tmp_path / "ms.npy")[0])
    assert ms == 110.0
    assert rep.whole_job_rate(world, 6, ms) == pytest.approx(2 * 6 / 0.110)
