"""Multi-GPU plumbing of the transcipher: one process per GPU, each an independent replica.

AES-CTR blocks are independent and the keys are read-only, so N GPUs split one CTR stream
with no data-path exchange: rank r of N transciphers the global blocks [r B, (r + 1) B) of
the stream nonce || counter (96-bit nonce, 32-bit big-endian block counter, as in GCM/CTR
usage), each rank with its own context and keys on its own GPU.  The only collectives are
the barrier around the timed region and the max-over-ranks of the step time
(torch.distributed: NCCL on the GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def stream_nonce(seed: int) -> bytes:
    """The 96-bit nonce of the CTR stream of a seed (shared by all ranks)."""
    return np.random.default_rng(seed).bytes(12)


def ctr_blocks(nonce: bytes, first: int, count: int) -> np.ndarray:
    """Counter blocks nonce || be32(first + i), i < count, as [count][16] uint8."""
    if len(nonce) != 12:
        raise ValueError("nonce must be 12 bytes")
    if first < 0 or count < 0 or first + count > 1 << 32:
        raise ValueError("block range outside the 32-bit counter")
    out = np.empty((count, 16), np.uint8)
    out[:, :12] = np.frombuffer(nonce, np.uint8)
    ctr = np.arange(first, first + count, dtype=np.uint64).astype(">u4")
    out[:, 12:] = ctr.view(np.uint8).reshape(count, 4)
    return out


def rank_counters(seed: int, rank: int, world: int, blocks: int) -> np.ndarray:
    """This rank's share of the global stream: blocks [rank * blocks, (rank + 1) * blocks)."""
    if not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    return ctr_blocks(stream_nonce(seed), rank * blocks, blocks)


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The maximum of `value` over all ranks (identity at world = 1)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def whole_job_rate(world: int, units_per_rank: int, ms_max: float, steps: int = 1) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / (ms_max * 1e-3)
