"""Sharding a population across ranks (one process per GPU).

Programs are independent, so a population splits into contiguous program
ranges with no exchange during evaluation.  ``evaluate_sharded`` evaluates
the local range with any evaluate function and, when every rank needs the
whole fitness vector (as the engine's selection does), gathers the ranges
with one all_gather over the process group (NCCL between GPUs; gloo on CPU).
"""
from __future__ import annotations

from typing import Callable, Tuple

import numpy as np


def shard_bounds(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous range [lo, hi) of program indices for `rank`; sizes differ
    by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_csr(words: np.ndarray, offsets: np.ndarray, rank: int, world: int):
    """The rank's programs as a standalone CSR population (offsets rebased to 0)."""
    n = offsets.shape[0] - 1
    lo, hi = shard_bounds(n, rank, world)
    w = words[offsets[lo]:offsets[hi]]
    off = offsets[lo:hi + 1] - offsets[lo]
    return np.ascontiguousarray(w), np.ascontiguousarray(off), lo, hi


def evaluate_sharded(evaluate: Callable[[np.ndarray, np.ndarray], np.ndarray], words: np.ndarray,
                     offsets: np.ndarray, rank: int, world: int, gather: bool = True) -> np.ndarray:
    """Evaluate this rank's share; with `gather`, return the full fitness
    vector assembled from every rank (torch.distributed must be initialised)."""
    w, off, lo, hi = shard_csr(words, offsets, rank, world)
    local = np.asarray(evaluate(w, off), dtype=np.float32)
    if not gather or world == 1:
        return local
    import torch
    import torch.distributed as dist
    n = offsets.shape[0] - 1
    sizes = [shard_bounds(n, r, world) for r in range(world)]
    width = max(h - l for l, h in sizes)
    buf = torch.zeros(width, dtype=torch.float32)
    buf[: hi - lo] = torch.from_numpy(local)
    if dist.get_backend() == "nccl":
        buf = buf.cuda()
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return np.concatenate([parts[r][: h - l].cpu().numpy() for r, (l, h) in enumerate(sizes)])
