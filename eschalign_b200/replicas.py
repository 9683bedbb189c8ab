"""Replicated panels, reads sharded across GPUs (one process per GPU, or
several devices in one process: score_on_devices).

Reads are independent, so the path shards with no collective on the data
path: every rank holds its own copy of the panel and scores a contiguous
slice of the batch.  Slices are balanced by DP cells (read length x panel
bases), not read count.  Results stay in read order: rank r's slice is
[bounds[r], bounds[r + 1]).  Collecting them on one rank (``gather``) is
bookkeeping after the timed work, over torch.distributed.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(lens, world: int) -> np.ndarray:
    """world + 1 read indices cutting `lens` into contiguous slices of about
    equal total length."""
    lens = np.asarray(lens, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    csum = np.concatenate([[0], np.cumsum(lens)])
    total = csum[-1]
    targets = total * np.arange(1, world) / world
    cuts = np.searchsorted(csum, targets, side="left")
    return np.concatenate([[0], np.clip(cuts, 0, lens.size), [lens.size]]).astype(np.int64)


def shard(packed, rank: int, world: int):
    """This rank's slice of a synth.Packed batch, and its first read index."""
    from .synth import Packed
    b = shard_bounds(packed.lens, world)
    lo, hi = int(b[rank]), int(b[rank + 1])
    lens = packed.lens[lo:hi]
    start = int(packed.off[lo]) if hi > lo else 0
    stop = int(packed.off[hi - 1]) + int(packed.lens[hi - 1]) if hi > lo else 0
    off = (packed.off[lo:hi] - start).astype(np.uint64)
    codes = packed.codes[start:stop] if stop > start else np.zeros(1, np.uint8)
    return Packed(codes, off, lens), lo


def score_on_devices(scorers, reads, both_strands: bool = False):
    """The same sharding inside one process: `scorers` are GpuScorers over
    one panel, scoring and mode, one per device (or several on one device);
    `reads` a synth.Packed batch or a (codes, off, lens) tuple.  Each scorer
    takes the cell-balanced slice shard() gives its index and scores it on a
    thread of its own (the library's calls release the interpreter lock, so
    the devices run at once).  Returns (results, ties) in read order, equal
    to one scorer's score_batch over the whole batch, and the slices'
    BatchResults.  No collective: the slices meet in host memory."""
    from concurrent.futures import ThreadPoolExecutor

    from .synth import Packed
    scorers = list(scorers)
    if not scorers:
        raise ValueError("score_on_devices needs at least one scorer")
    if not hasattr(reads, "lens"):
        reads = Packed(*reads)
    world = len(scorers)
    parts = [shard(reads, r, world)[0] for r in range(world)]
    with ThreadPoolExecutor(world) as pool:
        done = list(pool.map(lambda sp: sp[0].score_batch(sp[1].tuple(), both_strands=both_strands),
                             zip(scorers, parts)))
    return (np.concatenate([d.results for d in done]),
            np.concatenate([d.ties for d in done])), done


def gather(results: np.ndarray, ties: np.ndarray, rank: int, world: int, group=None):
    """Concatenate every rank's per-read results (and tie lists) on all ranks
    in read order (torch.distributed all_gather_object; CPU or GPU group)."""
    import torch.distributed as dist
    if world == 1:
        return results, ties
    parts = [None] * world
    dist.all_gather_object(parts, (rank, results, ties), group=group)
    parts.sort(key=lambda p: p[0])
    return (np.concatenate([p[1] for p in parts]), np.concatenate([p[2] for p in parts]))
