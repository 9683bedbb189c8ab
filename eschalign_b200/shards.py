"""Panel shards across GPUs, for panels too large to score on one GPU in
time (one process per GPU).

Where the reads are few and the panel large (a C3-scale panel of 10 000
references), replicas give each GPU the whole panel; here each rank holds a
contiguous range of references instead (balanced by bases), scores every
read against it, and the per-read results -- best, XS, tie count and the
first ties, as mapper.rs:444-472 reduces them -- are merged in one
exchange: an all-gather of the compact per-read states over the process
group (NCCL over NVLink for GPU tensors, gloo on CPU), then the library's
host-side merge (esg_merge_read_results) in rank order.  Candidate numbers
are made global ((reference << 1) | reverse, panel order) before the
exchange, so the merged tie lists are in the reference's candidate order.
No remote memory is read by a kernel; the exchange is the only collective.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native
from .scorer import RESULT_DTYPE, BatchResult, GpuScorer, _check, _ptr

NO_TIE = 0xFFFFFFFF


def shard_ranges(ref_lens, world: int):
    """world contiguous reference ranges [lo, hi) of about equal bases, each
    with at least one reference."""
    lens = np.asarray(ref_lens, dtype=np.int64)
    if world < 1 or world > lens.size:
        raise ValueError(f"{world} shards of {lens.size} references")
    csum = np.concatenate([[0], np.cumsum(lens)])
    cuts = [0]
    for k in range(1, world):
        c = int(np.searchsorted(csum, csum[-1] * k / world, side="left"))
        c = min(max(c, cuts[-1] + 1), lens.size - (world - k))
        cuts.append(c)
    cuts.append(lens.size)
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


def globalize_ties(ties: np.ndarray, base: int) -> np.ndarray:
    """Shard-local candidates (ref << 1 | reverse) to panel-wide ones."""
    t = np.array(ties, dtype=np.uint32, copy=True)
    listed = t != NO_TIE
    t[listed] += np.uint32(base << 1)
    return t


def merge(parts, cap: int):
    """Merge [(results, ties)] over disjoint candidate sets, in order, with
    the library's esg_merge_read_results.  Returns (results, ties)."""
    lib = _native.load()
    res = np.ascontiguousarray(parts[0][0], dtype=RESULT_DTYPE).copy()
    ties = np.ascontiguousarray(parts[0][1], dtype=np.uint32).copy()
    for r2, t2 in parts[1:]:
        r2 = np.ascontiguousarray(r2, dtype=RESULT_DTYPE)
        t2 = np.ascontiguousarray(t2, dtype=np.uint32)
        _check(lib, lib.esg_merge_read_results(res.ctypes.data, _ptr(ties, C.c_uint32),
                                               r2.ctypes.data, _ptr(t2, C.c_uint32), res.size,
                                               cap, res.ctypes.data, _ptr(ties, C.c_uint32)))
    return res, ties


def exchange(results: np.ndarray, ties: np.ndarray, world: int, group=None, device=None):
    """All-gather every rank's per-read states (results as 4 int32, ties as
    int32 words) in one collective; returns [(results, ties)] in rank order.
    `device`: a CUDA device for an NCCL group, None for gloo."""
    import torch
    import torch.distributed as dist
    n, cap = ties.shape
    packed = np.concatenate([np.ascontiguousarray(results).view(np.int32).reshape(n, 4),
                             ties.view(np.int32)], axis=1)
    t = torch.from_numpy(np.ascontiguousarray(packed))
    if device is not None:
        t = t.to(device)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    parts = []
    for o in outs:
        a = o.cpu().numpy()
        r = np.ascontiguousarray(a[:, :4]).view(RESULT_DTYPE).reshape(n)
        parts.append((r, np.ascontiguousarray(a[:, 4:]).view(np.uint32)))
    return parts


class PanelShards:
    """This rank's shard of a panel: a GpuScorer over its reference range,
    whose results merge with the other ranks' into the whole panel's."""

    def __init__(self, panel, scoring, mode, rank: int, world: int, device: int = 0,
                 tie_capacity: int = 8, group=None, nccl_device=None):
        refs = list(panel)
        self.ranges = shard_ranges([len(r) for r in refs], world)
        self.rank, self.world = rank, world
        self.lo, self.hi = self.ranges[rank]
        self.cap = tie_capacity
        self.n_refs = len(refs)
        self.group = group
        self.nccl_device = nccl_device
        self.scorer = GpuScorer(refs[self.lo:self.hi], scoring, mode, device=device,
                                tie_capacity=tie_capacity)

    def score_local(self, reads, both_strands: bool = False):
        """This shard's per-read results, candidates made panel-wide."""
        r = self.scorer.score_batch(reads, both_strands=both_strands)
        return r.results, globalize_ties(r.ties, self.lo)

    def score_batch(self, reads, both_strands: bool = False) -> BatchResult:
        """Every rank scores its shard, then one exchange and the merge: the
        whole panel's per-read results on every rank."""
        res, ties = self.score_local(reads, both_strands)
        parts = exchange(res, ties, self.world, self.group, self.nccl_device)
        res, ties = merge(parts, self.cap)
        return BatchResult(res, ties, None, self.n_refs, {}, self.cap)

    def close(self):
        self.scorer.close()
