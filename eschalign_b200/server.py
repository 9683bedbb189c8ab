"""Serving: a request queue over resident scorers (esg_server_* in the library).

No counterpart in the reference, which scores one stream of batches.  A
:class:`Server` holds resident :class:`~eschalign_b200.scorer.GpuScorer`
panels (one per panel x scoring x mode); a request names one of them and a
strand.  A worker thread per scorer batches the waiting requests
(continuous batching), admits each batch against free device memory and
keeps two batches in flight; results are what ``score_batch`` gives for the
same reads alone.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native
from .scorer import RESULT_DTYPE, BatchResult, GpuError, GpuScorer, _check, _inputs_of, _ptr

BOTH_STRANDS = 1


@dataclass
class Timing:
    queued_ms: float   # submit -> its batch went to the device
    total_ms: float    # submit -> results ready
    batch_reads: int
    batch_requests: int


class Server:
    """esg_server: resident scorers behind one request queue."""

    def __init__(self, scorers, max_batch_reads: int = 0, max_inflight: int = 0,
                 memory_budget: int = 0, memory_headroom: int = 0, max_batch_cells: int = 0):
        self._lib = _native.load()
        self._h = None
        opts = _native.EsgServerOptions(max_batch_reads, max_inflight, memory_budget,
                                        memory_headroom, max_batch_cells)
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_server_new(C.byref(opts), C.byref(h)))
        self._h = h
        self.scorers = list(scorers)
        self.slots = []
        for g in self.scorers:
            slot = C.c_uint32()
            _check(self._lib, self._lib.esg_server_add_scorer(self._h, g._h, C.byref(slot)))
            self.slots.append(slot.value)
        self._pending = {}

    def submit(self, slot: int, reads, both_strands: bool = False) -> int:
        """Queue a request for scorer `slot`; returns its ticket."""
        codes, off, lens = _inputs_of(reads)
        t = C.c_uint64()
        _check(self._lib, self._lib.esg_server_submit(
            self._h, int(slot), _ptr(codes, C.c_uint8), _ptr(off, C.c_uint64),
            _ptr(lens, C.c_uint32), lens.size, BOTH_STRANDS if both_strands else 0, C.byref(t)))
        self._pending[t.value] = (int(slot), int(lens.size))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(BatchResult of the request's reads, Timing).  Raises GpuError with
        kind 'Timeout' when the request is not done in time (wait again)."""
        slot, n = self._pending[ticket]
        cap = self.scorers[slot].cap
        res = np.zeros(n, dtype=RESULT_DTYPE)
        ties = np.zeros((n, cap), dtype=np.uint32)
        tm = _native.EsgRequestTiming()
        st = self._lib.esg_server_wait(self._h, ticket, int(timeout_ms), res.ctypes.data,
                                       _ptr(ties, C.c_uint32), C.byref(tm))
        if st != _TIMEOUT:
            del self._pending[ticket]
        _check(self._lib, st)
        return (BatchResult(res, ties, None, len(self.scorers[slot].panel), {}, cap),
                Timing(tm.queued_ms, tm.total_ms, tm.batch_reads, tm.batch_requests))

    def stats(self) -> dict:
        st = _native.EsgServerStats()
        _check(self._lib, self._lib.esg_server_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def close(self):
        if self._h:
            self._lib.esg_server_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_TIMEOUT = 9  # ESG_ERR_TIMEOUT

__all__ = ["Server", "Timing", "GpuScorer", "GpuError"]
