"""Host mirror of eschalign's GPU scorer (crates/eschalign/src/cuda/mod.rs:328-709).

Same names, argument meaning and error behaviour as the Rust ``GpuScorer``:

* :meth:`GpuScorer.new` / :meth:`GpuScorer.new_on_device` lay a panel out on
  a device under one scoring and one mode (cuda/mod.rs:345-443) and raise
  :class:`GpuError` where the reference returns ``Err(GpuError)``;
* :meth:`GpuScorer.score_batch` = :meth:`prepare` + :meth:`submit` +
  :meth:`finish` (cuda/mod.rs:524-708), ``prepare`` touching no device
  state so it can overlap a running batch.

What a batch returns differs by design: the reference hands back a full
``ScoreMatrix`` (mapper.rs:95-139) for the CPU to reduce; here each read's
best score, suboptimal score (XS), tie count and first tie candidates come
back reduced on the device (mapper.rs:444-472), and the full rows only when
asked for.  Every read is scored on the GPU -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _native
from .panel import Panel
from .scoring import Mode, Scoring

NO_SCORE = -(2**31)
RESULT_EMPTY = 1
RESULT_TIES_TRUNCATED = 2
RESULT_RESCORED32 = 4

KERNEL_AUTO = 0
KERNEL_PLAIN32 = 1
KERNEL_INT32 = 2
BOTH_STRANDS = 1
FULL_ROWS = 2

RESULT_DTYPE = np.dtype([("best", "<i4"), ("suboptimal", "<i4"),
                         ("n_tied", "<u4"), ("flags", "<u4")])

_STATUS = {
    1: "Unavailable", 2: "Driver", 3: "ReferenceTooLong", 4: "ScoringInvalid",
    5: "EmptyPanel", 6: "EmptyReference", 7: "BadArgument", 8: "OutOfMemory", 9: "Timeout",
}


class GpuError(RuntimeError):
    """GpuError (cuda/mod.rs:144-153) and the panel/scoring refusals of
    AlignError (error.rs:7-28), with the C status code."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.kind = _STATUS.get(status, "Unknown")
        super().__init__(f"{self.kind}: {message}")


def _check(lib, st: int):
    if st != 0:
        raise GpuError(st, lib.esg_last_error().decode(errors="replace"))


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def pack_reads(reads):
    """A list of code arrays -> contiguous (codes u8, off u64, len u32)."""
    lens = np.fromiter((len(r) for r in reads), dtype=np.uint32, count=len(reads))
    off = np.zeros(len(reads), dtype=np.uint64)
    if len(reads) > 1:
        off[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
    if lens.sum():
        codes = np.concatenate([np.asarray(r, dtype=np.uint8) for r in reads])
    else:
        codes = np.zeros(1, dtype=np.uint8)
    return np.ascontiguousarray(codes), off, lens


def _inputs_of(reads):
    """(codes, off, lens) arrays as the C ABI takes them, from a list of code
    arrays, a Packed-like object or a (codes, off, lens) tuple."""
    if hasattr(reads, "tuple") and callable(reads.tuple):
        reads = reads.tuple()
    if isinstance(reads, tuple) and len(reads) == 3:
        codes, off, lens = reads
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        lens = np.ascontiguousarray(lens, dtype=np.uint32)
        if codes.size == 0:
            codes = np.zeros(1, dtype=np.uint8)
        return codes, off, lens
    return pack_reads(reads)


def device_visible() -> bool:
    """cuda/mod.rs:130-140."""
    lib = _native.load()
    n = C.c_int32(0)
    lib.esg_device_count(C.byref(n))
    return n.value > 0


# Limits beside the reference's (cuda/mod.rs:90-99: MAX_READ_LEN 4096,
# MAX_REF_LEN 3072, MAX_REF_LEN_H2 1536): every non-empty read is scored
# here, and references up to 32 768 bases are taken by both kernels.
MAX_READ_LEN = None
MAX_REF_LEN = 32768
MAX_REF_LEN_H2 = MAX_REF_LEN


def fits_f16(n: int, max_ref_len: int, scoring: Scoring) -> bool:
    """cuda/mod.rs:116-122, for callers that route like the reference: a
    read whose whole DP stays within fp16's exact integers (2048)."""
    k = min(n, max_ref_len)
    m = max(abs(scoring.match_score), abs(scoring.mismatch))
    o, e = abs(scoring.gap_open), abs(scoring.gap_extend)
    return k * m + o + e + o <= 2048


def fits_i16(n: int, max_ref_len: int, scoring: Scoring) -> bool:
    """simd/mod.rs:222-227 (the reference's SIMD/GPU admission bound)."""
    lib = _native.load()
    s = _native.EsgScoring(*scoring.astuple())
    return bool(lib.esg_fits_i16(n, max_ref_len, C.byref(s)))


class ScoreMatrix:
    """mapper.rs:95-139: row-major scores, row k = query k in panel order.
    Every row is scored here (int32, so scores past int16 are kept)."""

    def __init__(self, n_refs: int, scores: np.ndarray, scored: np.ndarray):
        assert scores.shape == (scored.size, n_refs)
        self._n_refs = n_refs
        self.scores = scores
        self.scored = scored

    def __len__(self):
        return self.scored.size

    def n_refs(self) -> int:
        return self._n_refs

    def n_scored(self) -> int:
        return int(self.scored.sum())

    def row(self, k: int):
        return self.scores[k] if self.scored[k] else None


@dataclass
class ReadScores:
    best: int | None
    suboptimal: int | None
    n_tied: int
    ties: list          # (reference, reverse) in tie order, at most tie_capacity
    truncated: bool
    rescored32: bool


class BatchResult:
    """Per-read reduction of one batch (+ optional rows)."""

    def __init__(self, results, ties, rows, n_refs, stats, cap):
        self.results = results
        self.ties = ties
        self.rows = rows
        self.n_refs = n_refs
        self.stats = stats
        self.cap = cap

    def __len__(self):
        return self.results.size

    @property
    def best(self):
        return self.results["best"]

    @property
    def suboptimal(self):
        return self.results["suboptimal"]

    @property
    def n_tied(self):
        return self.results["n_tied"]

    @property
    def flags(self):
        return self.results["flags"]

    def read(self, k: int) -> ReadScores:
        r = self.results[k]
        if r["flags"] & RESULT_EMPTY:
            return ReadScores(None, None, 0, [], False, False)
        n = min(int(r["n_tied"]), self.cap)
        ties = [(int(c) >> 1, bool(int(c) & 1)) for c in self.ties[k, :n]]
        sub = None if r["suboptimal"] == NO_SCORE else int(r["suboptimal"])
        return ReadScores(int(r["best"]), sub, int(r["n_tied"]), ties,
                          bool(r["flags"] & RESULT_TIES_TRUNCATED),
                          bool(r["flags"] & RESULT_RESCORED32))

    def matrix(self) -> ScoreMatrix | None:
        if self.rows is None:
            return None
        return ScoreMatrix(self.n_refs, self.rows, np.ones(self.rows.shape[0], dtype=bool))


class PreparedBatch:
    """cuda/mod.rs:711-728: a batch planned on the host."""

    def __init__(self, scorer, handle, n_reads, flags, keep):
        self._scorer = scorer
        self._h = handle
        self.n_reads = n_reads
        self.flags = flags
        self._keep = keep

    def stats(self) -> dict:
        st = _native.EsgBatchStats()
        _check(self._scorer._lib, self._scorer._lib.esg_batch_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def work_split(self):
        """cuda/mod.rs:723-727: (queries on the int16x2 kernel, on int32)."""
        s = self.stats()
        return s["queries_batched"], s["queries_plain"]

    def free(self):
        if self._h:
            self._scorer._lib.esg_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


PendingBatch = PreparedBatch


PAIR_DTYPE = np.dtype([("best", "<i4"), ("next", "<i4"), ("n_tied", "<u4"), ("flags", "<u4"),
                       ("xs", "<i4", (2,)), ("primary", "<i4", (2,))])


@dataclass
class PairScores:
    """One pair's ranked candidates (pair.rs:195-234): the first tier's
    summed score, its members as (reference, template_reverse), the next
    tier's sum, per-mate XS outside the tier (pair.rs:297-314) and the
    primary's mate scores.  ``best is None``: no eligible candidate, the
    pair falls back to each mate on its own (pair.rs:366-387)."""
    best: int | None
    next: int | None
    n_tied: int
    ties: list
    xs: tuple
    primary: tuple
    truncated: bool
    rescored32: bool


class PairBatchResult:
    """What esg_finish_pairs returns for one paired batch."""

    def __init__(self, pairs, pair_ties, mates: BatchResult, adapters, stats, cap):
        self.pairs = pairs
        self.pair_ties = pair_ties
        self.mates = mates
        self.adapters = adapters
        self.stats = stats
        self.cap = cap

    def __len__(self):
        return self.pairs.size

    def pair(self, p: int) -> PairScores:
        r = self.pairs[p]
        opt = lambda v: None if v == NO_SCORE else int(v)  # noqa: E731
        n = min(int(r["n_tied"]), self.cap)
        ties = [(int(c) >> 1, bool(int(c) & 1)) for c in self.pair_ties[p, :n]]
        return PairScores(opt(r["best"]), opt(r["next"]), int(r["n_tied"]), ties,
                          (opt(r["xs"][0]), opt(r["xs"][1])),
                          (opt(r["primary"][0]), opt(r["primary"][1])),
                          bool(r["flags"] & RESULT_TIES_TRUNCATED),
                          bool(r["flags"] & RESULT_RESCORED32))

    def mate(self, p: int, m: int) -> ReadScores:
        """Mate m (0 or 1) of pair p alone, both strands (the Separate fallback)."""
        return self.mates.read(2 * p + m)


class GpuScorer:
    """A panel resident on a device under one scoring and one mode."""

    def __init__(self, panel: Panel, scoring: Scoring, mode: Mode, device: int = 0,
                 tie_capacity: int = 8, kernel: int = KERNEL_AUTO, stream: int | None = None):
        self._lib = _native.load()
        self._h = None
        if not isinstance(panel, Panel):
            panel = Panel.from_codes(panel)
        self.panel = panel
        self.scoring = scoring
        self.mode = Mode(mode)
        self.cap = int(tie_capacity)
        self.device = int(device)
        codes, off, lens = panel.packed()
        self._panel_arrays = (codes, off, lens)
        self._kernel = int(kernel)
        sc = _native.EsgScoring(*scoring.astuple())
        opts = _native.EsgOptions(self.cap, int(kernel), stream)
        h = C.c_void_p()
        st = self._lib.esg_scorer_new(int(device), _ptr(codes, C.c_uint8), _ptr(off, C.c_uint64),
                                      _ptr(lens, C.c_uint32), len(panel), C.byref(sc),
                                      int(self.mode), C.byref(opts), C.byref(h))
        _check(self._lib, st)
        self._h = h

    # -- cuda/mod.rs:345-350
    @classmethod
    def new(cls, panel, scoring, mode, **kw):
        return cls(panel, scoring, mode, device=0, **kw)

    @classmethod
    def new_on_device(cls, ordinal, panel, scoring, mode, **kw):
        return cls(panel, scoring, mode, device=ordinal, **kw)

    def close(self):
        if self._h:
            self._lib.esg_scorer_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- introspection (cuda/mod.rs:446-514)
    def info(self) -> dict:
        inf = _native.EsgInfo()
        _check(self._lib, self._lib.esg_scorer_info(self._h, C.byref(inf)))
        d = {k: getattr(inf, k) for k, _ in inf._fields_}
        d["device_name"] = inf.device_name.decode()
        return d

    def device_name(self) -> str:
        return self.info()["device_name"]

    # The reference has an int kernel and a half2 "fast" kernel
    # (cuda/mod.rs:452-514); here the plain int32 kernel stands for the
    # first and the batched int16x2 kernel for the second.
    def geometry(self):
        """The int32 kernel's (threads per block, groups, blocks)."""
        i = self.info()
        return (i["plain_threads"], 1, i["plain_blocks"])

    def geometry_h2(self):
        """The batched kernel's (threads per block, reference pairs, persistent
        blocks), or None where the scoring scheme rules it out."""
        i = self.info()
        if not i["batched_ok"]:
            return None
        return (i["batched_threads"], i["n_ref_pairs"], i["batched_blocks"])

    def registers(self):
        return self.info()["regs_plain"]

    def registers_h2(self):
        i = self.info()
        return i["regs_batched"] if i["batched_ok"] else None

    def local_bytes(self):
        return self.info()["local_bytes_plain"]

    def local_bytes_h2(self):
        i = self.info()
        return i["local_bytes_batched"] if i["batched_ok"] else None

    def set_kernel(self, kernel: int):
        _check(self._lib, self._lib.esg_scorer_set_kernel(self._h, int(kernel)))
        self._kernel = int(kernel)

    def set_plain(self, plain: bool):
        """Every query on the plain int32 kernel, or the batched kernel where
        it can take it."""
        self.set_kernel(KERNEL_PLAIN32 if plain else KERNEL_AUTO)

    def half2(self) -> bool:
        """GpuScorer::half2: the fast (batched) kernel is in use."""
        return bool(self.info()["batched_ok"]) and getattr(self, "_kernel", KERNEL_AUTO) == KERNEL_AUTO

    def set_half2(self, enabled: bool):
        """GpuScorer::set_half2 (cuda/mod.rs:500-502): the A/B lever; results
        are the same either way."""
        self.set_plain(not enabled)

    def half2_scores_len(self, n: int) -> bool:
        """GpuScorer::half2_scores_len: a query of n bases goes to the batched
        kernel (else the int32 kernel)."""
        return bool(self._lib.esg_batched_takes(self._h, int(n)))

    def autotune(self, lengths=None) -> dict:
        """Measure the tile shape on this panel (esg_scorer_autotune): the
        16/32-row stripe split, the length from which the int32 lanes take
        over, resident CTAs per SM, the panel-chunk target.  With `lengths`
        (a sample of the workload's read lengths) the split is chosen on a
        batch of that length histogram (esg_scorer_autotune_lengths)."""
        rep = _native.EsgTuneReport()
        if lengths is None:
            _check(self._lib, self._lib.esg_scorer_autotune(self._h, C.byref(rep)))
        else:
            lens = np.ascontiguousarray(lengths, dtype=np.uint32)
            _check(self._lib, self._lib.esg_scorer_autotune_lengths(
                self._h, _ptr(lens, C.c_uint32), int(lens.size), C.byref(rep)))
        n = rep.n_lengths

        def ms(a, k):
            return [round(v, 3) for v in a[:k]]

        return {"split_len": rep.split_len, "lengths": list(rep.lengths[:n]),
                "ms_rows16": ms(rep.ms_rows16, n), "ms_rows32": ms(rep.ms_rows32, n),
                "ms_int32": ms(rep.ms_int32, n), "int32_from": rep.int32_from,
                "ctas16": {"tried": list(rep.cand_ctas16[:rep.n_ctas16]),
                           "ms": ms(rep.ms_ctas16, rep.n_ctas16), "chosen": rep.ctas16},
                "ctas32": {"tried": list(rep.cand_ctas32[:rep.n_ctas32]),
                           "ms": ms(rep.ms_ctas32, rep.n_ctas32), "chosen": rep.ctas32},
                "chunk_target": {"tried": list(rep.chunk_targets[:rep.n_chunk_targets]),
                                 "ms": ms(rep.ms_chunks, rep.n_chunk_targets),
                                 "chosen": rep.chunk_target},
                "split_on_histogram": {"tried": list(rep.splits[:rep.n_splits]),
                                       "ms": ms(rep.ms_splits, rep.n_splits)}}

    def set_split(self, split_len: int):
        _check(self._lib, self._lib.esg_scorer_set_split(self._h, int(split_len)))

    def set_graphs(self, enabled: bool):
        """Launch each batch's device work as one CUDA graph (default) or
        kernel by kernel; results are the same."""
        _check(self._lib, self._lib.esg_scorer_set_graphs(self._h, int(bool(enabled))))

    def set_chunking(self, max_chunks: int):
        """Cap the panel chunks per tile (1: every task walks the whole panel)."""
        _check(self._lib, self._lib.esg_scorer_set_chunking(self._h, int(max_chunks)))

    def scores_len(self, n: int) -> bool:
        return bool(self._lib.esg_scores_len(self._h, n))

    # -- batches
    @staticmethod
    def _inputs(reads):
        return _inputs_of(reads)

    def prepare(self, reads, both_strands: bool = False, full_rows: bool = False) -> PreparedBatch:
        codes, off, lens = self._inputs(reads)
        flags = (BOTH_STRANDS if both_strands else 0) | (FULL_ROWS if full_rows else 0)
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_prepare(self._h, _ptr(codes, C.c_uint8),
                                                _ptr(off, C.c_uint64), _ptr(lens, C.c_uint32),
                                                lens.size, flags, C.byref(h)))
        pb = PreparedBatch(self, h, int(lens.size), flags, None)
        pb.lens = lens
        return pb

    def submit(self, batch: PreparedBatch) -> PendingBatch:
        _check(self._lib, self._lib.esg_submit(self._h, batch._h))
        return batch

    def relaunch(self, batch: PendingBatch, stream: int | None = None):
        _check(self._lib, self._lib.esg_relaunch(self._h, batch._h, stream))

    def read_results(self, batch: PendingBatch):
        """The batch's per-read results and ties as they stand in device
        memory now (after :meth:`relaunch`, the last launch's)."""
        n = batch.n_reads
        res = np.zeros(n, dtype=RESULT_DTYPE)
        ties = np.zeros((n, self.cap), dtype=np.uint32)
        _check(self._lib, self._lib.esg_batch_read_results(self._h, batch._h, res.ctypes.data,
                                                           _ptr(ties, C.c_uint32)))
        return res, ties

    def finish(self, batch: PendingBatch, keep: bool = False) -> BatchResult:
        n = batch.n_reads
        res = np.zeros(n, dtype=RESULT_DTYPE)
        ties = np.zeros((n, self.cap), dtype=np.uint32)
        rows = None
        nq = n * (2 if batch.flags & BOTH_STRANDS else 1)
        if batch.flags & FULL_ROWS:
            rows = np.zeros((nq, len(self.panel)), dtype=np.int32)
        _check(self._lib, self._lib.esg_finish(self._h, batch._h, res.ctypes.data,
                                               _ptr(ties, C.c_uint32),
                                               _ptr(rows, C.c_int32) if rows is not None else None))
        stats = batch.stats()
        if not keep:
            batch.free()
        return BatchResult(res, ties, rows, len(self.panel), stats, self.cap)

    def score_batch(self, reads, both_strands: bool = False, full_rows: bool = False) -> BatchResult:
        """cuda/mod.rs:524-528."""
        return self.finish(self.submit(self.prepare(reads, both_strands, full_rows)))

    def score_batches(self, batches, both_strands: bool = False, full_rows: bool = False,
                      timing: dict | None = None):
        """The CLI's GPU feeder (score_batches, align.rs:2801-2917) over this
        scorer: every item of `batches` (reads as `prepare` takes them) is
        prepared and queued while the one before it runs on the device, so
        the device does not drain between batches; yields each batch's
        result, in order.  `timing`, if given, accumulates the host seconds
        spent preparing, submitting and waiting to finish."""
        return self._feed(batches, lambda r: self.prepare(r, both_strands, full_rows),
                          self.finish, timing)

    def score_pair_batches(self, batches, adapters=None, min_score: int = 0,
                           both_strands: bool = True, full_rows: bool = False,
                           timing: dict | None = None):
        """score_batches for read pairs (the feeder's paired branch,
        align.rs:2844-2872): each item's mates trimmed and scored as
        `prepare_pairs` does; yields each batch's PairBatchResult."""
        return self._feed(batches,
                          lambda r: self.prepare_pairs(r, adapters, min_score, both_strands,
                                                       full_rows),
                          self.finish_pairs, timing)

    def _feed(self, batches, prepare, finish, timing):
        t = timing if timing is not None else {}
        for k in ("prepare_s", "submit_s", "finish_s"):
            t.setdefault(k, 0.0)
        pc = time.perf_counter
        in_flight = None
        try:
            for reads in batches:
                a = pc()
                nxt = prepare(reads)
                b = pc()
                self.submit(nxt)
                t["prepare_s"] += b - a
                t["submit_s"] += pc() - b
                if in_flight is not None:
                    done, in_flight = in_flight, nxt
                    a = pc()
                    res = finish(done)
                    t["finish_s"] += pc() - a
                    yield res
                else:
                    in_flight = nxt
            if in_flight is not None:
                done, in_flight = in_flight, None
                a = pc()
                res = finish(done)
                t["finish_s"] += pc() - a
                yield res
        finally:
            if in_flight is not None:  # abandoned: wait for it, drop it
                finish(in_flight)

    # -- traceback of winners (scalar.rs:182-364)
    def align(self, reads, jobs) -> "Alignments":
        """Trace (read, reference, reverse) jobs against `reads` (uploaded
        here): coordinates and CIGAR of each, as scalar::align gives them."""
        codes, off, lens = self._inputs(reads)
        jobs = _jobs_array(jobs)
        ref_len = self._panel_arrays[2]
        bound = int(lens[jobs[:, 0]].sum(dtype=np.uint64) + ref_len[jobs[:, 1]].sum(dtype=np.uint64)) \
            if jobs.shape[0] and (jobs[:, 0] < lens.size).all() and (jobs[:, 1] < ref_len.size).all() \
            else 0
        return _align_call(self._lib, self._lib.esg_align_reads,
                           (self._h, _ptr(codes, C.c_uint8), _ptr(off, C.c_uint64),
                            _ptr(lens, C.c_uint32), lens.size), jobs, bound)

    def align_batch(self, batch: PendingBatch, jobs) -> "Alignments":
        """The same against a finished batch's reads, still on the device
        (finish it with keep=True)."""
        jobs = _jobs_array(jobs)
        lens = getattr(batch, "lens", None)
        ref_len = self._panel_arrays[2]
        bound = 0
        if lens is not None and jobs.shape[0] and (jobs[:, 0] < lens.size).all() and \
                (jobs[:, 1] < ref_len.size).all():
            bound = int(lens[jobs[:, 0]].sum(dtype=np.uint64) +
                        ref_len[jobs[:, 1]].sum(dtype=np.uint64))
        return _align_call(self._lib, self._lib.esg_align_batch, (self._h, batch._h), jobs, bound)

    # -- mapping (mapper.rs:400-552)
    def map_reads(self, reads, min_score: int = 0, max_ties: int | None = None,
                  both_strands: bool = False, ref_letters=None, raw: bool = False):
        """Aligner::map_reads_scored over this scorer: per read the best, XS,
        tie count and the traced hits (primary first) with MD and NM.
        `ref_letters`: the panel's letters (a list of str/bytes, panel order)
        for MD; without them MD spells the panel's codes as A/C/G/T/N.
        Returns Mappings, or with `raw` the library's mapping itself
        (MappingHandle), for a consumer in the library such as the BAM
        encoder, with no copy."""
        codes, off, lens = self._inputs(reads)
        lp, lo, keep = self._letters(ref_letters)
        opts = _native.EsgMapOptions(int(min_score),
                                     0xFFFFFFFF if max_ties is None else int(max_ties),
                                     int(bool(both_strands)), 0)
        if max_ties is not None and not 0 <= int(max_ties) < 0xFFFFFFFF:
            raise ValueError("max_ties must be in [0, 2^32 - 1)")
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_map_reads(self._h, _ptr(codes, C.c_uint8),
                                                  _ptr(off, C.c_uint64), _ptr(lens, C.c_uint32),
                                                  lens.size, C.byref(opts), lp, lo, C.byref(h)))
        if raw:
            return MappingHandle(self._lib, h)
        try:
            return Mappings._copy(self._lib, h)
        finally:
            self._lib.esg_mapping_free(h)

    def map_pairs(self, mates, min_score: int = 0, max_ties: int | None = None,
                  max_insert: int = 500, both_strands: bool = False,
                  ref_letters=None, raw: bool = False):
        """Aligner::map_pairs_scored (pair.rs:157-390) over this scorer:
        mates 2p and 2p + 1 are pair p (adapters already trimmed).  Per pair
        Proper (score, tie count, per-mate XS, pair hits) or Separate (each
        mate as map_reads maps it on both strands).  `raw` as for map_reads."""
        codes, off, lens = self._inputs(mates)
        if lens.size % 2:
            raise ValueError("mates come in pairs")
        if max_ties is not None and not 0 <= int(max_ties) < 0xFFFFFFFF:
            raise ValueError("max_ties must be in [0, 2^32 - 1)")
        if not 0 <= int(max_insert) < 2**32:
            raise ValueError("max_insert must fit 32 bits")
        lp, lo, keep = self._letters(ref_letters)
        opts = _native.EsgPairMapOptions(int(min_score),
                                         0xFFFFFFFF if max_ties is None else int(max_ties),
                                         int(max_insert), int(bool(both_strands)))
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_map_pairs(self._h, _ptr(codes, C.c_uint8),
                                                  _ptr(off, C.c_uint64), _ptr(lens, C.c_uint32),
                                                  lens.size // 2, C.byref(opts), lp, lo,
                                                  C.byref(h)))
        if raw:
            return MappingHandle(self._lib, h)
        try:
            return Mappings._copy(self._lib, h, paired=True)
        finally:
            self._lib.esg_mapping_free(h)

    def _letters(self, ref_letters):
        """The panel's letters as (pointer, offsets pointer, arrays to keep)."""
        if ref_letters is None:
            return None, None, None
        if len(ref_letters) != len(self.panel):
            raise ValueError("ref_letters: one entry per reference")
        bl = [r.encode() if isinstance(r, str) else bytes(r) for r in ref_letters]
        for k, b in enumerate(bl):
            if len(b) != int(self._panel_arrays[2][k]):
                raise ValueError(f"ref_letters[{k}]: length differs from the reference")
        letters = np.frombuffer(b"".join(bl) or b"\0", dtype=np.uint8)
        loff = np.zeros(len(bl), dtype=np.uint64)
        if len(bl) > 1:
            loff[1:] = np.cumsum([len(b) for b in bl[:-1]], dtype=np.uint64)
        return _ptr(letters, C.c_uint8), _ptr(loff, C.c_uint64), (letters, loff)

    # -- paired-end (pair.rs:157-234, fed as align.rs:2844-2872 feeds it)
    def prepare_pairs(self, mates, adapters=None, min_score: int = 0, both_strands: bool = True,
                      full_rows: bool = False) -> PreparedBatch:
        """Mates 2p (mate 1) and 2p + 1 (mate 2), as sequenced.  ``adapters``:
        None, or dict(r1=codes, r2=codes, min_overlap=5, max_read_len=0)
        (adapter.rs:46-54; align.rs:934-949)."""
        codes, off, lens = self._inputs(mates)
        if lens.size % 2:
            raise ValueError("mates come in pairs: an even number of reads is needed")
        flags = (BOTH_STRANDS if both_strands else 0) | (FULL_ROWS if full_rows else 0)
        cfg_p, keep = None, None
        if adapters is not None:
            r1 = np.ascontiguousarray(adapters.get("r1", np.zeros(0)), dtype=np.uint8)
            r2 = np.ascontiguousarray(adapters.get("r2", np.zeros(0)), dtype=np.uint8)
            cfg = _native.EsgAdapterConfig(r1.ctypes.data if r1.size else None, r1.size,
                                           r2.ctypes.data if r2.size else None, r2.size,
                                           int(adapters.get("min_overlap", 5)),
                                           int(adapters.get("max_read_len", 0)))
            cfg_p, keep = C.byref(cfg), (r1, r2, cfg)
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_prepare_pairs(
            self._h, _ptr(codes, C.c_uint8), _ptr(off, C.c_uint64), _ptr(lens, C.c_uint32),
            lens.size // 2, cfg_p, int(min_score), flags, C.byref(h)))
        del keep
        b = PreparedBatch(self, h, int(lens.size), flags | BOTH_STRANDS, None)
        b.paired = True
        b.lens = lens  # untrimmed: an upper bound for the traceback's CIGAR room
        return b

    def finish_pairs(self, batch: PendingBatch, keep: bool = False) -> PairBatchResult:
        n = batch.n_reads
        npairs = n // 2
        pairs = np.zeros(npairs, dtype=PAIR_DTYPE)
        pties = np.zeros((npairs, self.cap), dtype=np.uint32)
        res = np.zeros(n, dtype=RESULT_DTYPE)
        ties = np.zeros((n, self.cap), dtype=np.uint32)
        ads = np.zeros(n, dtype=np.uint32)
        rows = (np.zeros((2 * n, len(self.panel)), dtype=np.int32)
                if batch.flags & FULL_ROWS else None)
        _check(self._lib, self._lib.esg_finish_pairs(
            self._h, batch._h, pairs.ctypes.data, _ptr(pties, C.c_uint32), res.ctypes.data,
            _ptr(ties, C.c_uint32), _ptr(ads, C.c_uint32),
            _ptr(rows, C.c_int32) if rows is not None else None))
        stats = batch.stats()
        if not keep:
            batch.free()
        mates = BatchResult(res, ties, rows, len(self.panel), stats, self.cap)
        return PairBatchResult(pairs, pties, mates, ads, stats, self.cap)

    def score_pairs(self, mates, adapters=None, min_score: int = 0, both_strands: bool = True,
                    full_rows: bool = False) -> PairBatchResult:
        """prepare_pairs + submit + finish_pairs."""
        return self.finish_pairs(self.submit(self.prepare_pairs(
            mates, adapters, min_score, both_strands, full_rows)))


ALIGN_DTYPE = np.dtype([("score", "<i4"), ("query_start", "<u4"), ("query_end", "<u4"),
                        ("ref_start", "<u4"), ("ref_end", "<u4"), ("n_ops", "<u4"),
                        ("ops_offset", "<u8")])
CIGAR_OPS = "MID"


def cigar_string(ops) -> str:
    """BAM CIGAR words (len << 4 | op) as text."""
    return "".join(f"{int(w) >> 4}{CIGAR_OPS[int(w) & 0xf]}" for w in ops)


def _jobs_array(jobs):
    jobs = np.ascontiguousarray(np.asarray(jobs, dtype=np.uint32).reshape(-1, 3))
    return jobs


class Alignments:
    """Traced alignments of a list of jobs: records (ALIGN_DTYPE) and the
    CIGAR words they point into."""

    def __init__(self, records, ops):
        self.records = records
        self.ops = ops

    def __len__(self):
        return self.records.size

    def ops_of(self, k: int):
        r = self.records[k]
        o = int(r["ops_offset"])
        return self.ops[o:o + int(r["n_ops"])]

    def cigar(self, k: int) -> str:
        return cigar_string(self.ops_of(k))


MAPPING_DTYPE = np.dtype([("best_score", "<i4"), ("suboptimal", "<i4"), ("n_tied", "<u4"),
                          ("flags", "<u4"), ("n_hits", "<u4"), ("reserved", "<u4"),
                          ("first_hit", "<u8")])
HIT_DTYPE = np.dtype([("reference", "<u4"), ("reverse", "<u4"), ("score", "<i4"),
                      ("query_start", "<u4"), ("query_end", "<u4"), ("ref_start", "<u4"),
                      ("ref_end", "<u4"), ("n_ops", "<u4"), ("ops_offset", "<u8"),
                      ("nm", "<u4"), ("md_len", "<u4"), ("md_offset", "<u8")])
MAPPING_HAS_BEST = 1
MAPPING_HAS_SUBOPTIMAL = 2
PAIR_MAPPING_DTYPE = np.dtype([("flags", "<u4"), ("score", "<i4"), ("n_tied", "<u4"),
                               ("n_hits", "<u4"), ("suboptimal", "<i4", (2,)),
                               ("first_hit", "<u8")])
PAIR_HIT_DTYPE = np.dtype([("reference", "<u4"), ("reverse", "<u4"), ("insert", "<u8"),
                           ("mates", HIT_DTYPE, (2,))])
PAIR_PROPER = 1
PAIR_HAS_XS = (2, 4)


class MappingHandle:
    """An esg_mapping the library owns (map_reads / map_pairs with raw=True),
    freed with free() or when collected; mappings() copies it out."""

    def __init__(self, lib, h):
        self._lib = lib
        self._h = h

    def mappings(self, paired: bool = False) -> "Mappings":
        return Mappings._copy(self._lib, self._h, paired)

    def free(self):
        if self._h:
            self._lib.esg_mapping_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Mappings:
    """esg_map_reads' output: per read a MAPPING_DTYPE record, its hits
    (HIT_DTYPE) and their CIGAR words and MD strings."""

    def __init__(self, reads, hits, ops, md: bytes, pairs=None, pair_hits=None):
        self.reads = reads
        self.hits = hits
        self.ops = ops
        self.md_bytes = md
        self.pairs = pairs
        self.pair_hits = pair_hits

    @classmethod
    def _copy(cls, lib, h, paired=False):
        def arr(fn, ct, dtype, count_t):
            n = count_t()
            p = fn(h, C.byref(n))
            if not n.value:
                return np.zeros(0, dtype=dtype)
            buf = (ct * (n.value * dtype.itemsize // C.sizeof(ct))).from_address(p)
            return np.frombuffer(buf, dtype=dtype).copy()
        reads = arr(lib.esg_mapping_reads, C.c_uint8, MAPPING_DTYPE, C.c_uint32)
        hits = arr(lib.esg_mapping_hits, C.c_uint8, HIT_DTYPE, C.c_uint64)
        ops = arr(lib.esg_mapping_ops, C.c_uint8, np.dtype("<u4"), C.c_uint64)
        md = arr(lib.esg_mapping_md, C.c_uint8, np.dtype("u1"), C.c_uint64).tobytes()
        pairs = pair_hits = None
        if paired:
            pairs = arr(lib.esg_mapping_pairs, C.c_uint8, PAIR_MAPPING_DTYPE, C.c_uint32)
            pair_hits = arr(lib.esg_mapping_pair_hits, C.c_uint8, PAIR_HIT_DTYPE, C.c_uint64)
        return cls(reads, hits, ops, md, pairs, pair_hits)

    def __len__(self):
        return (self.pairs if self.pairs is not None else self.reads).size

    def md(self, i: int) -> str:
        return self._md_of(self.hits[i])

    def ops_of(self, i: int):
        return self._ops_of(self.hits[i])

    def _md_of(self, h) -> str:
        o = int(h["md_offset"])
        return self.md_bytes[o:o + int(h["md_len"])].decode()

    def _ops_of(self, h):
        o = int(h["ops_offset"])
        return self.ops[o:o + int(h["n_ops"])]

    def _hit(self, h) -> dict:
        return {"reference": int(h["reference"]), "reverse": bool(h["reverse"]),
                "score": int(h["score"]), "query_start": int(h["query_start"]),
                "query_end": int(h["query_end"]), "ref_start": int(h["ref_start"]),
                "ref_end": int(h["ref_end"]), "cigar": cigar_string(self._ops_of(h)),
                "md": self._md_of(h), "nm": int(h["nm"])}

    def pair_mapping(self, p: int) -> dict:
        """Pair p as a plain dict (PairMapping, pair.rs:89-105)."""
        r = self.pairs[p]
        f = int(r["flags"])
        if not f & PAIR_PROPER:
            return {"proper": False, "mates": [self.mapping(2 * p), self.mapping(2 * p + 1)]}
        hits = []
        for i in range(int(r["first_hit"]), int(r["first_hit"]) + int(r["n_hits"])):
            ph = self.pair_hits[i]
            hits.append({"reference": int(ph["reference"]), "reverse": bool(ph["reverse"]),
                         "insert": int(ph["insert"]),
                         "mates": [self._hit(ph["mates"][0]), self._hit(ph["mates"][1])]})
        return {"proper": True, "score": int(r["score"]), "n_tied": int(r["n_tied"]),
                "suboptimal": [int(r["suboptimal"][m]) if f & PAIR_HAS_XS[m] else None
                               for m in range(2)],
                "hits": hits}

    def mapping(self, k: int) -> dict:
        """Read k as a plain dict (ReadMapping's fields, mapper.rs:60-70)."""
        r = self.reads[k]
        f = int(r["flags"])
        hits = [self._hit(self.hits[i])
                for i in range(int(r["first_hit"]), int(r["first_hit"]) + int(r["n_hits"]))]
        return {"best_score": int(r["best_score"]) if f & MAPPING_HAS_BEST else None,
                "n_tied": int(r["n_tied"]),
                "suboptimal": int(r["suboptimal"]) if f & MAPPING_HAS_SUBOPTIMAL else None,
                "hits": hits}


def _align_call(lib, fn, args_head, jobs, bound=0):
    """One call with room for `bound` words (an upper bound when known:
    runs <= read + reference length per job), a second if it was short."""
    jobs = _jobs_array(jobs)
    n = jobs.shape[0]
    rec = np.zeros(max(n, 1), dtype=ALIGN_DTYPE)
    need = C.c_uint64()
    cap = int(bound)
    ops = np.empty(max(cap, 1), dtype=np.uint32)  # only the words written are touched
    st = fn(*args_head, jobs.ctypes.data, n, rec.ctypes.data, _ptr(ops, C.c_uint32), cap,
            C.byref(need))
    if st == 7 and need.value > cap:  # room for the words, then again
        ops = np.empty(max(need.value, 1), dtype=np.uint32)
        st = fn(*args_head, jobs.ctypes.data, n, rec.ctypes.data, _ptr(ops, C.c_uint32),
                ops.size, C.byref(need))
    _check(lib, st)
    return Alignments(rec[:n], ops[:need.value])


def select_hits(scores: ReadScores, min_score: int = 0, max_ties: int | None = None):
    """The tie-set members a caller traces (mapper.rs:466-472): the first
    min(n_tied, max_ties + 1) ties when best >= min_score, else none."""
    if scores.best is None or scores.best < min_score:
        return []
    k = scores.n_tied if max_ties is None else min(scores.n_tied, max_ties + 1)
    if k > len(scores.ties):
        raise ValueError(f"{k} ties requested but only {len(scores.ties)} listed; "
                         "raise tie_capacity or ask for full rows")
    return scores.ties[:k]
