"""BAM input and output around the mapping stage (esg_bam_*), and the CLI's
unpaired and paired runs over them.

The reference's `eschalign` binary reads a BAM, FASTA or FASTQ in batches
(read_batches, crates/eschalign-cli/src/align.rs:604-660), maps them
(Aligner::map_reads_scored), turns each read's mapping into its output
records (build_records, align.rs:1084-1200) and writes them in input order or
coordinate order (write_in_order, align.rs:2345-2400; the sort, 2406-2450);
read pairs go through map_pairs_scored and build_pair_records
(align.rs:1203-1425, 1613-1750).  `align_bam` and `align_pairs_bam` do the
same with the library: batches from `BamReader` / `PairReader`, the mapping
stage on the device, `encode` / `encode_pairs` and `BamWriter` on host
threads.  The records are the reference CLI's byte for byte.
"""
from __future__ import annotations

import ctypes as C
import queue
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _native
from .scorer import (HIT_DTYPE, MAPPING_DTYPE, PAIR_HIT_DTYPE, PAIR_MAPPING_DTYPE,
                     GpuError, MappingHandle, Mappings, _check, _ptr)


def _lib():
    return _native.load()


class BamBatch:
    """A batch of primary input records and their reads as alphabet codes
    (reads over the reader's max_read_len have length 0: left unmapped)."""

    def __init__(self, h):
        self._h = h
        lib = _lib()
        codes, off, lens = C.c_void_p(), C.c_void_p(), C.c_void_p()
        n = C.c_uint32()
        _check(lib, lib.esg_bam_batch_reads(h, C.byref(codes), C.byref(off), C.byref(lens),
                                            C.byref(n)))
        self.n = n.value
        if self.n:
            self.lens = np.ctypeslib.as_array((C.c_uint32 * self.n).from_address(lens.value)).copy()
            self.off = np.ctypeslib.as_array((C.c_uint64 * self.n).from_address(off.value)).copy()
            total = int(self.lens.sum(dtype=np.uint64))
            self.codes = (np.ctypeslib.as_array((C.c_uint8 * total).from_address(codes.value)).copy()
                          if total else np.zeros(1, np.uint8))
        else:
            self.lens = np.zeros(0, np.uint32)
            self.off = np.zeros(0, np.uint64)
            self.codes = np.zeros(1, np.uint8)

    def __len__(self):
        return self.n

    def reads(self):
        """(codes, off, lens) for GpuScorer.map_reads."""
        return self.codes, self.off, self.lens

    def free(self):
        if self._h:
            _lib().esg_bam_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class BamReader:
    """esg_bam_open: a BGZF BAM's header and its primary records in batches."""

    def __init__(self, path: str, threads: int = 0, read_ids: str | None = None):
        self._lib = _lib()
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_bam_open(path.encode(), threads, C.byref(h)))
        self._h = h
        self._after_open(read_ids)

    def _after_open(self, read_ids):
        if read_ids is not None:
            st = self._lib.esg_bam_set_read_ids(self._h, read_ids.encode())
            if st:
                err = self._lib.esg_last_error().decode(errors="replace")
                self.close()
                raise GpuError(st, err)
        n = C.c_uint64()
        p = self._lib.esg_bam_header_text(self._h, C.byref(n))
        self.header_text = C.string_at(p, n.value) if n.value else b""

    def counts(self) -> dict:
        """Secondary / supplementary input records skipped, and reads left
        out by read_ids (two per pair)."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(self._lib, self._lib.esg_bam_reader_counts(self._h, C.byref(a), C.byref(b)))
        return {"not_primary": a.value, "filtered": b.value}

    def batches(self, max_reads: int = 50_000, max_read_len: int = 1000):
        while True:
            b = C.c_void_p()
            _check(self._lib, self._lib.esg_bam_read_batch(self._h, max_reads, max_read_len,
                                                           C.byref(b)))
            batch = BamBatch(b)
            if not len(batch):
                batch.free()
                return
            yield batch

    def close(self):
        if self._h:
            self._lib.esg_bam_close(self._h)
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


class PairReader(BamReader):
    """esg_bam_open_pairs: read pairs from two mate files, or from one
    interleaved FASTX / paired BAM file (path2 None), in batches of pairs
    (records 2p and 2p + 1)."""

    def __init__(self, path1: str, path2: str | None = None, threads: int = 0,
                 read_ids: str | None = None):
        self._lib = _lib()
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_bam_open_pairs(path1.encode(),
                                                       path2.encode() if path2 else None,
                                                       threads, C.byref(h)))
        self._h = h
        self._after_open(read_ids)

    def batches(self, max_pairs: int = 25_000):
        """Batches of at most max_pairs pairs, mates at full length (the
        adapter search, esg_pair_adapters, trims them and leaves mates over
        --max-read-len out)."""
        while True:
            b = C.c_void_p()
            _check(self._lib, self._lib.esg_bam_read_pair_batch(self._h, max_pairs,
                                                                C.byref(b)))
            batch = BamBatch(b)
            if not len(batch):
                batch.free()
                return
            yield batch


class BamRecords:
    """Encoded output records (esg_bam_encode): the uncompressed BAM record
    stream of a batch, in read order."""

    def __init__(self, h):
        self._h = h
        lib = _lib()
        nb, nr = C.c_uint64(), C.c_uint32()
        p = lib.esg_bam_records_bytes(h, C.byref(nb), C.byref(nr))
        self.n_records = nr.value
        self.nbytes = nb.value
        self._p = p

    def bytes(self) -> bytes:
        return C.string_at(self._p, self.nbytes) if self.nbytes else b""

    def outcomes(self) -> dict:
        """How the batch's reads (mates) went: unique best, tied, unmapped."""
        u, t, m = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib = _lib()
        _check(lib, lib.esg_bam_records_outcomes(self._h, C.byref(u), C.byref(t), C.byref(m)))
        return {"unique": u.value, "tied": t.value, "unmapped": m.value}

    def free(self):
        if self._h:
            _lib().esg_bam_records_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _names(ref_names):
    names = [n.encode() if isinstance(n, str) else bytes(n) for n in ref_names]
    return (C.c_char_p * max(len(names), 1))(*names), len(names)


def mapping_handle(m: Mappings):
    """An esg_mapping (esg_mapping_from_arrays) holding `m`'s arrays; free it
    with esg_mapping_free."""
    lib = _lib()
    reads = np.ascontiguousarray(m.reads, dtype=MAPPING_DTYPE)
    hits = np.ascontiguousarray(m.hits, dtype=HIT_DTYPE)
    ops = np.ascontiguousarray(m.ops, dtype=np.uint32)
    md = bytes(m.md_bytes)
    h = C.c_void_p()
    _check(lib, lib.esg_mapping_from_arrays(reads.ctypes.data, reads.size, hits.ctypes.data,
                                            hits.size, _ptr(ops, C.c_uint32), ops.size, md,
                                            len(md), C.byref(h)))
    if m.pairs is not None:
        pairs = np.ascontiguousarray(m.pairs, dtype=PAIR_MAPPING_DTYPE)
        phits = np.ascontiguousarray(m.pair_hits, dtype=PAIR_HIT_DTYPE)
        st = lib.esg_mapping_set_pairs(h, pairs.ctypes.data, pairs.size, phits.ctypes.data,
                                       phits.size)
        if st:
            err = lib.esg_last_error().decode(errors="replace")
            lib.esg_mapping_free(h)
            raise GpuError(st, err)
    return h


def _handle_of(mapping):
    """The esg_mapping pointer of a MappingHandle (or a raw handle as is)."""
    return mapping._h if isinstance(mapping, MappingHandle) else mapping


def encode(batch: BamBatch, mapping, ref_names, secondary: bool = False,
           threads: int = 0) -> BamRecords:
    """build_records (align.rs:1084-1200) for every read of `batch` from its
    mapping (a Mappings, or an esg_mapping handle)."""
    lib = _lib()
    own = isinstance(mapping, Mappings)
    h = mapping_handle(mapping) if own else _handle_of(mapping)
    names, n = _names(ref_names)
    opts = _native.EsgBamOptions(int(bool(secondary)), 0)
    out = C.c_void_p()
    try:
        _check(lib, lib.esg_bam_encode(batch._h, h, C.byref(opts), names, n, threads,
                                       C.byref(out)))
    finally:
        if own:
            lib.esg_mapping_free(h)
    return BamRecords(out)


def encode_pairs(batch: BamBatch, mapping, ref_names, adapter_bases=None,
                 secondary: bool = False, threads: int = 0) -> BamRecords:
    """build_pair_records (align.rs:1238-1425) for every pair of `batch`
    from its paired mapping (a Mappings with pairs, or an esg_mapping
    handle); adapter_bases per mate (esg_pair_adapters), or None when
    adapters were not searched."""
    lib = _lib()
    own = isinstance(mapping, Mappings)
    h = mapping_handle(mapping) if own else _handle_of(mapping)
    names, n = _names(ref_names)
    opts = _native.EsgBamOptions(int(bool(secondary)), 0)
    ads = None if adapter_bases is None else np.ascontiguousarray(adapter_bases, dtype=np.uint32)
    out = C.c_void_p()
    try:
        _check(lib, lib.esg_bam_encode_pairs(batch._h, h, None if ads is None else
                                             _ptr(ads, C.c_uint32), C.byref(opts), names, n,
                                             threads, C.byref(out)))
    finally:
        if own:
            lib.esg_mapping_free(h)
    return BamRecords(out)


class BamWriter:
    """esg_bam_writer_*: header, then pushed chunks in sequence order (or in
    coordinate order at close), BGZF-compressed on host threads, or on
    `device` (esg_bam_writer_use_device: one warp per block)."""

    def __init__(self, path: str, header_text: bytes, ref_names, ref_lens,
                 sort_coordinate: bool = False, threads: int = 0, device: int | None = None):
        self._lib = _lib()
        names, n = _names(ref_names)
        lens = np.ascontiguousarray(ref_lens, dtype=np.uint32)
        h = C.c_void_p()
        _check(self._lib, self._lib.esg_bam_writer_open(
            path.encode(), header_text, names, _ptr(lens, C.c_uint32), n,
            int(bool(sort_coordinate)), threads, C.byref(h)))
        self._h = h
        self.device = device
        if device is not None:
            try:
                _check(self._lib, self._lib.esg_bam_writer_use_device(h, int(device)))
            except Exception:
                self._lib.esg_bam_writer_close(h)
                self._h = None
                raise

    def blocks(self) -> tuple:
        """(blocks the device compressed so far, of them stored)."""
        b, s = C.c_uint64(), C.c_uint64()
        _check(self._lib, self._lib.esg_bam_writer_blocks(self._h, C.byref(b), C.byref(s)))
        return b.value, s.value

    def push(self, seq: int, records: BamRecords):
        _check(self._lib, self._lib.esg_bam_writer_push(self._h, seq, records._h))

    def close(self):
        if self._h:
            h, self._h = self._h, None
            _check(self._lib, self._lib.esg_bam_writer_close(h))

    def __enter__(self):
        return self

    def __exit__(self, exc_type, *exc):
        if exc_type is None:
            self.close()
            return
        try:  # the error in flight is the one to report
            self.close()
        except Exception:
            pass


def header_text(ref_names, ref_lens, sort_coordinate: bool = False,
                input_text: bytes = b"") -> bytes:
    """The output header as the CLI builds it (build_header,
    align.rs:1780-1808): @HD VN:1.6 with the sort order, an @SQ line per
    panel reference, the input's read groups, programs and comments, and a
    @PG line of its own chained (PP) after the input's last program."""
    so = "coordinate" if sort_coordinate else "unsorted"
    lines = [f"@HD\tVN:1.6\tSO:{so}"]
    for n, ln in zip(ref_names, ref_lens):
        lines.append(f"@SQ\tSN:{n if isinstance(n, str) else n.decode()}\tLN:{int(ln)}")
    kept = {"@RG": [], "@PG": [], "@CO": []}
    for line in input_text.decode(errors="replace").splitlines():
        if line[:3] in kept:
            kept[line[:3]].append(line)
    ids, parents = [], set()
    for line in kept["@PG"]:
        f = dict(x.split(":", 1) for x in line.split("\t")[1:] if ":" in x)
        if "ID" in f:
            ids.append(f["ID"])
        if "PP" in f:
            parents.add(f["PP"])
    pid, k = "eschalign-b200", 0
    while pid in ids:
        k += 1
        pid = f"eschalign-b200.{k}"
    leaves = [x for x in ids if x not in parents]
    pg = f"@PG\tID:{pid}\tPN:eschalign-b200" + (f"\tPP:{leaves[-1]}" if leaves else "")
    lines += kept["@RG"] + kept["@PG"] + [pg] + kept["@CO"]
    return ("\n".join(lines) + "\n").encode()


def _scorers(scorer):
    """One scorer, or several over the same panel and scoring."""
    return list(scorer) if isinstance(scorer, (list, tuple)) else [scorer]


def _deflate_device(scorers, deflate_on_device):
    """The device the writer compresses on: the first scorer's, when it has
    one and deflate_on_device is set."""
    if not deflate_on_device:
        return None
    dev = getattr(scorers[0], "device", None)
    return dev if isinstance(dev, int) else None


def _run(reader, batches, scorers, map_batch, encode_batch, out_path, ref_names, ref_lens,
         sort_coordinate, threads, stats, depth, deflate_device=None):
    """Read, map and encode/write on their own threads (the CLI's reader, GPU
    feeder and workers, align.rs:2078-2335): reading batch k + 1, mapping
    batch k, building and writing the records of batch k - 1, at most
    `depth` batches waiting between the stages.  With several scorers, one
    mapping thread per scorer: one thread's host share of the mapping
    (packing, tie lists, MD / NM, assembly) overlaps another's scoring on
    the device."""
    out = {"reads": 0, "records": 0, "batches": 0, "unique": 0, "tied": 0, "unmapped": 0}
    st = stats if stats is not None else {}
    for k in ("read", "map", "encode", "write"):
        st.setdefault(k, 0.0)
    free = queue.SimpleQueue()
    for sc in scorers:
        free.put(sc)
    lock = threading.Lock()

    def mapped(batch):
        t0 = time.perf_counter()
        sc = free.get()
        try:
            m = map_batch(sc, batch)
        finally:
            free.put(sc)
        with lock:
            st["map"] += time.perf_counter() - t0
        return batch, m

    with reader, BamWriter(out_path, header_text(ref_names, ref_lens, sort_coordinate,
                                                 reader.header_text),
                           ref_names, ref_lens, sort_coordinate, threads,
                           deflate_device) as wr, \
            ThreadPoolExecutor(1) as rpool, ThreadPoolExecutor(len(scorers)) as mpool, \
            ThreadPoolExecutor(1) as opool:
        def read_next():
            t0 = time.perf_counter()
            b = next(batches, None)
            st["read"] += time.perf_counter() - t0
            return b

        def emit(seq, mfut):
            batch, m = mfut.result()
            t0 = time.perf_counter()
            rec = encode_batch(batch, m)
            if isinstance(m, MappingHandle):
                m.free()
            t1 = time.perf_counter()
            wr.push(seq, rec)
            st["encode"] += t1 - t0
            st["write"] += time.perf_counter() - t1
            out["reads"] += len(batch)
            out["records"] += rec.n_records
            out["batches"] += 1
            for k, v in rec.outcomes().items():
                out[k] += v
            rec.free()
            batch.free()

        inflight = deque()
        try:
            nxt, seq = rpool.submit(read_next), 0
            while True:
                batch = nxt.result()
                if batch is None:
                    break
                nxt = rpool.submit(read_next)
                inflight.append(opool.submit(emit, seq, mpool.submit(mapped, batch)))
                seq += 1
                while len(inflight) > max(depth, len(scorers)):
                    inflight.popleft().result()
            while inflight:
                inflight.popleft().result()
        except BaseException:
            for p in (rpool, mpool, opool):
                p.shutdown(wait=True, cancel_futures=True)
            raise
        t0 = time.perf_counter()
    st["write"] += time.perf_counter() - t0  # the writer's close: its last blocks (or the sort)
    return out


def align_bam(scorer, in_path: str, out_path: str, ref_names, ref_letters,
              min_score: int = 0, max_ties: int | None = None, both_strands: bool = False,
              secondary: bool = False, sort_coordinate: bool = False,
              max_read_len: int = 1000, batch_size: int = 50_000, threads: int = 0,
              stats: dict | None = None, depth: int = 2, read_ids: str | None = None,
              deflate_on_device: bool = True) -> dict:
    """The CLI's unpaired run (align.rs:1822-2250, the --device gpu path) over
    a scorer: every batch of `in_path` (BAM, FASTA or FASTQ) mapped on the
    device (map_reads_scored with min_score / max_ties / both strands), its
    records built and written to `out_path` in input order (or coordinate
    order).  Returns counts.  Reading, mapping and encoding/writing overlap
    on three threads; `stats`, if given, receives the seconds each stage
    spent (read, map, encode, write; they overlap, so they add up to more
    than the wall time).  read_ids: --read-ids, a file of the names kept.
    `scorer` may be a list of scorers over the same panel and scoring: each
    maps on its own thread, so the device scores one batch while the host
    finishes another (the records do not depend on it).  With
    deflate_on_device, the output's BGZF blocks are compressed on the
    scorer's device (BamWriter's `device`); the records are the same."""
    rd = BamReader(in_path, threads, read_ids)
    scs = _scorers(scorer)
    return _run(rd, rd.batches(batch_size, max_read_len), scs,
                lambda sc, b: sc.map_reads(b.reads(), min_score=min_score, max_ties=max_ties,
                                           both_strands=both_strands, ref_letters=ref_letters,
                                           raw=True),
                lambda b, m: encode(b, m, ref_names, secondary, threads),
                out_path, ref_names, [len(r) for r in ref_letters], sort_coordinate, threads,
                stats, depth, _deflate_device(scs, deflate_on_device))


DEFAULT_ADAPTERS = "truseq"


def align_pairs_bam(scorer, path1: str, path2: str | None, out_path: str, ref_names, ref_letters,
                    min_score: int = 0, max_ties: int | None = None, max_insert: int = 500,
                    both_strands: bool = False, secondary: bool = False,
                    sort_coordinate: bool = False, max_read_len: int = 1000,
                    adapters=DEFAULT_ADAPTERS, batch_size: int = 50_000, threads: int = 0,
                    stats: dict | None = None, depth: int = 2,
                    read_ids: str | None = None, deflate_on_device: bool = True) -> dict:
    """The CLI's paired run (align.rs:1613-1750 over run, 1822-2250): pairs
    from two mate files, or one interleaved / paired-BAM file (path2 None),
    each mate trimmed of its 3' adapter (pair_adapters; `adapters` an
    adapter.config() dict, the TruSeq default, or None for
    --no-adapter-trim), the pairs mapped on the device (map_pairs_scored),
    their records built (build_pair_records) and written in input or
    coordinate order.  batch_size counts records, two per pair, as the
    CLI's --batch-size does; read_ids (--read-ids) selects pairs by name.
    `scorer` may be a list of scorers, as for align_bam."""
    from . import adapter as A
    if adapters == DEFAULT_ADAPTERS:
        adapters = A.config()
    cfg = None if adapters is None else dict(adapters, max_read_len=int(max_read_len))
    rd = PairReader(path1, path2, threads, read_ids)
    state = {}

    def map_batch(sc, b):
        codes, off, lens = b.reads()
        if cfg is not None:
            ads, aligned = A.pair_adapters((codes, off, lens), cfg)
        else:
            ads = None
            aligned = np.where((lens > max_read_len) if max_read_len else False, 0,
                               lens).astype(np.uint32)
        state[id(b)] = ads
        return sc.map_pairs((codes, off, aligned), min_score=min_score, max_ties=max_ties,
                            max_insert=max_insert, both_strands=both_strands,
                            ref_letters=ref_letters, raw=True)

    def encode_batch(b, m):
        return encode_pairs(b, m, ref_names, state.pop(id(b)), secondary, threads)

    scs = _scorers(scorer)
    return _run(rd, rd.batches((batch_size + 1) // 2), scs, map_batch,
                encode_batch, out_path,
                ref_names, [len(r) for r in ref_letters], sort_coordinate, threads, stats, depth,
                _deflate_device(scs, deflate_on_device))
