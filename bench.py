#!/usr/bin/env python
"""Benchmark of the panel-scoring hot path (one JSON line on rank 0).

Workload (C2, the plain-vs-batched scale-up case): 1 000 000 synthetic
reads, lengths lognormal (median 110, sigma 0.4) clipped to 20-1000, cut from
a 164-reference panel of 70-180 nt (8 % subs, 2 % ins, 1 % del) or random,
both strands, scored against every reference and reduced per read to best
score + XS + tie count + up to 8 ties.  A step is one pass over the whole
batch for one (mode, scheme); the headline is local 2,-1,-10,-1 and the
other three (mode, scheme) combinations are measured once each.

* value     GCUPS (10^9 DP cells/s; cells = read length x panel bases, summed
            over both strands, the reference's convention,
            crates/eschalign/examples/gpu_score_probe.rs:80-86) of the batched
            kernel with the batch resident on the device, CUDA events on the
            launching stream, L2 flushed between steps, max over ranks.
* e2e       the same metric through the public API with host buffers: the
            batch fed in chunks through prepare / submit / finish, two
            batches in flight, like eschalign's GPU feeder thread
            (crates/eschalign-cli/src/align.rs:2801-2917), host<->device
            copies inside the timed region.
* roofline  integer ALU: the batched kernel's algorithmic work (12 int ops a
            cell local, 11 semi-global, two cells per 32-bit lane op) against
            the integer lane-op peak measured by csrc/esg_probe.cu in the same
            run.
* --impl reference  the reference's CPU path (AVX-512BW score kernels +
            selection, restated in oracle/) on all host cores.

Other workloads (``--workload``), one JSON line each, same keys:

* c4  2 000 000 read pairs of 2 x 150 nt (inserts lognormal, median 90 nt,
      40-600; adapter read-through past short inserts, 1 % errors; 1 % subs,
      0.2 % indels) on the 164-reference panel, semi-global 2,-1,-10,-1:
      each mate trimmed of its adapter on the host (the reference's rule),
      all four mate queries scored, the (reference, template strand)
      candidates of both template strands ranked on the device; GCUPS and
      pairs/s.  CPU arm: trimming + AVX-512BW rows + the same ranking.
* c1  the reference's CPU-sized case: 10 000 reads (90 % cut from a
      reference, 8 % subs, 2 % ins, 1 % del; 10 % random) of 60-200 nt
      against the 164-reference panel, local 2,-1,-10,-1, forward strand;
      GPU device time and e2e beside the CPU path on the whole set.
* c5  serving: Poisson arrivals at each rate of --rates; a request is
      log-uniform 1-50 000 reads (C2 lengths) for panel A (C2's 164 refs)
      or B (2000 x 300 nt), local or semi-global, forward or both strands,
      through the library's request queue (esg_server: continuous batching
      over four resident scorers, admission by free device memory); per
      rate p50/p99/p99.9 latency (submit to results, the server's own
      clock) and aggregate GCUPS; a sample of requests re-scored alone must
      be equal.
* c3  the uneven panel: 10 000 references of 300-1000 nt, reads of
      50-1000 nt (70 % derived, 10 % subs, 3 % indels), local, both
      strands, autotuned tile shape; a bounded read sample per step (the
      full 200 000 reads are about 1.4e15 cells).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

HEADLINE = ((2, -1, -10, -1), "local")
COMBOS = [((2, -1, -10, -1), "local"), ((2, -1, -10, -1), "semiglobal"),
          ((1, -1, -2, -1), "local"), ((1, -1, -2, -1), "semiglobal")]
OPS_PER_CELL = {"local": 12, "semiglobal": 11}
C4_SCORING = (2, -1, -10, -1)
C3_SCORING = (2, -1, -10, -1)
# DRAM bytes per DP cell of the batched kernel: 8.29 MB read, 0 written, over
# the 2.678e11 cells of the 16-row launch in the ncu capture of a 60 000-read
# C2 case (profiles/k2_batched_c2.md); the traffic is the reads' codes and
# the plan, which grow with the reads, so it scales by cells to a full launch.
K2_DRAM_BYTES_PER_CELL = 8.288256e6 / 2.67805237160e11


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def args_parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--reads", type=int, default=1_000_000)
    ap.add_argument("--plain-reads", type=int, default=200_000)
    ap.add_argument("--chunk", type=int, default=125_000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--profile-case", type=int, default=0, metavar="READS",
                    help="score READS reads of the workload once per kernel and exit "
                         "(a small target for ncu)")
    ap.add_argument("--bam-case", type=int, default=0, metavar="READS",
                    help="run the unpaired BAM stage alone on READS reads of the workload, "
                         "print its figures and exit (a target for ncu)")
    ap.add_argument("--bam-scorers", type=int, default=2,
                    help="--bam-case: scorers mapping at once, one thread each")
    ap.add_argument("--mode", default="local", choices=["local", "semiglobal"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--pairs", type=int, default=2_000_000, help="c4: read pairs")
    ap.add_argument("--pair-chunk", type=int, default=125_000,
                    help="c4: pairs per prepare/submit/finish batch in the e2e feeder")
    ap.add_argument("--c3-reads", type=int, default=4000, help="c3: reads per step")
    ap.add_argument("--rates", default="10,30,100,300,1000,2000",
                    help="c5: Poisson arrival rates swept (requests/s)")
    ap.add_argument("--requests", type=int, default=1000, help="c5: requests per rate")
    ap.add_argument("--max-batch-cells", type=int, default=0,
                    help="c5: DP cells per server batch at most (0: the server's default)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch each batch's kernels one by one instead of as one CUDA graph")
    ap.add_argument("--split", type=int, default=-1,
                    help="16/32-row split in nt, set instead of autotuning (for runs under a "
                         "profiler, whose serialised launches would skew the autotuner)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.path = tempfile.mktemp(prefix="esg_clocks_", suffix=".csv")
        self.proc = None
        self.gpu = gpu_index

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            lines = [ln.strip() for ln in open(self.path) if ln.strip()]
        except OSError:
            lines = []
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def int_peak(device):
    import ctypes as C

    from eschalign_b200 import _native
    lib = _native.load_probe()
    rates = (C.c_double * 16)()
    per_clk = (C.c_double * 16)()
    n = C.c_int(0)
    sms = C.c_int(0)
    st = lib.esg_probe_int_peak(device, 4000, rates, per_clk, C.byref(n), C.byref(sms))
    if st != 0:
        return None
    ops = {lib.esg_probe_op_name(k).decode(): {"lane_ops_per_s": rates[k],
                                                "per_sm_per_clk": per_clk[k]}
           for k in range(n.value)}
    peak = max(ops["iadd32"]["lane_ops_per_s"], ops["imax32"]["lane_ops_per_s"])
    return {"peak_lane_ops_per_s": peak, "ops": ops, "sms": sms.value}


def roofline_of(peak, per_gpu_cells_s, mode, traffic):
    achieved = per_gpu_cells_s * OPS_PER_CELL[mode] / 2.0
    return {"bound": "int_alu", "achieved": achieved / 1e12,
            "peak": (peak["peak_lane_ops_per_s"] / 1e12) if peak else None,
            "unit": "T lane-ops/s",
            "frac": (achieved / peak["peak_lane_ops_per_s"]) if peak else None,
            "traffic": traffic, "kernel": "k2_batched",
            "note": f"achieved = cells/s x {OPS_PER_CELL[mode]} int ops / 2 cells per "
                    "int16x2 lane-op; peak = measured iadd32/imax32 lane-op rate "
                    "(csrc/esg_probe.cu), measured in this run"}


def cpu_baseline(refs, reads, scoring, mode, seconds, threads=0, chunk=64):
    """The reference's CPU path (AVX-512BW kernels + selection, restated in
    oracle/) on a bounded sample of the workload, all host threads; `chunk`
    reads per work unit (the reference's 64; fewer for a small sample of
    long reads, so every core has work)."""
    from oracle import oracle as O
    O.build()
    O.lib().eo_cpu_set_chunk(chunk)
    prof = O.Profile(refs, scoring)
    panel_bases = sum(len(r) for r in refs)
    local = mode == "local"
    # calibrate on about 1e11 cells (a second or so), at least 16 reads
    cells_per_read = 2 * panel_bases * reads.bases() / max(1, len(reads))
    n_cal = int(min(len(reads), 2000, max(16, 1e11 / max(cells_per_read, 1.0))))
    cal = reads.slice(0, n_cal)
    t = time.perf_counter()
    _, _, _, used = prof.map_batch(*cal.tuple(), local=local, both_strands=True, threads=threads)
    dt = time.perf_counter() - t
    n = int(min(len(reads), max(n_cal, n_cal * seconds / max(dt, 1e-3))))
    sample = reads.slice(0, n)
    t = time.perf_counter()
    res, ties, _, used = prof.map_batch(*sample.tuple(), local=local, both_strands=True,
                                        threads=threads)
    dt = time.perf_counter() - t
    cells = 2 * sample.bases() * panel_bases
    O.lib().eo_cpu_set_chunk(64)
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": int(used), "kind": "port",
            "sample": f"first {n} of {len(reads)} reads, both strands, {mode} "
                      f"{','.join(map(str, scoring))}; {dt:.1f} s; reads/s {n / dt:.0f}; "
                      f"{chunk} reads per work unit",
            "reads_per_s": n / dt, "seconds": dt, "_results": (res, ties)}


def same_results(a, ta, b, tb):
    """Per-read results equal field for field, and the listed ties (the
    first min(n_tied, capacity)) equal in order."""
    if not all(np.array_equal(a[f], b[f]) for f in ("best", "suboptimal", "n_tied")):
        return False
    if not np.array_equal(a["flags"] & 3, b["flags"] & 3):
        return False
    cap = min(ta.shape[1], tb.shape[1])
    n_l = np.minimum(a["n_tied"], cap)
    mask = np.arange(cap)[None, :] < n_l[:, None]
    return bool(np.array_equal(ta[:, :cap][mask], tb[:, :cap][mask]))


def cpu_pairs_baseline(refs, pairs, scoring, seconds, threads=0):
    """The reference's CPU path for pairs (trimming, AVX-512BW rows, ranking;
    oracle/esg_cpu_avx512.c eo_cpu_map_pairs) on a bounded sample."""
    from oracle import oracle as O
    O.build()
    prof = O.Profile(refs, scoring)
    panel_bases = sum(len(r) for r in refs)
    n_all = len(pairs) // 2
    n_cal = min(n_all, 1000)
    t = time.perf_counter()
    prof.map_pairs(*pairs.slice(0, 2 * n_cal).tuple(), local=False, threads=threads)
    dt = time.perf_counter() - t
    n = int(min(n_all, max(n_cal, n_cal * seconds / max(dt, 1e-3))))
    sample = pairs.slice(0, 2 * n)
    t = time.perf_counter()
    _, _, _, _, ads, used = prof.map_pairs(*sample.tuple(), local=False, threads=threads)
    dt = time.perf_counter() - t
    cells = 2 * (sample.bases() - int(ads.sum(dtype=np.uint64))) * panel_bases
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": int(used), "kind": "port",
            "sample": f"first {n} of {n_all} pairs: trim, 4 mate rows, both template strands "
                      f"ranked, semiglobal {','.join(map(str, scoring))}; {dt:.1f} s",
            "pairs_per_s": n / dt, "seconds": dt}


def traceback_stage(g, refs, reads, scoring, local, skip_cpu):
    """The stage after scoring: trace each read's first tie (the primary,
    mapper.rs:494-495) through esg_align_batch from a scored batch's reads on
    the device; wall time incl. the host plan and copies.  Beside it the
    CPU restatement (scalar align per job on all host threads) on a sample."""
    b = g.submit(g.prepare(reads.tuple(), both_strands=True))
    res = g.finish(b, keep=True)
    has = np.nonzero(res.results["n_tied"] > 0)[0]
    jobs = np.stack([has, res.ties[has, 0] >> 1, res.ties[has, 0] & 1], 1).astype(np.uint32)
    # warm-up at the full size: the first call of a size grows the scorer's
    # memory pool and pages in the host buffers
    g.align_batch(b, jobs)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        al = g.align_batch(b, jobs)
        times.append(time.perf_counter() - t0)
    dt = sorted(times)[1]  # the median of three calls
    b.free()
    ref_len = np.array([len(r) for r in refs], dtype=np.int64)
    cells = int((reads.lens[jobs[:, 0]].astype(np.int64) * ref_len[jobs[:, 1]]).sum())
    out = {"jobs": int(jobs.shape[0]), "seconds": round(dt, 4),
           "seconds_each": [round(x, 4) for x in times],
           "alignments_per_s": jobs.shape[0] / dt, "gcups": cells / dt / 1e9,
           "cigar_words": int(al.ops.size),
           "timing": "median of three calls after one of the same size, wall time of the "
                     "call with host buffers (plan, copies, kernels)"}
    if not skip_cpu:
        from oracle import oracle as O
        n = min(jobs.shape[0], 40_000)
        t0 = time.perf_counter()
        _, _, used = O.align_batch(*reads.tuple(), refs, jobs[:n], scoring, local)
        dt_c = time.perf_counter() - t0
        out["cpu"] = {"alignments_per_s": n / dt_c, "cores": used, "kind": "port",
                      "sample": f"first {n} jobs, scalar traceback per job"}
    return out


def map_stage(g, refs, reads, scoring, local, skip_cpu):
    """The whole mapping stage through esg_map_reads (mapper.rs:400-552):
    scoring with the fused reduction, every tie traced (max_ties unset),
    MD / NM; wall time of the call with host buffers.  Beside it the same
    stage on the host cores as the reference's CPU path runs it (the
    oracle's cpu_map_reads: AVX-512 scores and tie sets, scalar traceback,
    MD / NM, all in C on every thread) on a bounded sample."""
    g.map_reads(reads.slice(0, 1000).tuple(), both_strands=True)  # warm-up
    t0 = time.perf_counter()
    h = g.map_reads(reads.tuple(), both_strands=True, raw=True)
    dt = time.perf_counter() - t0
    t1 = time.perf_counter()
    m = h.mappings()  # the arrays copied out to Python, as the Python binding returns them
    dt_copy = time.perf_counter() - t1
    h.free()
    mapped = int((m.reads["n_hits"] > 0).sum())
    out = {"reads": len(reads), "seconds": round(dt, 4), "reads_per_s": len(reads) / dt,
           "reads_per_s_with_python_copy": len(reads) / (dt + dt_copy),
           "mapped": mapped, "hits": int(m.hits.size),
           "options": "both strands, min_score 0, every tie traced, MD/NM without letters; "
                      "the mapping as the C ABI returns it (esg_map_reads)"}
    if not skip_cpu:
        from oracle import oracle as O
        n = min(len(reads), 40_000)
        prof = O.Profile(refs, scoring)
        sub = reads.slice(0, n)
        O.cpu_map_reads(*sub.slice(0, 500).tuple(), refs, scoring, local, both_strands=True,
                        profile=prof)  # warm-up
        t0 = time.perf_counter()
        *_, used = O.cpu_map_reads(*sub.tuple(), refs, scoring, local, both_strands=True,
                                   profile=prof)
        dt_c = time.perf_counter() - t0
        out["cpu"] = {"reads_per_s": n / dt_c, "kind": "port", "cores": int(used),
                      "sample": f"first {n} reads: AVX-512 scores and tie sets, scalar "
                                "traceback of every taken tie, MD / NM, in C on all threads"}
    return out


def unmapped_bam(path, reads, seed=11):
    """`reads` as an unaligned BAM, the CLI's usual input: flag 4, names
    r0000000.., Phred qualities 2-40, an RG:Z tag; BGZF at level 1.  Built
    with array operations (a loop over a million records takes seconds)."""
    import zlib
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(seed)
    n = len(reads)
    lens = reads.lens.astype(np.int64)
    plen = (lens + 1) // 2
    aux = np.frombuffer(b"RGZgrp1\0", np.uint8)
    size = 32 + 9 + plen + lens + aux.size            # block_size
    start = np.zeros(n + 1, np.int64)
    np.cumsum(size + 4, out=start[1:])
    buf = np.zeros(int(start[-1]), np.uint8)
    hdr = np.zeros(n, np.dtype([("bs", "<u4"), ("ref", "<i4"), ("pos", "<i4"), ("lrn", "u1"),
                                ("mapq", "u1"), ("bin", "<u2"), ("ncig", "<u2"), ("flag", "<u2"),
                                ("lseq", "<u4"), ("nref", "<i4"), ("npos", "<i4"),
                                ("tlen", "<i4")]))
    hdr["bs"], hdr["ref"], hdr["pos"], hdr["lrn"] = size, -1, -1, 9
    hdr["bin"], hdr["flag"], hdr["lseq"], hdr["nref"], hdr["npos"] = 4680, 4, lens, -1, -1
    buf[(start[:-1, None] + np.arange(36)).ravel()] = hdr.view(np.uint8)
    k = np.arange(n)
    name = np.zeros((n, 9), np.uint8)
    name[:, 0] = ord("r")
    for d in range(7):
        name[:, 7 - d] = ord("0") + (k // 10 ** d) % 10
    buf[(start[:-1, None] + 36 + np.arange(9)).ravel()] = name.ravel()
    # 4-bit sequence: each read padded to an even length, then paired
    code4 = np.array([1, 2, 4, 8, 15], np.uint8)[np.minimum(reads.codes[:int(lens.sum())], 4)]
    poff = np.zeros(n + 1, np.int64)
    np.cumsum(2 * plen, out=poff[1:])
    pad = np.zeros(int(poff[-1]), np.uint8)
    roff = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=roff[1:])
    pad[np.repeat(poff[:-1] - roff[:-1], lens) + np.arange(int(roff[-1]))] = code4
    packed = pad[0::2] << 4 | pad[1::2]
    pk = np.zeros(n + 1, np.int64)
    np.cumsum(plen, out=pk[1:])
    seq_at = start[:-1] + 45
    buf[np.repeat(seq_at - pk[:-1], plen) + np.arange(int(pk[-1]))] = packed
    qual_at = seq_at + plen
    buf[np.repeat(qual_at - roff[:-1], lens) + np.arange(int(roff[-1]))] = \
        rng.integers(2, 41, int(roff[-1]), dtype=np.uint8)
    aux_at = qual_at + lens
    buf[(aux_at[:, None] + np.arange(aux.size)).ravel()] = np.tile(aux, n)
    text = b"@HD\tVN:1.6\tSO:unsorted\n@RG\tID:grp1\tSM:s\n"
    head = b"BAM\1" + len(text).to_bytes(4, "little") + text + (0).to_bytes(4, "little")
    raw = memoryview(np.concatenate([np.frombuffer(head, np.uint8), buf]))

    def block(i):
        src = raw[i:i + 0xff00]
        c = zlib.compressobj(1, zlib.DEFLATED, -15)
        body = c.compress(src) + c.flush()
        return (b"\x1f\x8b\x08\x04\0\0\0\0\0\xff\x06\0BC\x02\0" +
                (len(body) + 25).to_bytes(2, "little") + body +
                zlib.crc32(src).to_bytes(4, "little") + len(src).to_bytes(4, "little"))
    with ThreadPoolExecutor(os.cpu_count() or 4) as pool, open(path, "wb") as fh:
        for b in pool.map(block, range(0, len(raw), 0xff00)):
            fh.write(b)
        fh.write(bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000"))
    return len(raw)


class CpuMapper:
    """The CPU path's mapping stage for the BAM run's CPU arm: map_reads as
    the reference's CPU path runs it (the oracle's cpu_map_reads: AVX-512
    scores and ties, scalar traceback, MD / NM, in C on every thread), its
    mappings handed to the library's BAM encoder."""

    def __init__(self, refs, scoring, local):
        from oracle import oracle as O
        self.O, self.refs, self.scoring, self.local = O, refs, scoring, local
        self.prof = O.Profile(refs, scoring)

    def map_reads(self, reads, min_score=0, max_ties=None, both_strands=False,
                  ref_letters=None, raw=False):
        O = self.O
        res, jobs, al, ops, mds, nm, _ = O.cpu_map_reads(
            *reads, self.refs, self.scoring, self.local, min_score=min_score,
            max_ties=max_ties, both_strands=both_strands, ref_letters=ref_letters,
            profile=self.prof)
        ms = O.cpu_mappings(res, jobs, al, ops, mds, nm)
        return _mappings_of(ms)


def _hit_of(h, words, md):
    """One map_reads-form hit dict as a HIT_DTYPE record, its CIGAR words
    and MD appended to `words` and `md`."""
    from eschalign_b200.scorer import HIT_DTYPE
    e = np.zeros((), HIT_DTYPE)
    for f in ("reference", "reverse", "score", "query_start", "query_end", "ref_start",
              "ref_end", "nm"):
        e[f] = int(h[f])
    w, num = [], ""
    for ch in h["cigar"]:
        if ch.isdigit():
            num += ch
        else:
            w.append(int(num) << 4 | "MIDNSHP=X".index(ch))
            num = ""
    e["ops_offset"], e["n_ops"] = len(words), len(w)
    words += w
    e["md_offset"], e["md_len"] = len(md), len(h["md"])
    md += h["md"].encode()
    return e


def _read_entry(r, m, hits, words, md):
    r["first_hit"], r["n_hits"], r["n_tied"] = len(hits), len(m["hits"]), m["n_tied"]
    if m["best_score"] is not None:
        r["best_score"], r["flags"] = m["best_score"], 1
    if m["suboptimal"] is not None:
        r["suboptimal"], r["flags"] = m["suboptimal"], r["flags"] | 2
    hits += [_hit_of(h, words, md) for h in m["hits"]]


def _mappings_of(ms, pms=None):
    """The oracle's per-read (or, with pms, per-pair) dicts as the arrays
    esg_map_reads / esg_map_pairs return."""
    from eschalign_b200.scorer import (HIT_DTYPE, MAPPING_DTYPE, PAIR_HIT_DTYPE,
                                       PAIR_MAPPING_DTYPE, Mappings)
    hits, words, md = [], [], bytearray()
    if pms is None:
        out = np.zeros(len(ms), MAPPING_DTYPE)
        for k, m in enumerate(ms):
            _read_entry(out[k], m, hits, words, md)
        return Mappings(out, np.array(hits, HIT_DTYPE), np.array(words, np.uint32), bytes(md))
    out = np.zeros(2 * len(pms), MAPPING_DTYPE)
    pairs = np.zeros(len(pms), PAIR_MAPPING_DTYPE)
    phits = []
    for p, pm in enumerate(pms):
        if not pm["proper"]:
            for m in range(2):
                _read_entry(out[2 * p + m], pm["mates"][m], hits, words, md)
            continue
        pr = pairs[p]
        sub = pm["suboptimal"]
        pr["flags"] = 1 | (2 if sub[0] is not None else 0) | (4 if sub[1] is not None else 0)
        pr["score"], pr["n_tied"], pr["n_hits"] = pm["score"], pm["n_tied"], len(pm["hits"])
        pr["suboptimal"] = [x if x is not None else 0 for x in sub]
        pr["first_hit"] = len(phits)
        for h in pm["hits"]:
            e = np.zeros((), PAIR_HIT_DTYPE)
            e["reference"], e["reverse"], e["insert"] = h["reference"], h["reverse"], h["insert"]
            e["mates"][0] = _hit_of(h["mates"][0], words, md)
            e["mates"][1] = _hit_of(h["mates"][1], words, md)
            phits.append(e)
    return Mappings(out, np.array(hits, HIT_DTYPE), np.array(words, np.uint32), bytes(md),
                    pairs, np.array(phits, PAIR_HIT_DTYPE))


class CpuPairMapper(CpuMapper):
    """map_pairs on the host cores for the paired BAM run's CPU arm (the
    oracle's cpu_map_pairs: AVX-512 ranking, scalar traceback, pair
    constraints, MD / NM, in C on every thread)."""

    def map_pairs(self, mates, min_score=0, max_ties=None, max_insert=500, both_strands=False,
                  ref_letters=None, raw=False):
        pms, _ = self.O.cpu_map_pairs(*mates, self.refs, self.scoring, self.local,
                                      min_score=min_score, max_ties=max_ties,
                                      max_insert=max_insert, both_strands=both_strands,
                                      ref_letters=ref_letters, profile=self.prof)
        return _mappings_of(None, pms)


def bam_stage(g, refs, reads, batch_size=50_000, cpu_reads=0, scoring=HEADLINE[0]):
    """The CLI's unpaired run through the library (bam.align_bam): an
    unaligned BAM of the workload's reads read, mapped on the device (every
    tie traced, MD / NM from the panel's letters), its records built and
    written as BGZF; wall time, input order, default batch size 50 000;
    `g` one scorer or several (one mapping thread each).  With cpu_reads,
    the CPU path on the first cpu_reads reads beside it: the same run with
    the mapping stage on the host cores (CpuMapper), the BAM I/O the same."""
    from eschalign_b200 import bam as EB
    names = [f"ref{k}" for k in range(len(refs))]
    letters = [bytes(b"ACGTN"[int(c)] for c in r) for r in refs]
    with tempfile.TemporaryDirectory() as tmp:
        src, dst = os.path.join(tmp, "in.bam"), os.path.join(tmp, "out.bam")
        raw = unmapped_bam(src, reads)
        in_bytes = os.path.getsize(src)
        warm = os.path.join(tmp, "warm.bam")
        unmapped_bam(warm, reads.slice(0, 2000))
        EB.align_bam(g, warm, dst, names, letters, both_strands=True, batch_size=1000)
        st = {}
        t0 = time.perf_counter()
        n = EB.align_bam(g, src, dst, names, letters, both_strands=True,
                         batch_size=batch_size, max_read_len=1000, stats=st)
        dt = time.perf_counter() - t0
        out_bytes = os.path.getsize(dst)
        # the same run with the blocks deflated on the host threads (zlib 6)
        sh = {}
        t0 = time.perf_counter()
        EB.align_bam(g, src, dst, names, letters, both_strands=True, batch_size=batch_size,
                     max_read_len=1000, stats=sh, deflate_on_device=False)
        dh = time.perf_counter() - t0
        host = {"reads_per_s": n["reads"] / dh, "seconds": round(dh, 3),
                "output_bgzf_bytes": os.path.getsize(dst),
                "stage_seconds": {k: round(v, 3) for k, v in sh.items()}}
        cpu = None
        if cpu_reads:
            small = os.path.join(tmp, "cpu.bam")
            unmapped_bam(small, reads.slice(0, cpu_reads))
            mapper = CpuMapper(refs, scoring, True)
            t0 = time.perf_counter()
            nc = EB.align_bam(mapper, small, dst, names, letters, both_strands=True,
                              batch_size=batch_size, max_read_len=1000)
            dc = time.perf_counter() - t0
            cpu = {"reads_per_s": nc["reads"] / dc, "kind": "port",
                   "cores": os.cpu_count(),
                   "sample": f"first {nc['reads']} reads: the same BAM run with the mapping "
                             "stage on the host cores (AVX-512 scores and ties, scalar "
                             "traceback, MD / NM, in C on all threads)"}
    out = {"reads": n["reads"], "records": n["records"], "seconds": round(dt, 3),
           "reads_per_s": n["reads"] / dt, "batch_reads": batch_size,
            "input_bgzf_bytes": in_bytes, "input_raw_bytes": raw, "output_bgzf_bytes": out_bytes,
            "stage_seconds": {k: round(v, 3) for k, v in st.items()},
           "scorers": len(g) if isinstance(g, (list, tuple)) else 1,
           "options": "both strands, min_score 0, every tie traced, MD/NM from letters, "
                      "input order; read, map (one thread per scorer) and encode/write "
                      "overlapped; output blocks deflated on the device",
           "host_deflate": host}
    if cpu:
        out["cpu"] = cpu
    return out


def fastq_files(path1, path2, pairs, seed=12):
    """Mates 2p and 2p + 1 of `pairs` as two FASTQ files (names p0000000..,
    Phred qualities 2-40), the CLI's usual paired input.  Built with array
    operations."""
    rng = np.random.default_rng(seed)
    letters = np.frombuffer(b"ACGTN", np.uint8)
    for m, path in ((0, path1), (1, path2)):
        idx = np.arange(m, len(pairs), 2)
        lens = pairs.lens[idx].astype(np.int64)
        offs = pairs.off[idx].astype(np.int64)
        n = idx.size
        size = 10 + lens + 3 + lens + 1         # @name\n seq \n+\n qual \n
        start = np.zeros(n + 1, np.int64)
        np.cumsum(size, out=start[1:])
        buf = np.full(int(start[-1]), ord("\n"), np.uint8)
        k = np.arange(n)
        head = np.zeros((n, 9), np.uint8)
        head[:, 0] = ord("@")
        head[:, 1] = ord("p")
        for d in range(7):
            head[:, 8 - d] = ord("0") + (k // 10 ** d) % 10
        buf[(start[:-1, None] + np.arange(9)).ravel()] = head.ravel()
        total = int(lens.sum())
        src = np.repeat(offs, lens) + (np.arange(total) - np.repeat(np.cumsum(lens) - lens, lens))
        seq_at = start[:-1] + 10
        rel = np.arange(total) - np.repeat(np.cumsum(lens) - lens, lens)
        buf[np.repeat(seq_at, lens) + rel] = letters[np.minimum(pairs.codes[src], 4)]
        plus_at = seq_at + lens
        buf[plus_at + 1] = ord("+")
        buf[np.repeat(plus_at + 3, lens) + rel] = rng.integers(35, 74, total, dtype=np.uint8)
        with open(path, "wb") as fh:
            fh.write(memoryview(buf))


def bam_pairs_stage(g, refs, pairs, n=500_000, batch_size=50_000, cpu_pairs=0):
    """The CLI's paired run through the library (bam.align_pairs_bam): the
    first n pairs as two FASTQ files, each mate trimmed of its adapter,
    mapped on the device (map_pairs_scored: every tie traced, MD / NM from
    the panel's letters), its records built and written as BGZF; wall time,
    input order, default batch size 50 000 records."""
    from eschalign_b200 import bam as EB
    names = [f"ref{k}" for k in range(len(refs))]
    letters = [bytes(b"ACGTN"[int(c)] for c in r) for r in refs]
    sub = pairs.slice(0, 2 * min(n, len(pairs) // 2))
    with tempfile.TemporaryDirectory() as tmp:
        p1, p2 = os.path.join(tmp, "r1.fq"), os.path.join(tmp, "r2.fq")
        w1, w2 = os.path.join(tmp, "w1.fq"), os.path.join(tmp, "w2.fq")
        dst = os.path.join(tmp, "out.bam")
        fastq_files(p1, p2, sub)
        fastq_files(w1, w2, sub.slice(0, 2000))
        EB.align_pairs_bam(g, w1, w2, dst, names, letters, min_score=40, batch_size=1000)
        st = {}
        t0 = time.perf_counter()
        r = EB.align_pairs_bam(g, p1, p2, dst, names, letters, min_score=40,
                               batch_size=batch_size, stats=st)
        dt = time.perf_counter() - t0
        out_bytes = os.path.getsize(dst)
        in_bytes = os.path.getsize(p1) + os.path.getsize(p2)
        sh = {}
        t0 = time.perf_counter()
        EB.align_pairs_bam(g, p1, p2, dst, names, letters, min_score=40,
                           batch_size=batch_size, stats=sh, deflate_on_device=False)
        dh = time.perf_counter() - t0
        host = {"pairs_per_s": r["reads"] / 2 / dh, "seconds": round(dh, 3),
                "output_bgzf_bytes": os.path.getsize(dst),
                "stage_seconds": {k: round(v, 3) for k, v in sh.items()}}
        cpu = None
        if cpu_pairs:
            c1, c2 = os.path.join(tmp, "c1.fq"), os.path.join(tmp, "c2.fq")
            fastq_files(c1, c2, sub.slice(0, 2 * cpu_pairs))
            mapper = CpuPairMapper(refs, C4_SCORING, False)
            t0 = time.perf_counter()
            rc = EB.align_pairs_bam(mapper, c1, c2, dst, names, letters, min_score=40,
                                    batch_size=batch_size)
            dc = time.perf_counter() - t0
            cpu = {"pairs_per_s": rc["reads"] / 2 / dc, "kind": "port", "cores": os.cpu_count(),
                   "sample": f"first {rc['reads'] // 2} pairs: the same paired BAM run with "
                             "the paired mapping stage on the host cores (AVX-512 ranking, "
                             "scalar traceback, MD / NM, in C on all threads)"}
    out = {"pairs": r["reads"] // 2, "records": r["records"], "seconds": round(dt, 3),
           "scorers": len(g) if isinstance(g, (list, tuple)) else 1,
           "pairs_per_s": r["reads"] / 2 / dt, "batch_records": batch_size,
           "input_fastq_bytes": in_bytes, "output_bgzf_bytes": out_bytes,
           "stage_seconds": {k: round(v, 3) for k, v in st.items()},
           "options": "semi-global, --min-score 40, max insert 500, forward template strand, "
                      "TruSeq adapters trimmed, every tie traced, MD/NM from letters, "
                      "input order; output blocks deflated on the device",
           "host_deflate": host}
    if cpu:
        out["cpu"] = cpu
    return out


def map_pairs_stage(g, refs, pairs, scoring, local, skip_cpu, n=100_000):
    """The whole paired mapping stage: adapters trimmed by the library
    (esg_pair_adapters), then esg_map_pairs (pair.rs:157-390: the device
    ranking, the first tiers traced, deeper tiers from full rows, the
    Separate fallback, MD / NM); wall time of both calls with host buffers,
    the CLI's paired options (--min-score 40, max insert 500, both template
    strands).  Beside it the same stage on the host cores (the oracle's
    cpu_map_pairs: C trimming and AVX-512 ranking, scalar traceback of the
    first tiers, MD / NM, all threads) on a bounded sample."""
    from eschalign_b200 import adapter
    sub = pairs.slice(0, 2 * n)
    codes, off, _ = sub.tuple()

    def run(k0, k1):
        part = sub.slice(2 * k0, 2 * k1)
        _, aligned = adapter.pair_adapters(part.tuple())
        c, o, _ = part.tuple()
        return g.map_pairs((c, o, aligned), min_score=40, max_insert=500, both_strands=True,
                           raw=True)

    run(0, 1000).free()  # warm-up
    t0 = time.perf_counter()
    h = run(0, len(sub) // 2)
    dt = time.perf_counter() - t0
    t1 = time.perf_counter()
    m = h.mappings(paired=True)  # copied out to Python, as the Python binding returns it
    dt_copy = time.perf_counter() - t1
    h.free()
    n_pairs = len(sub) // 2
    proper = int((m.pairs["flags"] & 1).sum())
    out = {"pairs": n_pairs, "seconds": round(dt, 4), "pairs_per_s": n_pairs / dt,
           "pairs_per_s_with_python_copy": n_pairs / (dt + dt_copy),
           "proper": proper, "pair_hits": int(m.pair_hits.size),
           "options": "trim + map: min_score 40, max_insert 500, both template strands, "
                      "every tie traced, MD/NM without letters; the mapping as the C ABI "
                      "returns it (esg_map_pairs)"}
    if not skip_cpu:
        from oracle import oracle as O
        k = min(n_pairs, 20_000)
        prof = O.Profile(refs, scoring)
        part = sub.slice(0, 2 * k)
        O.cpu_map_pairs(*part.slice(0, 200).tuple(), refs, scoring, local, min_score=40,
                        max_insert=500, both_strands=True, profile=prof, trim=True)  # warm-up
        t0 = time.perf_counter()
        _, used = O.cpu_map_pairs(*part.tuple(), refs, scoring, local, min_score=40,
                                  max_insert=500, both_strands=True, profile=prof, trim=True)
        dt_c = time.perf_counter() - t0
        out["cpu"] = {"pairs_per_s": k / dt_c, "kind": "port", "cores": int(used),
                      "sample": f"first {k} pairs: trimming, AVX-512 rows and ranking, scalar "
                                "traceback of the first tiers, MD / NM, in C on all threads"}
    return out


def reference_gpu_arms(refs, reads, scoring, local, device):
    """Comparison arms: the reference's own align_score_kernel (int) and
    align_score_kernel_h2 (half2), compiled ahead of time for sm_100a from its
    source and launched as its GpuScorer does (oracle/ref_gpu, built where
    the reference tree is present), on `reads` and their reverse complements
    -- the queries its CLI feeder submits for both strands.  A reported
    baseline, like cpu_baseline; None where the arms were not built."""
    from oracle import oracle as O
    if not (os.path.exists(O.REF_GPU_LIB) and os.path.exists(O.REF_GPU_CUBIN)):
        return None
    rg = O.RefGpu(refs, device=device)
    fwd = reads.list()
    qc, qo, ql = O.pack(fwd + [O.revcomp(r) for r in fwd])
    cells = int(ql.sum(dtype=np.uint64)) * sum(len(r) for r in refs)
    out = {"kind": "reference", "sample": f"{len(fwd)} reads + reverse complements"}
    for kernel, name in ((0, "int"), (1, "half2")):
        _, ms = rg.score(qc, qo, ql, scoring, local, kernel=kernel, reps=2, rows=False)
        out[f"{name}_gcups"] = cells / (ms / 1e3) / 1e9
        out[f"{name}_geometry"] = rg.geometry(kernel)
    rg.close()
    return out


def run_reference(a, rank, world):
    """--impl reference: rank 0 times the CPU path; other ranks exit."""
    if rank != 0:
        return
    from eschalign_b200 import synth
    per_step = max(2.0, min(a.cpu_seconds, 120.0 / max(1, a.steps + a.warmup)))
    extra = {}
    if a.workload == "c4":
        refs = synth.panel_tiles()
        data = synth.pairs_c4(refs, n=a.pairs)[0]
        fn = lambda s: cpu_pairs_baseline(refs, data, C4_SCORING, s)  # noqa: E731
        warm = lambda: cpu_pairs_baseline(refs, data.slice(0, 2000), C4_SCORING, 0.5)  # noqa: E731
        workload = (f"C4 {a.pairs} pairs 2x150 x 164-ref panel, semiglobal 2,-1,-10,-1, "
                    "adapter trimming, both template strands ranked")
        dtype = "int16"
    elif a.workload == "c3":
        refs = synth.panel_c3()
        data = synth.reads_c3(refs, n=a.c3_reads)
        fn = lambda s: cpu_baseline(refs, data, C3_SCORING, "local", s, chunk=1)  # noqa: E731
        warm = lambda: cpu_baseline(refs, data.slice(0, 64), C3_SCORING, "local", 0.5,  # noqa: E731
                                    chunk=1)
        workload = "C3 10000 refs (300-1000 nt) x reads 50-1000 nt, both strands, local"
        dtype = "int16"
    elif a.workload == "c1":
        refs = synth.panel_tiles()
        data = synth.reads_c1(refs)
        panel_bases = sum(len(r) for r in refs)

        def fn(_s):
            from oracle import oracle as O
            O.build()
            prof = O.Profile(refs, C3_SCORING)
            t0 = time.perf_counter()
            _, _, _, used = prof.map_batch(*data.tuple(), local=True, both_strands=False)
            dt = time.perf_counter() - t0
            return {"value": data.bases() * panel_bases / dt / 1e9, "unit": "GCUPS",
                    "cores": int(used), "kind": "port", "seconds": dt,
                    "sample": f"all {len(data)} reads, forward strand, local 2,-1,-10,-1"}
        warm = lambda: fn(0)  # noqa: E731
        workload = "C1 10 000 reads x 164-ref panel, forward strand, local 2,-1,-10,-1"
        dtype = "int16"
    elif a.workload == "c5":
        # the reference has no serving mode: its CPU path's throughput on the
        # request mix's large panel (2000 x 300 nt), both strands
        refs = synth.panel(2000, 300, 300, 0x5EED_0C5B)
        rng = np.random.default_rng(0x5EED_0C05)
        data = synth.mixed_reads(rng, refs, synth.lognormal_lengths(rng, 50_000, 110, 0.4, 20,
                                                                    1000), 0.9, 0.08, 0.02, 0.01)
        fn = lambda s: cpu_baseline(refs, data, C3_SCORING, "local", s)  # noqa: E731
        warm = lambda: cpu_baseline(refs, data.slice(0, 500), C3_SCORING, "local", 0.5)  # noqa: E731
        workload = ("C5 request mix: the reference has no serving mode; its CPU path on "
                    "panel B (2000 x 300 nt) reads, both strands, local 2,-1,-10,-1")
        dtype = "int16"
    else:
        refs = synth.panel_tiles()
        data = synth.reads_c2(refs, n=a.reads)
        scoring, mode = HEADLINE
        fn = lambda s: cpu_baseline(refs, data, scoring, mode, s)  # noqa: E731
        warm = lambda: cpu_baseline(refs, data.slice(0, 2000), scoring, mode, 0.5)  # noqa: E731
        workload = "C2 1M reads x 164-ref panel, both strands, local 2,-1,-10,-1"
        dtype = "int16"
    for _ in range(a.warmup):
        warm()
    vals, last = [], None
    for _ in range(a.steps):
        last = fn(per_step)
        vals.append(last["value"])
    v = statistics.median(vals)
    if a.workload == "c4":
        extra["pairs_per_s"] = last["pairs_per_s"] * v / last["value"]
    elif a.workload == "c2":
        cells_per_read = 2 * (data.bases() / len(data)) * sum(len(r) for r in refs)
        extra["reads_per_s"] = v * 1e9 / cells_per_read
    line = {
        "impl": "reference", "metric": "GCUPS", "value": v, "unit": "GCUPS", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * last["seconds"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic", **extra,
        "config": {"workload": workload, "refs": len(refs)},
        "cpu_baseline": {k: v2 for k, v2 in {**last, "value": v}.items()
                         if k not in ("seconds", "reads_per_s", "pairs_per_s")
                         and not k.startswith("_")},
        "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class Ctx:
    """Per-rank device plumbing: stream, L2 flush buffer, barrier, max over
    ranks, and the device timer of a batch's launch sequence."""

    def __init__(self, torch, dist, dev, local_rank, world):
        self.torch, self.dist, self.dev = torch, dist, dev
        self.local_rank, self.world = local_rank, world
        self.stream = torch.cuda.Stream(device=dev)
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > L2 (126 MB)

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max_over_ranks(self, x):
        if self.world == 1:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x):
        if self.world == 1:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def device_time(self, scorer, batch, steps, warmup, sampler=None):
        torch, stream = self.torch, self.stream
        for _ in range(warmup):
            scorer.relaunch(batch, stream.cuda_stream)
        torch.cuda.synchronize()
        self.barrier()
        total = 0.0
        with (sampler if sampler is not None else _Null()):
            for k in range(steps):
                with torch.cuda.stream(stream):
                    self.flush.fill_(k & 0xFF)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                scorer.relaunch(batch, stream.cuda_stream)
                e1.record(stream)
                e1.synchronize()
                total += e0.elapsed_time(e1) / 1e3
        torch.cuda.synchronize()
        self.barrier()
        return total


def feeder(ctx, run, steps):
    """The end-to-end passes through the library's GPU feeder
    (GpuScorer.score_batches / score_pair_batches, the CLI's score_batches,
    crates/eschalign-cli/src/align.rs:2801-2917): run(timing) yields each
    chunk's result, chunk k + 1 prepared and queued before chunk k is waited
    for, so the device never drains between chunks.  Returns (seconds of the
    timed passes, passes, h2d bytes, d2h bytes per pass); the host time split
    is left in feeder.last_split.  The first pass warms the pinned pool and
    the allocator and is not timed."""
    times, h2d, d2h = [], 0, 0
    host = {"prepare_s": 0.0, "submit_s": 0.0, "finish_s": 0.0}
    pc = time.perf_counter
    for it in range(steps + 1):
        ctx.barrier()
        t0 = pc()
        h2d = d2h = 0
        split = {}
        for res in run(split):
            h2d += res.stats["h2d_bytes"]
            d2h += res.stats["d2h_bytes"]
        ctx.torch.cuda.synchronize()
        dt = pc() - t0
        if it > 0:
            times.append(dt)
            for k in host:
                host[k] += split[k] / steps
    feeder.last_split = {k: round(v, 4) for k, v in host.items()}
    return ctx.max_over_ranks(sum(times)), len(times), h2d, d2h


def tune(g, a, lengths=None):
    """The autotuner's report (on the workload's length histogram when a
    sample of its read lengths is given), or the pinned split (--split)."""
    if a.no_graphs:
        g.set_graphs(False)
    if a.split >= 0:
        g.set_split(a.split)
        return {"split_len": a.split, "pinned": True}
    return g.autotune(lengths)


def common_line(a, ctx, value, ms_per_step, workload, extra_config, e2e, roofline, clocks,
                launches, dtype="int16x2"):
    return {
        "metric": "GCUPS", "value": value, "unit": "GCUPS", "n_gpus": ctx.world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic",
        "config": {"workload": workload, **extra_config, "parallelism": f"replicas x{ctx.world}",
                   "l2": "flushed (256 MB write) between timed steps"},
        "e2e": e2e, "roofline": roofline, "clocks": clocks, "gpu_launches": launches,
    }


# ---------------------------------------------------------------- C2
def run_c2(a, ctx, rank):
    from eschalign_b200 import (KERNEL_AUTO, KERNEL_INT32, KERNEL_PLAIN32, GpuScorer, Mode,
                                Scoring, synth)
    world, local_rank = ctx.world, ctx.local_rank
    refs = synth.panel_tiles()
    panel_bases = sum(len(r) for r in refs)
    if a.bam_case:
        reads = synth.reads_c2(refs, n=a.bam_case)
        gs = [GpuScorer(refs, Scoring(*HEADLINE[0]), Mode.parse(a.mode), device=local_rank)
              for _ in range(max(1, a.bam_scorers))]
        for g in gs:
            g.set_split(a.split if a.split >= 0 else 512)
        print(json.dumps({"bam_case": a.bam_case, **bam_stage(gs, refs, reads)}), flush=True)
        for g in gs:
            g.close()
        return
    if a.profile_case:
        reads = synth.reads_c2(refs, n=a.profile_case)
        for kernel in (KERNEL_AUTO, KERNEL_INT32, KERNEL_PLAIN32):
            g = GpuScorer(refs, Scoring(*HEADLINE[0]), Mode.parse(a.mode), device=local_rank,
                          kernel=kernel)
            if a.split >= 0:
                g.set_split(a.split)
            r = g.score_batch(reads.tuple(), both_strands=True)
            print(json.dumps({"profile_case": a.profile_case, "kernel": kernel,
                              "stats": r.stats}), flush=True)
            g.close()
        return
    # weak scaling: the job is a.reads reads per GPU, cut into this rank's
    # slice the way the library shards a batch (replicas.shard: contiguous,
    # balanced by cells); one GPU scores the whole a.reads
    if world > 1:
        from eschalign_b200 import replicas
        reads, _ = replicas.shard(synth.reads_c2(refs, n=a.reads * world), rank, world)
    else:
        reads = synth.reads_c2(refs, n=a.reads)
    extras = {}
    scoring, mode = HEADLINE
    g = GpuScorer(refs, Scoring(*scoring), Mode.parse(mode), device=local_rank,
                  stream=ctx.stream.cuda_stream)
    tune_rep = tune(g, a, reads.lens[:20000])  # tile shape for this panel, before any timing
    info = g.info()
    batch = g.submit(g.prepare(reads.tuple(), both_strands=True))
    first = g.finish(batch, keep=True)
    st = first.stats
    cells = st["cells"]
    sampler = ClockSampler(local_rank)
    t = ctx.device_time(g, batch, a.steps, a.warmup, sampler)
    clocks = sampler.summary()
    t_max = ctx.max_over_ranks(t)
    job_cells = ctx.sum_over_ranks(cells)  # every rank's slice
    job_reads = ctx.sum_over_ranks(len(reads))
    value = job_cells * a.steps / t_max / 1e9
    # the timed launches' results (the last one's, in device memory) against
    # the submit's, every read
    timed_res, timed_ties = g.read_results(batch)
    parity = {"reads": len(reads),
              "timed_launch_equals_submit": same_results(timed_res, timed_ties, first.results,
                                                         first.ties)}
    peak = int_peak(local_rank)
    roofline = roofline_of(peak, cells * a.steps / t, mode,
                           K2_DRAM_BYTES_PER_CELL * cells if K2_DRAM_BYTES_PER_CELL else None)
    if peak:
        extras["int_probe"] = {k: round(v["lane_ops_per_s"] / 1e12, 3)
                               for k, v in peak["ops"].items()}
        extras["int_probe_per_sm_clk"] = {k: round(v["per_sm_per_clk"], 2)
                                          for k, v in peak["ops"].items()}
    batch.free()

    if not a.no_extras:
        combos = {}
        for sc_, md in COMBOS[1:]:
            g2 = GpuScorer(refs, Scoring(*sc_), Mode.parse(md), device=local_rank,
                           stream=ctx.stream.cuda_stream)
            tune(g2, a, reads.lens[:20000])
            b2 = g2.submit(g2.prepare(reads.tuple(), both_strands=True))
            r2 = g2.finish(b2, keep=True)
            t2 = ctx.max_over_ranks(ctx.device_time(g2, b2, 1, 1))
            combos[f"{md} {','.join(map(str, sc_))}"] = round(world * r2.stats["cells"] / t2 / 1e9, 1)
            b2.free()
            g2.close()
        combos[f"{mode} {','.join(map(str, scoring))}"] = round(value, 1)
        extras["gcups_by_combo"] = combos
        # the int32 arms on a sample of the same batch: every query on the
        # int32 lanes, and int32 one thread per (query, reference) -- the
        # plain kernel's design; results equal the batched kernel's
        sub = reads.slice(0, min(a.plain_reads, len(reads)))
        for kernel, key in ((KERNEL_INT32, "int32_lanes_gcups"), (KERNEL_PLAIN32, "plain_gcups")):
            g.set_kernel(kernel)
            bp = g.submit(g.prepare(sub.tuple(), both_strands=True))
            rp = g.finish(bp, keep=True)
            tp = ctx.max_over_ranks(ctx.device_time(g, bp, 1, 1))
            extras[key] = world * rp.stats["cells"] / tp / 1e9
            n_sub = len(sub)
            parity[f"{key[:-6]}_equals_batched"] = same_results(
                rp.results, rp.ties, first.results[:n_sub], first.ties[:n_sub])
            bp.free()
        g.set_kernel(KERNEL_AUTO)
        extras["batched_over_plain"] = value / extras["plain_gcups"]
        extras["batched_over_int32_lanes"] = value / extras["int32_lanes_gcups"]
        extras["plain_sample"] = f"first {len(sub)} reads, both strands"
        extras["traceback"] = traceback_stage(g, refs, sub, scoring, mode == "local",
                                              a.no_cpu_baseline or rank != 0 or world != 1)
        extras["map"] = map_stage(g, refs, reads, scoring, mode == "local",
                                  a.no_cpu_baseline or rank != 0 or world != 1)
        if world == 1:
            # the BAM run, a single-GPU figure: a second scorer over the same
            # panel maps while the other's host share of the mapping runs
            g2 = GpuScorer(refs, Scoring(*scoring), Mode.parse(mode), device=local_rank)
            g2.set_split(info["split_len"])
            extras["bam"] = bam_stage([g, g2], refs, reads,
                                      cpu_reads=0 if a.no_cpu_baseline else 40_000)
            g2.close()
        arms = reference_gpu_arms(refs, sub, scoring, mode == "local", local_rank)
        if arms:
            arms["batched_over_ref_half2"] = value / arms["half2_gcups"]
            # the reference's own one-thread-per-pair int kernel
            arms["batched_over_ref_int"] = value / arms["int_gcups"]
            extras["reference_gpu_kernels"] = arms

    chunks = [reads.slice(k, k + a.chunk) for k in range(0, len(reads), a.chunk)]
    te, n_pass, h2d, d2h = feeder(
        ctx, lambda tm: g.score_batches((c.tuple() for c in chunks), both_strands=True,
                                        timing=tm), max(1, a.steps))
    e2e = {"value": job_cells * n_pass / te / 1e9, "unit": "GCUPS",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "reads_per_s": job_reads * n_pass / te, "chunk_reads": a.chunk,
           "host_seconds_per_pass": feeder.last_split}
    g.close()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(refs, reads, scoring, mode, a.cpu_seconds)
        extras["cpu_reads_per_s"] = cpu.pop("reads_per_s")
        cpu.pop("seconds", None)
        # the CPU path's results on its sample (the first reads of the
        # workload) against the GPU's for the same reads
        c_res, c_ties = cpu.pop("_results")
        n = len(c_res)
        parity["cpu_sample_reads"] = n
        parity["cpu_sample_equal"] = same_results(first.results[:n], first.ties[:n], c_res,
                                                  c_ties)
    if rank == 0:
        line = common_line(
            a, ctx, value, 1e3 * t_max / a.steps,
            "C2: 1M reads (lognormal median 110 nt) x 164-ref panel (70-180 nt), both "
            "strands, local 2,-1,-10,-1, best + XS + 8 ties per read",
            {"reads": int(job_reads), "refs": len(refs), "panel_bases": panel_bases,
             "cells_per_step": int(job_cells),
             "sharding": "replicas.shard: contiguous slices balanced by cells"},
            e2e, roofline, clocks, st["kernels"] * a.steps)
        line["reads_per_s"] = job_reads * a.steps / t_max
        line["kernel_info"] = {k: info[k] for k in (
            "regs_batched", "regs_plain", "local_bytes_batched", "batched_blocks",
            "panel_bytes", "sm_count", "split_len")}
        line["autotune"] = tune_rep
        line["batch_stats"] = {k: st[k] for k in ("queries_batched", "queries_plain",
                                                  "queries_rescored", "tasks", "lanes_used")}
        line["parity"] = parity
        if cpu:
            line["cpu_baseline"] = cpu
        line.update(extras)
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- C1
def run_c1(a, ctx, rank):
    from eschalign_b200 import GpuScorer, Mode, Scoring, synth
    world, local_rank = ctx.world, ctx.local_rank
    scoring = (2, -1, -10, -1)
    refs = synth.panel_tiles()
    panel_bases = sum(len(r) for r in refs)
    reads = synth.reads_c1(refs)
    g = GpuScorer(refs, Scoring(*scoring), Mode.LOCAL, device=local_rank,
                  stream=ctx.stream.cuda_stream)
    tune_rep = tune(g, a, reads.lens)
    batch = g.submit(g.prepare(reads.tuple()))
    st = g.finish(batch, keep=True).stats
    cells = st["cells"]
    sampler = ClockSampler(local_rank)
    t = ctx.device_time(g, batch, a.steps, a.warmup, sampler)
    clocks = sampler.summary()
    t_max = ctx.max_over_ranks(t)
    value = world * cells * a.steps / t_max / 1e9
    peak = int_peak(local_rank)
    roofline = roofline_of(peak, cells * a.steps / t, "local", None)
    batch.free()
    te, n_pass, h2d, d2h = feeder(ctx, lambda tm: g.score_batches([reads.tuple()], timing=tm),
                                  max(3, a.steps))
    e2e = {"value": world * cells * n_pass / te / 1e9, "unit": "GCUPS",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "reads_per_s": world * len(reads) * n_pass / te}
    g.close()
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        prof = O.Profile(refs, scoring)
        prof.map_batch(*reads.tuple(), local=True, both_strands=False)  # warm-up
        t0 = time.perf_counter()
        _, _, _, used = prof.map_batch(*reads.tuple(), local=True, both_strands=False)
        dt = time.perf_counter() - t0
        cpu = {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": int(used), "kind": "port",
               "sample": f"all {len(reads)} reads, forward strand; {dt:.3f} s; "
                         f"reads/s {len(reads) / dt:.0f}"}
    if rank == 0:
        line = common_line(
            a, ctx, value, 1e3 * t_max / a.steps,
            "C1: 10 000 reads (60-200 nt, 90 % derived) x 164-ref panel (70-180 nt), local "
            "2,-1,-10,-1, forward strand, int32 scores",
            {"reads": len(reads), "refs": len(refs), "panel_bases": panel_bases,
             "cells_per_step": cells},
            e2e, roofline, clocks, st["kernels"] * a.steps)
        line["reads_per_s"] = world * len(reads) * a.steps / t_max
        line["autotune"] = tune_rep
        line["batch_stats"] = {k: st[k] for k in ("queries_batched", "tasks", "panel_chunks",
                                                  "kernels")}
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- C4
def run_c4(a, ctx, rank):
    from eschalign_b200 import GpuScorer, Mode, Scoring, adapter, synth
    world, local_rank = ctx.world, ctx.local_rank
    refs = synth.panel_tiles()
    panel_bases = sum(len(r) for r in refs)
    t0 = time.perf_counter()
    pairs, _ = synth.pairs_c4(refs, n=a.pairs)
    gen_s = time.perf_counter() - t0
    n_pairs = len(pairs) // 2
    cfg = adapter.config()
    g = GpuScorer(refs, Scoring(*C4_SCORING), Mode.SEMIGLOBAL, device=local_rank,
                  stream=ctx.stream.cuda_stream)
    # the lengths the scorer sees: mates after adapter trimming
    _, trimmed = adapter.pair_adapters(pairs.slice(0, 40_000).tuple(), cfg)
    tune_rep = tune(g, a, trimmed)
    batch = g.submit(g.prepare_pairs(pairs.tuple(), adapters=cfg, both_strands=True))
    st = g.finish_pairs(batch, keep=True).stats
    cells = st["cells"]
    sampler = ClockSampler(local_rank)
    t = ctx.device_time(g, batch, a.steps, a.warmup, sampler)
    clocks = sampler.summary()
    t_max = ctx.max_over_ranks(t)
    value = world * cells * a.steps / t_max / 1e9
    peak = int_peak(local_rank)
    roofline = roofline_of(peak, cells * a.steps / t, "semiglobal", None)
    batch.free()
    map_pairs = bam_pairs = None
    if not a.no_extras:
        map_pairs = map_pairs_stage(g, refs, pairs, C4_SCORING, False,
                                    a.no_cpu_baseline or rank != 0 or world != 1)
        if world == 1:
            g2 = GpuScorer(refs, Scoring(*C4_SCORING), Mode.SEMIGLOBAL, device=local_rank)
            g2.set_split(g.info()["split_len"])
            bam_pairs = bam_pairs_stage([g, g2], refs, pairs,
                                        cpu_pairs=0 if a.no_cpu_baseline else 20_000)
            g2.close()
    step_pairs = a.pair_chunk
    chunks = [pairs.slice(2 * k, 2 * (k + step_pairs)) for k in range(0, n_pairs, step_pairs)]
    te, n_pass, h2d, d2h = feeder(
        ctx, lambda tm: g.score_pair_batches((c.tuple() for c in chunks), adapters=cfg,
                                             both_strands=True, timing=tm),
        max(1, min(2, a.steps)))
    e2e = {"value": world * cells * n_pass / te / 1e9, "unit": "GCUPS",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "pairs_per_s": world * n_pairs * n_pass / te, "chunk_pairs": step_pairs,
           "host_seconds_per_pass": feeder.last_split}
    g.close()
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_pairs_baseline(refs, pairs, C4_SCORING, a.cpu_seconds)
        cpu.pop("seconds", None)
    if rank == 0:
        line = common_line(
            a, ctx, value, 1e3 * t_max / a.steps,
            f"C4: {n_pairs} pairs 2x150 (insert lognormal median 90, adapter read-through) x "
            "164-ref panel, semiglobal 2,-1,-10,-1; mates trimmed on the host, 4 mate queries "
            "per pair, both template strands ranked on the device (best sum, tie set, next "
            "tier, per-mate XS) + each mate's own both-strand result",
            {"pairs": n_pairs, "refs": len(refs), "panel_bases": panel_bases,
             "cells_per_step": cells, "mates_trimmed": st["mates_trimmed"],
             "bases_trimmed": st["bases_trimmed"], "generate_s": round(gen_s, 1)},
            e2e, roofline, clocks, st["kernels"] * a.steps)
        line["pairs_per_s"] = world * n_pairs * a.steps / t_max
        line["reads_per_s"] = 2 * line["pairs_per_s"]
        line["autotune"] = tune_rep
        line["batch_stats"] = {k: st[k] for k in ("queries_batched", "queries_plain",
                                                  "queries_rescored", "tasks", "lanes_used",
                                                  "kernels")}
        if cpu:
            line["cpu_baseline"] = cpu
        if map_pairs:
            line["map_pairs"] = map_pairs
        if bam_pairs:
            line["bam_pairs"] = bam_pairs
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- C3
def run_c3(a, ctx, rank):
    from eschalign_b200 import GpuScorer, Mode, Scoring, synth
    world, local_rank = ctx.world, ctx.local_rank
    refs = synth.panel_c3()
    panel_bases = sum(len(r) for r in refs)
    reads = synth.reads_c3(refs, n=a.c3_reads)
    g = GpuScorer(refs, Scoring(*C3_SCORING), Mode.LOCAL, device=local_rank,
                  stream=ctx.stream.cuda_stream)
    tune_rep = tune(g, a, reads.lens)
    info = g.info()
    batch = g.submit(g.prepare(reads.tuple(), both_strands=True))
    st = g.finish(batch, keep=True).stats
    cells = st["cells"]
    sampler = ClockSampler(local_rank)
    t = ctx.device_time(g, batch, a.steps, a.warmup, sampler)
    clocks = sampler.summary()
    t_max = ctx.max_over_ranks(t)
    value = world * cells * a.steps / t_max / 1e9
    peak = int_peak(local_rank)
    roofline = roofline_of(peak, cells * a.steps / t, "local", None)
    batch.free()
    te, n_pass, h2d, d2h = feeder(
        ctx, lambda tm: g.score_batches([reads.tuple()], both_strands=True, timing=tm), 1)
    e2e = {"value": world * cells * n_pass / te / 1e9, "unit": "GCUPS",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    g.close()
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(refs, reads, C3_SCORING, "local", a.cpu_seconds, chunk=1)
        cpu.pop("seconds", None)
        cpu.pop("reads_per_s", None)
        cpu.pop("_results", None)
    if rank == 0:
        line = common_line(
            a, ctx, value, 1e3 * t_max / a.steps,
            f"C3: {len(reads)} reads (50-1000 nt, 70 % derived) x 10 000-ref panel "
            "(300-1000 nt), both strands, local 2,-1,-10,-1, autotuned tile shape",
            {"reads": len(reads), "refs": len(refs), "panel_bases": panel_bases,
             "cells_per_step": cells},
            e2e, roofline, clocks, st["kernels"] * a.steps)
        line["autotune"] = tune_rep
        line["kernel_info"] = {k: info[k] for k in ("panel_bytes", "split_len",
                                                    "batched_blocks")}
        line["batch_stats"] = {k: st[k] for k in ("queries_batched", "queries_plain",
                                                  "queries_rescored", "tasks", "lanes_used",
                                                  "kernels")}
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- C5
def run_c5(a, ctx, rank):
    import threading

    from eschalign_b200 import GpuScorer, Mode, Scoring, synth
    from eschalign_b200.server import Server
    world, local_rank = ctx.world, ctx.local_rank
    scoring = (2, -1, -10, -1)
    panels = {"A": synth.panel_tiles(), "B": synth.panel(2000, 300, 300, 0x5EED_0C5B)}
    pbases = {k: sum(len(r) for r in v) for k, v in panels.items()}
    rng = np.random.default_rng(0x5EED_0C05)
    pool_n = 400_000
    pools = {"A": synth.reads_c2(panels["A"], n=pool_n, seed=0x5EED_0C5A),
             "B": synth.mixed_reads(rng, panels["B"],
                                    synth.lognormal_lengths(rng, pool_n, 110, 0.4, 20, 1000),
                                    0.9, 0.08, 0.02, 0.01)}
    specs = [("A", Mode.LOCAL), ("A", Mode.SEMIGLOBAL), ("B", Mode.LOCAL), ("B", Mode.SEMIGLOBAL)]
    scorers = []
    tunes = {}
    for pk, md in specs:
        g = GpuScorer(panels[pk], Scoring(*scoring), md, device=local_rank)
        tunes[f"{pk} {md.label}"] = tune(g, a, pools[pk].lens[:20000])["split_len"]
        scorers.append(g)
    rates = [float(x) for x in a.rates.split(",") if x]
    per_rate = []
    verify = []
    clocks = None
    with Server(scorers, max_batch_cells=a.max_batch_cells) as sv:
        for ri, rate in enumerate(rates):
            # the same requests (sizes, panels, modes, strands, reads) at
            # every rate, so rates differ only in arrival times; the
            # arrivals of each rate are its own Poisson draw
            rr = np.random.default_rng(0x5EED_0C05)
            n_req = a.requests
            sizes = np.floor(np.exp(rr.uniform(0, np.log(50_000), n_req))).astype(np.int64)
            slots = rr.integers(0, 4, n_req)
            both = rr.random(n_req) < 0.5
            starts = [int(rr.integers(0, pool_n - sizes[k] + 1)) for k in range(n_req)]
            gaps = np.random.default_rng([0x5EED_0C05, ri]).exponential(1.0 / rate, n_req)
            reqs = []
            for k in range(n_req):
                pk = specs[slots[k]][0]
                start = starts[k]
                reqs.append((int(slots[k]), pools[pk].slice(start, start + int(sizes[k])),
                             bool(both[k])))
            cells = sum(int(r[1].bases()) * (2 if r[2] else 1) * pbases[specs[r[0]][0]]
                        for r in reqs)
            tickets = [None] * n_req
            results = [None] * n_req
            ready = threading.Semaphore(0)

            def waiter():
                for k in range(n_req):
                    ready.acquire()
                    results[k] = sv.wait(tickets[k])

            th = threading.Thread(target=waiter)
            th.start()
            sampler = ClockSampler(local_rank)
            with sampler:
                t0 = time.perf_counter()
                due = t0
                for k in range(n_req):
                    due += gaps[k]
                    dt = due - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                    slot, rd, bs = reqs[k]
                    tickets[k] = sv.submit(slot, rd.tuple(), bs)
                    ready.release()
                th.join()
                t_end = time.perf_counter()
            if ri == len(rates) - 1:
                clocks = sampler.summary()
            else:
                sampler.summary()
            lat = np.array([results[k][1].total_ms for k in range(n_req)])
            small = sizes <= 1000

            def pct(x, q):
                return round(float(np.percentile(x, q)), 2) if x.size else None
            queued = np.array([results[k][1].queued_ms for k in range(n_req)])
            bsz = np.array([results[k][1].batch_requests for k in range(n_req)])
            span = t_end - t0
            per_rate.append({
                "rate_req_s": rate, "requests": n_req, "reads": int(sizes.sum()),
                "achieved_req_s": round(n_req / span, 1),
                "gcups": round(cells / span / 1e9, 1),
                "p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2),
                "p999_ms": round(float(np.percentile(lat, 99.9)), 2),
                "small_le_1000_reads": {"requests": int(small.sum()),
                                        "p50_ms": pct(lat[small], 50),
                                        "p99_ms": pct(lat[small], 99)},
                "large": {"requests": int((~small).sum()), "p50_ms": pct(lat[~small], 50),
                          "p99_ms": pct(lat[~small], 99)},
                "mean_queued_ms": round(float(queued.mean()), 2),
                "mean_requests_per_batch": round(float(bsz.mean()), 2),
                "seconds": round(span, 2),
                "h2d_bytes": int(sum(r[1].bases() for r in reqs)),
                "d2h_bytes": int(sizes.sum()) * (16 + 4 * scorers[0].cap)})
            # bit-exact in the mix: a sample re-scored alone after the run
            for k in list(np.argsort(sizes)[:3]) + [int(np.argmax(sizes))]:
                verify.append((reqs[k], results[k][0]))
        st = sv.stats()
    ok = 0
    alone = {}
    for (slot, rd, bs), got in verify:
        pk, md = specs[slot]
        key = (pk, md)
        if key not in alone:
            alone[key] = GpuScorer(panels[pk], Scoring(*scoring), md, device=local_rank)
        want = alone[key].score_batch(rd.tuple(), both_strands=bs)
        same = all(np.array_equal(got.results[f], want.results[f])
                   for f in ("best", "suboptimal", "n_tied", "flags"))
        n = rd.lens.size
        for i in range(n):
            m = min(int(want.results["n_tied"][i]), got.cap)
            same = same and np.array_equal(got.ties[i, :m], want.ties[i, :m])
        ok += int(same)
    for g in list(alone.values()) + scorers:
        g.close()
    best = max(per_rate, key=lambda x: x["gcups"])
    peak = int_peak(local_rank)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(panels["B"], pools["B"], scoring, "local", a.cpu_seconds)
        cpu.pop("seconds", None)
        cpu.pop("reads_per_s", None)
        cpu.pop("_results", None)
        cpu["sample"] = "panel B (2000 x 300 nt) reads: " + cpu["sample"]
    if rank == 0:
        line = common_line(
            a, ctx, best["gcups"], 1e3 * best["seconds"],
            "C5: serving, Poisson arrivals at " + a.rates + " req/s, requests of log-uniform "
            "1-50 000 C2-length reads for panel A (164 x 70-180 nt) or B (2000 x 300 nt), "
            "local or semi-global 2,-1,-10,-1, forward or both strands, through esg_server",
            {"requests_per_rate": a.requests, "panels": {k: len(v) for k, v in panels.items()},
             "max_batch_cells": a.max_batch_cells or "server default (1.5e11)"},
            {"value": best["gcups"], "unit": "GCUPS", "h2d_bytes_per_step": best["h2d_bytes"],
             "d2h_bytes_per_step": best["d2h_bytes"],
             "note": "serving is end to end: host requests in, results out"},
            roofline_of(peak, best["gcups"] * 1e9, "local", None), clocks,
            int(st["kernels"]))
        line["value_note"] = ("aggregate GCUPS at the busiest rate (all requests, wall clock); "
                              "gpu_launches = kernels of every batch of the sweep")
        line["latency_by_rate"] = per_rate
        line["server_stats"] = st
        line["bit_exact_alone_vs_mix"] = f"{ok} of {len(verify)} sampled requests equal"
        line["autotune_split"] = tunes
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)


def main():
    a = args_parse()
    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    if a.impl == "reference":
        run_reference(a, rank, world)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    ctx = Ctx(torch, dist, dev, local_rank, world)
    {"c1": run_c1, "c2": run_c2, "c3": run_c3, "c4": run_c4,
     "c5": run_c5}[a.workload](a, ctx, rank)
    if world > 1:
        dist.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


if __name__ == "__main__":
    main()
