#!/usr/bin/env python
"""Benchmark of the panel-scoring hot path (one JSON line on rank 0).

Workload (BASELINE config "plain vs batched scale-up"): 1 000 000 synthetic
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
            batch fed in chunks through prepare / submit / finish,
            double-buffered like eschalign's GPU feeder thread
            (crates/eschalign-cli/src/align.rs:2801-2917), host<->device
            copies inside the timed region.
* roofline  integer ALU: the batched kernel's algorithmic work (12 int ops a
            cell local, 11 semi-global, two cells per 32-bit lane op) against
            the integer lane-op peak measured by csrc/esg_probe.cu in the same
            run.
* --impl reference  the reference's CPU path (AVX-512BW score kernels +
            selection, restated in oracle/) on all host cores.
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
# DRAM bytes per DP cell of the batched kernel: 3.22 MB over 9.71e10 cells in
# the ncu capture of a 20 000-read C2 launch (profiles/k2_batched_c2.md);
# traffic grows with the reads, so it scales by cells to the full launch.
K2_DRAM_BYTES_PER_CELL = 3.22e6 / 9.7056e10


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
    ap.add_argument("--mode", default="local", choices=["local", "semiglobal"])
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


def cpu_baseline(refs, reads, scoring, mode, seconds, threads=0):
    """The reference's CPU path (AVX-512BW kernels + selection, restated in
    oracle/) on a bounded sample of the workload, all host threads."""
    from oracle import oracle as O
    O.build()
    prof = O.Profile(refs, scoring)
    panel_bases = sum(len(r) for r in refs)
    local = mode == "local"
    n_cal = min(len(reads), 2000)
    cal = reads.subset(np.arange(n_cal))
    t = time.perf_counter()
    _, _, _, used = prof.map_batch(*cal.tuple(), local=local, both_strands=True, threads=threads)
    dt = time.perf_counter() - t
    n = int(min(len(reads), max(n_cal, n_cal * seconds / max(dt, 1e-3))))
    sample = reads.subset(np.arange(n))
    t = time.perf_counter()
    _, _, _, used = prof.map_batch(*sample.tuple(), local=local, both_strands=True,
                                   threads=threads)
    dt = time.perf_counter() - t
    cells = 2 * sample.bases() * panel_bases
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": int(used), "kind": "port",
            "sample": f"first {n} of {len(reads)} reads, both strands, {mode} "
                      f"{','.join(map(str, scoring))}; {dt:.1f} s; reads/s {n / dt:.0f}",
            "reads_per_s": n / dt, "seconds": dt}


def run_reference(a, rank, world):
    """--impl reference: rank 0 times the CPU path; other ranks exit."""
    if rank != 0:
        return
    from eschalign_b200 import synth
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=a.reads)
    scoring, mode = HEADLINE
    per_step = max(2.0, min(a.cpu_seconds, 120.0 / max(1, a.steps + a.warmup)))
    for _ in range(a.warmup):
        cpu_baseline(refs, reads.subset(np.arange(2000)), scoring, mode, 0.5)
    vals, last = [], None
    for _ in range(a.steps):
        last = cpu_baseline(refs, reads, scoring, mode, per_step)
        vals.append(last["value"])
    v = statistics.median(vals)
    cells_per_read = 2 * (reads.bases() / len(reads)) * sum(len(r) for r in refs)
    line = {
        "impl": "reference", "metric": "GCUPS", "value": v, "unit": "GCUPS", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * last["seconds"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16",
        "data": "synthetic", "reads_per_s": v * 1e9 / cells_per_read,
        "config": {"workload": "C2 1M reads x 164-ref panel, both strands, local 2,-1,-10,-1",
                   "reads": a.reads, "refs": len(refs)},
        "cpu_baseline": {**last, "value": v},
        "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
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

    from eschalign_b200 import GpuScorer, Mode, Scoring, synth
    from eschalign_b200 import KERNEL_PLAIN32, KERNEL_AUTO

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    refs = synth.panel_tiles()
    panel_bases = sum(len(r) for r in refs)
    if a.profile_case:
        reads = synth.reads_c2(refs, n=a.profile_case)
        for kernel in (KERNEL_AUTO, KERNEL_PLAIN32):
            g = GpuScorer(refs, Scoring(*HEADLINE[0]), Mode.parse(a.mode), device=local_rank,
                          kernel=kernel)
            r = g.score_batch(reads.tuple(), both_strands=True)
            print(json.dumps({"profile_case": a.profile_case, "kernel": kernel,
                              "stats": r.stats}), flush=True)
            g.close()
        return
    reads = synth.reads_c2(refs, n=a.reads)  # weak scaling: every rank scores the full batch
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > L2 (126 MB)

    def device_time(scorer, batch, steps, warmup, sampler=None):
        for _ in range(warmup):
            scorer.relaunch(batch, stream.cuda_stream)
        torch.cuda.synchronize()
        barrier()
        total = 0.0
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            for k in range(steps):
                with torch.cuda.stream(stream):
                    flush.fill_(k & 0xFF)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                scorer.relaunch(batch, stream.cuda_stream)
                e1.record(stream)
                e1.synchronize()
                total += e0.elapsed_time(e1) / 1e3
        torch.cuda.synchronize()
        barrier()
        return total

    results = {}
    extras = {}
    # ---- headline: batched kernel, local 2,-1,-10,-1, inputs resident
    scoring, mode = HEADLINE
    g = GpuScorer(refs, Scoring(*scoring), Mode.parse(mode), device=local_rank,
                  stream=stream.cuda_stream)
    tune = g.autotune()  # tile shape for this panel, before any timing
    info = g.info()
    batch = g.submit(g.prepare(reads.tuple(), both_strands=True))
    first = g.finish(batch, keep=True)
    st = first.stats
    cells = st["cells"]
    launches_per_step = st["kernels"]
    sampler = ClockSampler(local_rank)
    t = device_time(g, batch, a.steps, a.warmup, sampler)
    clocks = sampler.summary()
    t_max = max_over_ranks(t)
    value = world * cells * a.steps / t_max / 1e9
    ms_per_step = 1e3 * t_max / a.steps
    reads_per_s = world * len(reads) * a.steps / t_max
    results["headline"] = value

    # ---- roofline of the batched kernel (integer ALU)
    peak = int_peak(local_rank)
    per_gpu_cells_s = cells * a.steps / t
    achieved = per_gpu_cells_s * OPS_PER_CELL[mode] / 2.0
    roofline = {"bound": "int_alu", "achieved": achieved / 1e12,
                "peak": (peak["peak_lane_ops_per_s"] / 1e12) if peak else None,
                "unit": "T lane-ops/s",
                "frac": (achieved / peak["peak_lane_ops_per_s"]) if peak else None,
                "traffic": (K2_DRAM_BYTES_PER_CELL * cells if K2_DRAM_BYTES_PER_CELL else None),
                "kernel": "k2_batched",
                "note": "achieved = cells/s x 12 int ops (11 semi-global) / 2 cells per "
                        "int16x2 lane-op; peak = measured iadd32/imax32 lane-op rate "
                        "(csrc/esg_probe.cu), measured in this run"}
    if peak:
        extras["int_probe"] = {k: round(v["lane_ops_per_s"] / 1e12, 3)
                               for k, v in peak["ops"].items()}
        extras["int_probe_per_sm_clk"] = {k: round(v["per_sm_per_clk"], 2)
                                          for k, v in peak["ops"].items()}
    batch.free()

    # ---- the other (mode, scheme) combinations, one timed step each
    if not a.no_extras:
        combos = {}
        for sc_, md in COMBOS[1:]:
            g2 = GpuScorer(refs, Scoring(*sc_), Mode.parse(md), device=local_rank,
                           stream=stream.cuda_stream)
            g2.autotune()
            b2 = g2.submit(g2.prepare(reads.tuple(), both_strands=True))
            r2 = g2.finish(b2, keep=True)
            t2 = max_over_ranks(device_time(g2, b2, 1, 1))
            combos[f"{md} {','.join(map(str, sc_))}"] = round(world * r2.stats["cells"] / t2 / 1e9, 1)
            b2.free()
            g2.close()
        combos[f"{mode} {','.join(map(str, scoring))}"] = round(value, 1)
        extras["gcups_by_combo"] = combos

        # ---- plain one-thread-per-pair kernel on a sample of the same batch
        sub = reads.subset(np.arange(min(a.plain_reads, len(reads))))
        g.set_kernel(KERNEL_PLAIN32)
        bp = g.submit(g.prepare(sub.tuple(), both_strands=True))
        rp = g.finish(bp, keep=True)
        tp = max_over_ranks(device_time(g, bp, 1, 1))
        plain = world * rp.stats["cells"] / tp / 1e9
        bp.free()
        g.set_kernel(KERNEL_AUTO)
        extras["plain_gcups"] = plain
        extras["batched_over_plain"] = value / plain
        extras["plain_sample"] = f"first {len(sub)} reads, both strands"

    # ---- e2e through the public API with host buffers (double-buffered feeder)
    chunks = [reads.subset(np.arange(k, min(k + a.chunk, len(reads))))
              for k in range(0, len(reads), a.chunk)]
    e2e_steps = max(1, min(2, a.steps))
    h2d = d2h = 0
    e2e_times = []
    for it in range(e2e_steps + 1):
        barrier()
        t0 = time.perf_counter()
        pending = None
        h2d = d2h = 0
        for c in chunks + [None]:
            prepared = g.prepare(c.tuple(), both_strands=True) if c is not None else None
            if pending is not None:
                out = g.finish(pending)
                h2d += out.stats["h2d_bytes"]
                d2h += out.stats["d2h_bytes"]
            pending = g.submit(prepared) if prepared is not None else None
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if it > 0:  # the first pass is a warm-up (pinned pool, allocator)
            e2e_times.append(dt)
    te = max_over_ranks(sum(e2e_times))
    e2e = {"value": world * cells * len(e2e_times) / te / 1e9, "unit": "GCUPS",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "reads_per_s": world * len(reads) * len(e2e_times) / te,
           "chunk_reads": a.chunk}
    g.close()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(refs, reads, scoring, mode, a.cpu_seconds)
        extras["cpu_reads_per_s"] = cpu.pop("reads_per_s")
        cpu.pop("seconds", None)

    if rank == 0:
        line = {
            "metric": "GCUPS", "value": value, "unit": "GCUPS", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16x2",
            "data": "synthetic",
            "config": {"workload": "C2: 1M reads (lognormal median 110 nt) x 164-ref panel "
                                   "(70-180 nt), both strands, local 2,-1,-10,-1, best + XS + "
                                   "8 ties per read",
                       "reads": a.reads, "refs": len(refs), "panel_bases": panel_bases,
                       "cells_per_step": cells, "parallelism": f"replicas x{world}",
                       "l2": "flushed (256 MB write) between timed steps"},
            "reads_per_s": reads_per_s,
            "e2e": e2e,
            "roofline": roofline,
            "clocks": clocks,
            "gpu_launches": launches_per_step * a.steps,
            "kernel_info": {k: info[k] for k in ("regs_batched", "regs_plain",
                                                 "local_bytes_batched", "batched_blocks",
                                                 "panel_bytes", "sm_count", "split_len")},
            "autotune": tune,
            "batch_stats": {k: st[k] for k in ("queries_batched", "queries_plain",
                                               "queries_rescored", "tasks", "lanes_used")},
        }
        if cpu:
            line["cpu_baseline"] = cpu
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


if __name__ == "__main__":
    main()
