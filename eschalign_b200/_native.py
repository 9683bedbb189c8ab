"""Build and load the native scorer library (``libeschalign_b200.so``).

The library is compiled ahead of time for sm_100a with nvcc (no JIT, no
NVRTC) from ``csrc/esg_api.cu`` and lives next to this file.  Loading fails
loudly when it is missing: there is no CPU path behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_NAME = "libeschalign_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)
PROBE_PATH = os.path.join(HERE, "libesg_probe.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build eschalign_b200")


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".h"))] + [os.path.join(INCLUDE, "eschalign_b200.h")]


def _compile(src, out: str, verbose: bool) -> None:
    srcs = [src] if isinstance(src, str) else list(src)
    cmd = [nvcc(), *ARCH_FLAGS, *NVCC_FLAGS, *(os.path.join(CSRC, f) for f in srcs), "-o",
           out + ".tmp"]
    if "esg_bam.cu" in srcs:
        cmd.append("-lz")
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile csrc/esg_api.cu into libeschalign_b200.so and the integer-pipe
    probe csrc/esg_probe.cu into libesg_probe.so (sm_100a, ahead of time)."""
    newest = max(os.path.getmtime(s) for s in sources())
    for src, out in ((("esg_api.cu", "esg_server.cu", "esg_trace.cu", "esg_map.cu",
                        "esg_bam.cu", "esg_noalloc.cu"), LIB_PATH),
                     ("esg_probe.cu", PROBE_PATH)):
        if force or not os.path.exists(out) or os.path.getmtime(out) < newest:
            _compile(src, out, verbose)
    return LIB_PATH


def load_probe():
    """The integer-pipe peak probe (measurement only, not part of the ABI)."""
    if not os.path.exists(PROBE_PATH):
        build()
    lib = C.CDLL(PROBE_PATH)
    lib.esg_probe_int_peak.restype = C.c_int
    lib.esg_probe_int_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int)]
    lib.esg_probe_op_name.restype = C.c_char_p
    lib.esg_probe_op_name.argtypes = [C.c_int]
    return lib


# ------------------------------------------------------------------ ABI types
class EsgScoring(C.Structure):
    _fields_ = [("match_score", C.c_int32), ("mismatch", C.c_int32),
                ("gap_open", C.c_int32), ("gap_extend", C.c_int32)]


class EsgOptions(C.Structure):
    _fields_ = [("tie_capacity", C.c_uint32), ("kernel", C.c_int32), ("stream", C.c_void_p)]


class EsgInfo(C.Structure):
    _fields_ = [("device_name", C.c_char * 256), ("device", C.c_int32), ("sm_count", C.c_int32),
                ("n_refs", C.c_uint32), ("max_ref_len", C.c_uint32),
                ("n_ref_pairs", C.c_uint32), ("panel_bytes", C.c_uint32),
                ("batched_ok", C.c_int32), ("regs_batched", C.c_int32),
                ("regs_plain", C.c_int32), ("local_bytes_batched", C.c_int32),
                ("local_bytes_plain", C.c_int32), ("batched_blocks", C.c_int32),
                ("batched_threads", C.c_int32), ("plain_blocks", C.c_int32),
                ("plain_threads", C.c_int32), ("split_len", C.c_uint32), ("tuned", C.c_int32)]


class EsgTuneReport(C.Structure):
    _fields_ = [("n_lengths", C.c_uint32), ("lengths", C.c_uint32 * 8),
                ("ms_rows16", C.c_float * 8), ("ms_rows32", C.c_float * 8),
                ("split_len", C.c_uint32), ("ms_int32", C.c_float * 8),
                ("int32_from", C.c_uint32),
                ("n_ctas16", C.c_uint32), ("cand_ctas16", C.c_uint32 * 4),
                ("ms_ctas16", C.c_float * 4), ("ctas16", C.c_uint32),
                ("n_ctas32", C.c_uint32), ("cand_ctas32", C.c_uint32 * 4),
                ("ms_ctas32", C.c_float * 4), ("ctas32", C.c_uint32),
                ("n_chunk_targets", C.c_uint32), ("chunk_targets", C.c_uint32 * 8),
                ("ms_chunks", C.c_float * 8), ("chunk_target", C.c_uint32),
                ("n_splits", C.c_uint32), ("splits", C.c_uint32 * 8),
                ("ms_splits", C.c_float * 8)]


class EsgBatchStats(C.Structure):
    _fields_ = [("n_reads", C.c_uint32), ("n_queries", C.c_uint32), ("n_empty", C.c_uint32),
                ("queries_batched", C.c_uint32), ("queries_plain", C.c_uint32),
                ("queries_rescored", C.c_uint32), ("tasks", C.c_uint32),
                ("lanes_used", C.c_uint32), ("kernels", C.c_uint32), ("cells", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("n_pairs", C.c_uint32),
                ("mates_trimmed", C.c_uint32), ("bases_trimmed", C.c_uint64),
                ("panel_chunks", C.c_uint32), ("reserved", C.c_uint32),
                ("device_bytes", C.c_uint64)]


class EsgAdapterConfig(C.Structure):
    _fields_ = [("r1", C.c_void_p), ("r1_len", C.c_uint32), ("r2", C.c_void_p),
                ("r2_len", C.c_uint32), ("min_overlap", C.c_uint32),
                ("max_read_len", C.c_uint32)]


class EsgAlignJob(C.Structure):
    _fields_ = [("read", C.c_uint32), ("ref", C.c_uint32), ("reverse", C.c_uint32)]


class EsgAlignment(C.Structure):
    _fields_ = [("score", C.c_int32), ("query_start", C.c_uint32), ("query_end", C.c_uint32),
                ("ref_start", C.c_uint32), ("ref_end", C.c_uint32), ("n_ops", C.c_uint32),
                ("ops_offset", C.c_uint64)]


class EsgMapOptions(C.Structure):
    _fields_ = [("min_score", C.c_int32), ("max_ties", C.c_uint32),
                ("both_strands", C.c_uint32), ("reserved", C.c_uint32)]


class EsgPairMapOptions(C.Structure):
    _fields_ = [("min_score", C.c_int32), ("max_ties", C.c_uint32),
                ("max_insert", C.c_uint32), ("both_strands", C.c_uint32)]


class EsgBamOptions(C.Structure):
    _fields_ = [("secondary", C.c_uint32), ("reserved", C.c_uint32)]


class EsgServerOptions(C.Structure):
    _fields_ = [("max_batch_reads", C.c_uint32), ("max_inflight", C.c_uint32),
                ("memory_budget", C.c_uint64), ("memory_headroom", C.c_uint64),
                ("max_batch_cells", C.c_uint64)]


class EsgRequestTiming(C.Structure):
    _fields_ = [("queued_ms", C.c_double), ("total_ms", C.c_double),
                ("batch_reads", C.c_uint32), ("batch_requests", C.c_uint32)]


class EsgServerStats(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("completed", C.c_uint64), ("refused", C.c_uint64),
                ("batches", C.c_uint64), ("cells", C.c_uint64), ("bytes_in_flight", C.c_uint64),
                ("peak_bytes_in_flight", C.c_uint64), ("admission_waits", C.c_uint32),
                ("kernels", C.c_uint32)]


# every entry point include/eschalign_b200.h declares: name -> (restype, argtypes)
_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i32p = C.POINTER(C.c_int32)
SIGNATURES = {
    "esg_abi_version": (C.c_int, []),
    "esg_status_string": (C.c_char_p, [C.c_int32]),
    "esg_last_error": (C.c_char_p, []),
    "esg_device_count": (C.c_int32, [_i32p]),
    "esg_fits_i16": (C.c_int32, [C.c_uint64, C.c_uint64, C.POINTER(EsgScoring)]),
    "esg_scorer_new": (C.c_int32, [C.c_int32, _u8p, _u64p, _u32p, C.c_uint32,
                                   C.POINTER(EsgScoring), C.c_int32, C.POINTER(EsgOptions),
                                   C.POINTER(C.c_void_p)]),
    "esg_scorer_free": (None, [C.c_void_p]),
    "esg_scorer_info": (C.c_int32, [C.c_void_p, C.POINTER(EsgInfo)]),
    "esg_scorer_set_kernel": (C.c_int32, [C.c_void_p, C.c_int32]),
    "esg_scores_len": (C.c_int32, [C.c_void_p, C.c_uint64]),
    "esg_batched_takes": (C.c_int32, [C.c_void_p, C.c_uint64]),
    "esg_scorer_autotune": (C.c_int32, [C.c_void_p, C.POINTER(EsgTuneReport)]),
    "esg_scorer_autotune_lengths": (C.c_int32, [C.c_void_p, _u32p, C.c_uint32,
                                                C.POINTER(EsgTuneReport)]),
    "esg_scorer_set_split": (C.c_int32, [C.c_void_p, C.c_uint32]),
    "esg_scorer_set_chunking": (C.c_int32, [C.c_void_p, C.c_uint32]),
    "esg_score_batch": (C.c_int32, [C.c_void_p, _u8p, _u64p, _u32p, C.c_uint32, C.c_uint32,
                                    C.c_void_p, _u32p, _i32p]),
    "esg_prepare": (C.c_int32, [C.c_void_p, _u8p, _u64p, _u32p, C.c_uint32, C.c_uint32,
                                C.POINTER(C.c_void_p)]),
    "esg_submit": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "esg_finish": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, _u32p, _i32p]),
    "esg_batch_free": (None, [C.c_void_p]),
    "esg_batch_stats_get": (C.c_int32, [C.c_void_p, C.POINTER(EsgBatchStats)]),
    "esg_relaunch": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "esg_scorer_set_graphs": (C.c_int32, [C.c_void_p, C.c_int32]),
    "esg_batch_read_results": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, _u32p]),
    "esg_pair_adapters": (C.c_int32, [_u8p, _u64p, _u32p, C.c_uint32,
                                      C.POINTER(EsgAdapterConfig), _u32p, _u32p]),
    "esg_prepare_pairs": (C.c_int32, [C.c_void_p, _u8p, _u64p, _u32p, C.c_uint32,
                                      C.POINTER(EsgAdapterConfig), C.c_int32, C.c_uint32,
                                      C.POINTER(C.c_void_p)]),
    "esg_finish_pairs": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, _u32p, C.c_void_p,
                                     _u32p, _u32p, _i32p]),
    "esg_score_pairs": (C.c_int32, [C.c_void_p, _u8p, _u64p, _u32p, C.c_uint32,
                                    C.POINTER(EsgAdapterConfig), C.c_int32, C.c_uint32,
                                    C.c_void_p, _u32p, C.c_void_p, _u32p, _u32p, _i32p]),
    "esg_merge_read_results": (C.c_int32, [C.c_void_p, _u32p, C.c_void_p, _u32p, C.c_uint32,
                                           C.c_uint32, C.c_void_p, _u32p]),
    "esg_align_batch": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                    _u32p, C.c_uint64, _u64p]),
    "esg_align_reads": (C.c_int32, [C.c_void_p, _u8p, _u64p, _u32p, C.c_uint32, C.c_void_p,
                                    C.c_uint32, C.c_void_p, _u32p, C.c_uint64, _u64p]),
    "esg_map_reads": (C.c_int32, [C.c_void_p, _u8p, _u64p, _u32p, C.c_uint32,
                                  C.POINTER(EsgMapOptions), _u8p, _u64p, C.POINTER(C.c_void_p)]),
    "esg_map_pairs": (C.c_int32, [C.c_void_p, _u8p, _u64p, _u32p, C.c_uint32,
                                  C.POINTER(EsgPairMapOptions), _u8p, _u64p,
                                  C.POINTER(C.c_void_p)]),
    "esg_mapping_pairs": (C.c_void_p, [C.c_void_p, _u32p]),
    "esg_mapping_pair_hits": (C.c_void_p, [C.c_void_p, _u64p]),
    "esg_mapping_reads": (C.c_void_p, [C.c_void_p, _u32p]),
    "esg_mapping_hits": (C.c_void_p, [C.c_void_p, _u64p]),
    "esg_mapping_ops": (C.c_void_p, [C.c_void_p, _u64p]),
    "esg_mapping_md": (C.c_void_p, [C.c_void_p, _u64p]),
    "esg_mapping_free": (None, [C.c_void_p]),
    "esg_mapping_from_arrays": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, _u32p,
                                            C.c_uint64, C.c_char_p, C.c_uint64,
                                            C.POINTER(C.c_void_p)]),
    "esg_mapping_set_pairs": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                          C.c_uint64]),
    "esg_server_new": (C.c_int32, [C.POINTER(EsgServerOptions), C.POINTER(C.c_void_p)]),
    "esg_server_add_scorer": (C.c_int32, [C.c_void_p, C.c_void_p, _u32p]),
    "esg_server_submit": (C.c_int32, [C.c_void_p, C.c_uint32, _u8p, _u64p, _u32p, C.c_uint32,
                                      C.c_uint32, _u64p]),
    "esg_server_wait": (C.c_int32, [C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, _u32p,
                                    C.POINTER(EsgRequestTiming)]),
    "esg_server_stats_get": (C.c_int32, [C.c_void_p, C.POINTER(EsgServerStats)]),
    "esg_server_free": (None, [C.c_void_p]),
    "esg_bam_open": (C.c_int32, [C.c_char_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "esg_bam_header_text": (C.c_void_p, [C.c_void_p, _u64p]),
    "esg_bam_read_batch": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    "esg_bam_open_pairs": (C.c_int32, [C.c_char_p, C.c_char_p, C.c_uint32,
                                       C.POINTER(C.c_void_p)]),
    "esg_bam_read_pair_batch": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "esg_bam_set_read_ids": (C.c_int32, [C.c_void_p, C.c_char_p]),
    "esg_bam_reader_counts": (C.c_int32, [C.c_void_p, _u64p, _u64p]),
    "esg_bam_batch_reads": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p), _u32p]),
    "esg_bam_batch_free": (None, [C.c_void_p]),
    "esg_bam_close": (None, [C.c_void_p]),
    "esg_bam_encode": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(EsgBamOptions),
                                   C.POINTER(C.c_char_p), C.c_uint32, C.c_uint32,
                                   C.POINTER(C.c_void_p)]),
    "esg_bam_encode_pairs": (C.c_int32, [C.c_void_p, C.c_void_p, _u32p, C.POINTER(EsgBamOptions),
                                         C.POINTER(C.c_char_p), C.c_uint32, C.c_uint32,
                                         C.POINTER(C.c_void_p)]),
    "esg_bam_records_bytes": (C.c_void_p, [C.c_void_p, _u64p, _u32p]),
    "esg_bam_records_outcomes": (C.c_int32, [C.c_void_p, _u64p, _u64p, _u64p]),
    "esg_bam_records_free": (None, [C.c_void_p]),
    "esg_bam_writer_open": (C.c_int32, [C.c_char_p, C.c_char_p, C.POINTER(C.c_char_p), _u32p,
                                        C.c_uint32, C.c_int32, C.c_uint32,
                                        C.POINTER(C.c_void_p)]),
    "esg_bam_writer_push": (C.c_int32, [C.c_void_p, C.c_uint64, C.c_void_p]),
    "esg_bam_writer_close": (C.c_int32, [C.c_void_p]),
    "esg_bam_writer_use_device": (C.c_int32, [C.c_void_p, C.c_int32]),
    "esg_bam_writer_blocks": (C.c_int32, [C.c_void_p, _u64p, _u64p]),
    "esg_bgzf_deflate_host": (C.c_uint32, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "esg_bgzf_code_lengths": (C.c_int32, [_u32p, C.c_uint32, C.c_uint32, C.c_void_p]),
    "esg_score_rows_noalloc": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_uint32, C.POINTER(EsgScoring), C.c_int32,
                                           C.c_void_p, C.c_void_p]),
}

_lib = None


def load(path: str | None = None):
    """Load the library (building it first if only the sources are here)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        if os.path.isdir(CSRC) and (shutil.which("nvcc") or os.path.exists("/usr/local/cuda/bin/nvcc")):
            build()
        else:
            raise ImportError(f"{LIB_NAME} is not built ({path}); run eschalign_b200.build()")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.esg_abi_version() != 1:
        raise ImportError("libeschalign_b200.so ABI version mismatch")
    _lib = lib
    return lib
