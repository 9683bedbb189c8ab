"""ctypes view of the CPU checker (oracle/_build/libesg_oracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference legs, never by the product package.

* :func:`score` -- scalar Gotoh, crates/eschalign/src/scalar.rs:120-163;
* :func:`select` -- tie set / XS, crates/eschalign/src/mapper.rs:444-472;
* :class:`Profile` -- the AVX-512BW inter-sequence kernels,
  crates/eschalign/src/simd/avx512.rs:43-107 and :278-354, with the
  reference's dispatch (mapper.rs:216-222);
* :func:`md_nm` -- MD / NM as samtools calmd writes them,
  crates/eschalign/src/sam.rs:55-121;
* :func:`map_reads` -- Aligner::map_reads_scored, mapper.rs:400-552.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libesg_oracle.so")

NO_SCORE = -(2**31)
RESULT_EMPTY = 1
RESULT_TIES_TRUNCATED = 2


class EoResult(C.Structure):
    _fields_ = [("best", C.c_int32), ("suboptimal", C.c_int32),
                ("n_tied", C.c_uint32), ("flags", C.c_uint32)]


RESULT_DTYPE = np.dtype([("best", "<i4"), ("suboptimal", "<i4"),
                         ("n_tied", "<u4"), ("flags", "<u4")])
PAIR_DTYPE = np.dtype([("best", "<i4"), ("next", "<i4"), ("n_tied", "<u4"), ("flags", "<u4"),
                       ("xs", "<i4", (2,)), ("primary", "<i4", (2,))])


def build() -> str:
    """Compile the checker with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def reference_root():
    """The reference checkout, where this machine has one: the directory
    named by ESCHALIGN_REFERENCE, else a `reference` directory beside this
    repository; None when neither exists (on a GPU box the built files
    travel instead)."""
    for cand in (os.environ.get("ESCHALIGN_REFERENCE"),
                 os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "crates", "eschalign")):
            return cand
    return None


REF_GPU_LIB = os.path.join(HERE, "_ref", "libref_gpu.so")
REF_GPU_CUBIN = os.path.join(HERE, "_ref", "ref_kernels.cubin")


def build_ref_gpu() -> bool:
    """Compile the reference's own GPU kernels (comparison arms) when its
    tree is present here; elsewhere whatever was built travels as files."""
    root = reference_root()
    if root is None:
        return os.path.exists(REF_GPU_LIB) and os.path.exists(REF_GPU_CUBIN)
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={root}"], check=True)
    return True


class RefGpu:
    """The reference's align_score_kernel (kernel 0, int) and
    align_score_kernel_h2 (kernel 1, half2), laid out and launched as
    crates/eschalign/src/cuda/mod.rs does (oracle/ref_gpu/ref_gpu.cu).
    Comparison arms only."""

    def __init__(self, refs, device=0):
        self._L = C.CDLL(REF_GPU_LIB)
        L = self._L
        L.rg_new.restype = C.c_int
        L.rg_new.argtypes = [C.c_int, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_uint32, C.POINTER(C.c_void_p)]
        L.rg_score.restype = C.c_int
        L.rg_score.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_uint32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                               C.c_int, C.c_void_p, C.POINTER(C.c_float)]
        L.rg_error.restype = C.c_char_p
        L.rg_error.argtypes = [C.c_void_p]
        L.rg_free.argtypes = [C.c_void_p]
        L.rg_geometry.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        self.n_refs = len(refs)
        c, o, l = pack(refs)
        self._h = C.c_void_p()
        rc = L.rg_new(device, REF_GPU_CUBIN.encode(), c.ctypes.data, o.ctypes.data, l.ctypes.data,
                      len(refs), C.byref(self._h))
        if rc:
            msg = L.rg_error(self._h).decode()
            L.rg_free(self._h)
            self._h = None
            raise RuntimeError(msg)

    def geometry(self, kernel):
        g = (C.c_int * 4)()
        self._L.rg_geometry(self._h, kernel, g)
        return tuple(g)

    def score(self, codes, off, lens, scoring, local, kernel=0, reps=1, rows=True):
        """(int16 rows [q, n_refs] or None, mean ms per launch)."""
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        lens = np.ascontiguousarray(lens, dtype=np.uint32)
        out = np.zeros((lens.size, self.n_refs), dtype=np.int16) if rows else None
        ms = C.c_float()
        rc = self._L.rg_score(self._h, kernel, codes.ctypes.data, off.ctypes.data,
                              lens.ctypes.data, lens.size, *scoring, int(bool(local)), reps,
                              out.ctypes.data if rows else None, C.byref(ms))
        if rc:
            raise RuntimeError(self._L.rg_error(self._h).decode())
        return out, ms.value

    def close(self):
        if self._h:
            self._L.rg_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u8p = C.POINTER(C.c_uint8)
        u32p = C.POINTER(C.c_uint32)
        u64p = C.POINTER(C.c_uint64)
        i32p = C.POINTER(C.c_int32)
        L.eo_encode_base.restype = C.c_uint8
        L.eo_encode_base.argtypes = [C.c_uint8]
        L.eo_score.restype = C.c_int32
        L.eo_score.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t] + [C.c_int32] * 4 + [C.c_int]
        L.eo_fits_i16.restype = C.c_int
        L.eo_fits_i16.argtypes = [C.c_size_t, C.c_size_t] + [C.c_int32] * 4
        L.eo_scoring_validate.restype = C.c_int
        L.eo_scoring_validate.argtypes = [C.c_int32] * 4
        L.eo_select.restype = None
        L.eo_select.argtypes = [i32p, i32p, C.c_uint32, C.c_uint32, C.POINTER(EoResult), u32p]
        L.eo_score_matrix.restype = None
        L.eo_score_matrix.argtypes = [u8p, u64p, u32p, C.c_uint32, u8p, u64p, u32p, C.c_uint32,
                                      C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                      C.c_int, i32p]
        L.eo_scalar_map_batch.restype = C.c_int
        L.eo_scalar_map_batch.argtypes = [u8p, u64p, u32p, C.c_uint32, u8p, u64p, u32p,
                                          C.c_uint32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                          C.c_int, C.c_int, C.c_int, C.c_uint32,
                                          C.c_void_p, u32p, i32p]
        L.eo_profile_build.restype = C.c_void_p
        L.eo_profile_build.argtypes = [u8p, u64p, u32p, C.c_uint32] + [C.c_int32] * 4
        L.eo_profile_free.restype = None
        L.eo_profile_free.argtypes = [C.c_void_p]
        L.eo_cpu_has_avx512bw.restype = C.c_int
        L.eo_profile_score_all.restype = None
        L.eo_profile_score_all.argtypes = [C.c_void_p, u8p, C.c_size_t, C.c_int, C.c_int, i32p]
        L.eo_adapter_find.restype = C.c_size_t
        L.eo_adapter_find.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, C.c_size_t]
        L.eo_adapter_detect_pair.restype = None
        L.eo_adapter_detect_pair.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, u8p, C.c_size_t,
                                             u8p, C.c_size_t, C.c_size_t,
                                             C.POINTER(C.c_size_t)]
        L.eo_pair_adapters.restype = None
        L.eo_pair_adapters.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, u8p, C.c_size_t,
                                       u8p, C.c_size_t, C.c_size_t, C.c_size_t,
                                       C.POINTER(C.c_size_t)]
        L.eo_pair_select.restype = None
        L.eo_pair_select.argtypes = [i32p, i32p, i32p, i32p, C.c_uint32, C.c_int, C.c_int32,
                                     C.c_uint32, C.c_void_p, u32p]
        L.eo_pairs_from_rows.restype = None
        L.eo_pairs_from_rows.argtypes = [i32p, u32p, C.c_uint32, C.c_uint32, C.c_int, C.c_int32,
                                         C.c_uint32, C.c_void_p, u32p]
        L.eo_scalar_map_pairs.restype = C.c_int
        L.eo_scalar_map_pairs.argtypes = [u8p, u64p, u32p, C.c_uint32, u8p, u64p, u32p,
                                          C.c_uint32, C.c_int32, C.c_int32, C.c_int32,
                                          C.c_int32, C.c_int, C.c_int, C.c_int32, C.c_int,
                                          C.c_uint32, C.c_void_p, u32p]
        L.eo_cpu_map_pairs.restype = C.c_int
        L.eo_cpu_map_pairs.argtypes = [C.c_void_p, u8p, u64p, u32p, C.c_uint32, u8p, C.c_size_t,
                                       u8p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_int, C.c_int,
                                       C.c_int32, C.c_int, C.c_uint32, C.c_void_p, u32p,
                                       C.c_void_p, u32p, u32p]
        L.eo_cpu_set_chunk.restype = None
        L.eo_cpu_set_chunk.argtypes = [C.c_int]
        L.eo_align.restype = C.c_int
        L.eo_align.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, C.c_int32, C.c_int32, C.c_int32,
                               C.c_int32, C.c_int, C.c_void_p, u32p, C.c_size_t]
        L.eo_align_batch.restype = C.c_int
        L.eo_align_batch.argtypes = [u8p, u64p, u32p, u8p, u64p, u32p, u32p, u32p, u8p, C.c_uint32,
                                     C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int, C.c_int,
                                     C.c_void_p, u32p, C.c_size_t]
        L.eo_md_nm.restype = C.c_long
        L.eo_md_nm.argtypes = [u8p, C.c_size_t, C.c_int, u8p, u8p, C.c_void_p, u32p, C.c_char_p,
                               C.c_size_t, u32p]
        L.eo_md_nm_batch.restype = C.c_int
        L.eo_md_nm_batch.argtypes = [u8p, u64p, u32p, u8p, u64p, u8p, u32p, u32p, u8p,
                                     C.c_void_p, u32p, C.c_size_t, C.c_uint32, C.c_int,
                                     C.c_void_p, C.c_size_t, u32p, u32p]
        L.eo_cpu_map_batch.restype = C.c_int
        L.eo_cpu_map_batch.argtypes = [C.c_void_p, u8p, u64p, u32p, C.c_uint32, C.c_int, C.c_int,
                                       C.c_int, C.c_uint32, C.c_void_p, u32p, i32p]
        _lib = L
    return _lib


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def encode(letters) -> np.ndarray:
    """alphabet.rs:29-50 via the C table."""
    if isinstance(letters, str):
        letters = letters.encode()
    L = lib()
    return np.array([L.eo_encode_base(b) for b in letters], dtype=np.uint8)


def revcomp(codes: np.ndarray) -> np.ndarray:
    """alphabet.rs:58-64."""
    c = np.asarray(codes, dtype=np.uint8)[::-1]
    return np.where(c == 4, 4, 3 - c).astype(np.uint8)


ALIGN_DTYPE = np.dtype([("score", "<i4"), ("query_start", "<u4"), ("query_end", "<u4"),
                        ("ref_start", "<u4"), ("ref_end", "<u4"), ("n_ops", "<u4")])
CIGAR_OPS = "MID"


def align(q, r, scoring, local: bool):
    """scalar.rs:182-364: (record of ALIGN_DTYPE, ops as BAM CIGAR words)."""
    q = np.ascontiguousarray(q, dtype=np.uint8)
    r = np.ascontiguousarray(r, dtype=np.uint8)
    out = np.zeros(1, dtype=ALIGN_DTYPE)
    ops = np.zeros(q.size + r.size + 1, dtype=np.uint32)
    rc = lib().eo_align(_p(q, C.c_uint8), q.size, _p(r, C.c_uint8), r.size, *scoring,
                        int(bool(local)), out.ctypes.data, _p(ops, C.c_uint32), ops.size)
    if rc:
        raise RuntimeError(f"eo_align failed ({rc})")
    return out[0], ops[:int(out[0]["n_ops"])]


def align_batch(codes, off, lens, refs, jobs, scoring, local, threads=0):
    """eo_align_batch: (records, ops [n_jobs, stride], threads used)."""
    rc_, ro, rl = pack(refs)
    jobs = np.asarray(jobs, dtype=np.uint32).reshape(-1, 3)
    jr = np.ascontiguousarray(jobs[:, 0])
    jf = np.ascontiguousarray(jobs[:, 1])
    jv = np.ascontiguousarray(jobs[:, 2].astype(np.uint8))
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    off = np.ascontiguousarray(off, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    stride = int(lens.max(initial=0)) + int(rl.max(initial=0)) + 1
    out = np.zeros(jobs.shape[0], dtype=ALIGN_DTYPE)
    ops = np.zeros((max(jobs.shape[0], 1), stride), dtype=np.uint32)
    used = lib().eo_align_batch(_p(codes, C.c_uint8), _p(off, C.c_uint64), _p(lens, C.c_uint32),
                                _p(rc_, C.c_uint8), _p(ro, C.c_uint64), _p(rl, C.c_uint32),
                                _p(jr, C.c_uint32), _p(jf, C.c_uint32), _p(jv, C.c_uint8),
                                jobs.shape[0], *scoring, int(bool(local)), threads,
                                out.ctypes.data, _p(ops, C.c_uint32), stride)
    if used < 0:
        raise RuntimeError("eo_align_batch: ops stride too small")
    return out, ops, used


def cigar_string(ops) -> str:
    return "".join(f"{int(w) >> 4}{CIGAR_OPS[int(w) & 0xf]}" for w in ops)


def rescore(q, r, a, ops, scoring) -> int:
    """Alignment::rescore (scalar.rs:90-117): the ops scored on their own."""
    ma, mi, o, e = scoring
    i, j, total = int(a["query_start"]), int(a["ref_start"]), 0
    for w in ops:
        op, n = int(w) & 0xf, int(w) >> 4
        if op == 0:
            for _ in range(n):
                x, y = int(q[i]), int(r[j])
                total += ma if (x == y or x == 4 or y == 4) else mi
                i += 1
                j += 1
        else:
            total += o + (n - 1) * e
            if op == 1:
                i += n
            else:
                j += n
    return total


def score(q, r, scoring, local: bool) -> int:
    """scalar.rs:120-163."""
    q = np.ascontiguousarray(q, dtype=np.uint8)
    r = np.ascontiguousarray(r, dtype=np.uint8)
    ma, mi, o, e = scoring
    return int(lib().eo_score(_p(q, C.c_uint8), q.size, _p(r, C.c_uint8), r.size,
                              ma, mi, o, e, int(bool(local))))


def fits_i16(n, max_ref_len, scoring) -> bool:
    return bool(lib().eo_fits_i16(n, max_ref_len, *scoring))


def validate(scoring) -> int:
    return int(lib().eo_scoring_validate(*scoring))


def pack(seqs):
    """List of code arrays -> (codes, off u64, len u32)."""
    lens = np.array([len(s) for s in seqs], dtype=np.uint32)
    off = np.zeros(len(seqs), dtype=np.uint64)
    if len(seqs) > 1:
        off[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
    codes = (np.concatenate([np.asarray(s, dtype=np.uint8) for s in seqs])
             if len(seqs) and lens.sum() else np.zeros(1, dtype=np.uint8))
    return np.ascontiguousarray(codes), off, lens


def select(fwd, rev=None, cap=8):
    """mapper.rs:444-472 on one read's rows."""
    fwd = np.ascontiguousarray(fwd, dtype=np.int32)
    revp = None
    if rev is not None:
        rev = np.ascontiguousarray(rev, dtype=np.int32)
        revp = _p(rev, C.c_int32)
    res = EoResult()
    ties = np.zeros(max(cap, 1), dtype=np.uint32)
    lib().eo_select(_p(fwd, C.c_int32), revp, fwd.size, cap, C.byref(res), _p(ties, C.c_uint32))
    n = min(res.n_tied, cap)
    return (res.best, res.suboptimal, res.n_tied, res.flags, ties[:n].tolist())


def score_matrix(queries, refs, scoring, local, threads=0) -> np.ndarray:
    qc, qo, ql = pack(queries)
    rc, ro, rl = pack(refs)
    out = np.zeros((len(queries), len(refs)), dtype=np.int32)
    lib().eo_score_matrix(_p(qc, C.c_uint8), _p(qo, C.c_uint64), _p(ql, C.c_uint32), len(queries),
                          _p(rc, C.c_uint8), _p(ro, C.c_uint64), _p(rl, C.c_uint32), len(refs),
                          *scoring, int(bool(local)), threads, _p(out, C.c_int32))
    return out


def scalar_map_batch(reads, refs, scoring, local, both_strands, cap=8, threads=0, rows=False):
    """Scalar oracle end to end: per-read results, ties, optional rows."""
    qc, qo, ql = pack(reads)
    rc, ro, rl = pack(refs)
    n = len(reads)
    res = np.zeros(n, dtype=RESULT_DTYPE)
    ties = np.zeros((n, max(cap, 1)), dtype=np.uint32)
    out_rows = (np.zeros(((2 if both_strands else 1) * n, len(refs)), dtype=np.int32)
                if rows else None)
    lib().eo_scalar_map_batch(_p(qc, C.c_uint8), _p(qo, C.c_uint64), _p(ql, C.c_uint32), n,
                              _p(rc, C.c_uint8), _p(ro, C.c_uint64), _p(rl, C.c_uint32), len(refs),
                              *scoring, int(bool(both_strands)), int(bool(local)), threads, cap,
                              res.ctypes.data, _p(ties, C.c_uint32),
                              _p(out_rows, C.c_int32) if rows else None)
    return res, ties, out_rows


class Profile:
    """The AVX-512BW baseline over one panel (simd/mod.rs:292-331)."""

    def __init__(self, refs, scoring):
        L = lib()
        if not L.eo_cpu_has_avx512bw():
            raise RuntimeError("this CPU has no AVX-512BW")
        self.refs = [np.asarray(r, dtype=np.uint8) for r in refs]
        self._c, self._o, self._l = pack(self.refs)
        self.scoring = tuple(scoring)
        self.n_refs = len(refs)
        self._h = L.eo_profile_build(_p(self._c, C.c_uint8), _p(self._o, C.c_uint64),
                                     _p(self._l, C.c_uint32), len(refs), *scoring)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().eo_profile_free(h)
            self._h = None

    def score_all(self, q, local, kernel=0) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.uint8)
        out = np.zeros(self.n_refs, dtype=np.int32)
        lib().eo_profile_score_all(self._h, _p(q, C.c_uint8), q.size, int(bool(local)), kernel,
                                   _p(out, C.c_int32))
        return out

    def map_batch(self, codes, off, lens, local, both_strands, cap=8, threads=0, rows=False):
        """The CPU baseline end to end on packed reads; returns (results,
        ties, rows or None, threads used)."""
        n = int(lens.size)
        res = np.zeros(n, dtype=RESULT_DTYPE)
        ties = np.zeros((n, max(cap, 1)), dtype=np.uint32)
        out_rows = (np.zeros(((2 if both_strands else 1) * n, self.n_refs), dtype=np.int32)
                    if rows else None)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        lens = np.ascontiguousarray(lens, dtype=np.uint32)
        used = lib().eo_cpu_map_batch(self._h, _p(codes, C.c_uint8), _p(off, C.c_uint64),
                                      _p(lens, C.c_uint32), n, int(bool(both_strands)),
                                      int(bool(local)), threads, cap, res.ctypes.data,
                                      _p(ties, C.c_uint32),
                                      _p(out_rows, C.c_int32) if rows else None)
        return res, ties, out_rows, used

    def map_pairs(self, codes, off, lens, local, both_strands=True, min_score=0, cap=8,
                  threads=0, a1=None, a2=None, min_overlap=5, max_read_len=0):
        """The reference's CPU path for pairs (eo_cpu_map_pairs): returns
        (pair results, pair ties, mate results, mate ties, adapters, threads)."""
        n = int(lens.size) // 2
        x1 = _codes(TRUSEQ_R1 if a1 is None else a1)
        x2 = _codes(TRUSEQ_R2 if a2 is None else a2)
        res = np.zeros(n, dtype=PAIR_DTYPE)
        ties = np.zeros((n, max(cap, 1)), dtype=np.uint32)
        mres = np.zeros(2 * n, dtype=RESULT_DTYPE)
        mties = np.zeros((2 * n, max(cap, 1)), dtype=np.uint32)
        ads = np.zeros(2 * n, dtype=np.uint32)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        lens = np.ascontiguousarray(lens, dtype=np.uint32)
        used = lib().eo_cpu_map_pairs(self._h, _p(codes, C.c_uint8), _p(off, C.c_uint64),
                                      _p(lens, C.c_uint32), n, _p(x1, C.c_uint8), x1.size,
                                      _p(x2, C.c_uint8), x2.size, min_overlap, max_read_len,
                                      int(bool(both_strands)), int(bool(local)), min_score,
                                      threads, cap, res.ctypes.data, _p(ties, C.c_uint32),
                                      mres.ctypes.data, _p(mties, C.c_uint32),
                                      _p(ads, C.c_uint32))
        return res, ties, mres, mties, ads, used


TRUSEQ_R1 = b"AGATCGGAAGAGCACACGTCTGAACTCCAGTCA"  # adapter.rs:40
TRUSEQ_R2 = b"AGATCGGAAGAGCGTCGTGTAGGGAAAGAGTGT"  # adapter.rs:42


def _codes(x) -> np.ndarray:
    """Letters (bytes/str) or codes (uint8 array) -> contiguous codes."""
    if isinstance(x, np.ndarray):
        return np.ascontiguousarray(x, dtype=np.uint8)
    return np.ascontiguousarray(encode(x) if len(x) else np.zeros(0, np.uint8))


def adapter_find(read, adapter=TRUSEQ_R1, min_overlap=5) -> int:
    """adapter.rs:68-91 (letters or codes)."""
    q, a = _codes(read), _codes(adapter)
    return int(lib().eo_adapter_find(_p(q, C.c_uint8), q.size, _p(a, C.c_uint8), a.size,
                                     min_overlap))


def adapter_detect_pair(r1, r2, a1=TRUSEQ_R1, a2=TRUSEQ_R2, min_overlap=5):
    """adapter.rs:95-110 (letters or codes)."""
    q1, q2, x1, x2 = _codes(r1), _codes(r2), _codes(a1), _codes(a2)
    out = (C.c_size_t * 2)()
    lib().eo_adapter_detect_pair(_p(q1, C.c_uint8), q1.size, _p(q2, C.c_uint8), q2.size,
                                 _p(x1, C.c_uint8), x1.size, _p(x2, C.c_uint8), x2.size,
                                 min_overlap, out)
    return [int(out[0]), int(out[1])]


def pair_adapters(r1, r2, a1=TRUSEQ_R1, a2=TRUSEQ_R2, min_overlap=5, max_read_len=0):
    """crates/eschalign-cli/src/align.rs:934-949 (letters or codes)."""
    q1, q2, x1, x2 = _codes(r1), _codes(r2), _codes(a1), _codes(a2)
    out = (C.c_size_t * 2)()
    lib().eo_pair_adapters(_p(q1, C.c_uint8), q1.size, _p(q2, C.c_uint8), q2.size,
                           _p(x1, C.c_uint8), x1.size, _p(x2, C.c_uint8), x2.size,
                           min_overlap, max_read_len, out)
    return [int(out[0]), int(out[1])]


def trim_pairs(mates, a1=TRUSEQ_R1, a2=TRUSEQ_R2, min_overlap=5, max_read_len=0):
    """The aligned bases of each mate (align.rs:2844-2863): mate less its 3'
    adapter, empty when over max_read_len.  Returns (trimmed mates, adapters)."""
    out, ads = [], []
    for p in range(len(mates) // 2):
        m1, m2 = _codes(mates[2 * p]), _codes(mates[2 * p + 1])
        ad = pair_adapters(m1, m2, a1, a2, min_overlap, max_read_len)
        for m, a in ((m1, ad[0]), (m2, ad[1])):
            if max_read_len and m.size > max_read_len:
                out.append(np.zeros(0, np.uint8))
            else:
                out.append(m[:m.size - a])
        ads.extend(ad)
    return out, np.array(ads, dtype=np.uint32)


def pair_select(f0, r0, f1, r1, both_strands=True, min_score=0, cap=8):
    """pair.rs:195-234, :297-314 on one pair's four rows."""
    rows = [np.ascontiguousarray(x, dtype=np.int32) for x in (f0, r0, f1, r1)]
    res = np.zeros(1, dtype=PAIR_DTYPE)
    ties = np.zeros(max(cap, 1), dtype=np.uint32)
    lib().eo_pair_select(*[_p(x, C.c_int32) for x in rows], rows[0].size, int(bool(both_strands)),
                         min_score, cap, res.ctypes.data, _p(ties, C.c_uint32))
    return res[0], ties[:min(int(res[0]["n_tied"]), cap)].tolist()


def pairs_from_rows(rows, lens, n_refs, both_strands=True, min_score=0, cap=8):
    """The ranking over rows laid out as the CUDA path returns them
    (forward rows of the 2n mates, then reverse-complement rows)."""
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    n = lens.size // 2
    res = np.zeros(n, dtype=PAIR_DTYPE)
    ties = np.zeros((n, max(cap, 1)), dtype=np.uint32)
    lib().eo_pairs_from_rows(_p(rows, C.c_int32), _p(lens, C.c_uint32), n, n_refs,
                             int(bool(both_strands)), min_score, cap, res.ctypes.data,
                             _p(ties, C.c_uint32))
    return res, ties


def scalar_map_pairs(mates, refs, scoring, local, both_strands, min_score=0, cap=8, threads=0):
    """Pairs (mate codes, 2 per pair, trimmed) end to end with the scalar oracle."""
    qc, qo, ql = pack(mates)
    rc, ro, rl = pack(refs)
    n = len(mates) // 2
    res = np.zeros(n, dtype=PAIR_DTYPE)
    ties = np.zeros((n, max(cap, 1)), dtype=np.uint32)
    lib().eo_scalar_map_pairs(_p(qc, C.c_uint8), _p(qo, C.c_uint64), _p(ql, C.c_uint32), n,
                              _p(rc, C.c_uint8), _p(ro, C.c_uint64), _p(rl, C.c_uint32), len(refs),
                              *scoring, int(bool(both_strands)), int(bool(local)), min_score,
                              threads, cap, res.ctypes.data, _p(ties, C.c_uint32))
    return res, ties


# ------------------------------------------------------------------ mapping
def _norm(b: int) -> int:
    """sam.rs:55-61: upper case, U as T."""
    u = b - 32 if 97 <= b <= 122 else b
    return 84 if u == 85 else u


def calmd_match(read_base: int, ref_base: int) -> bool:
    """sam.rs:63-69."""
    q, r = _norm(read_base), _norm(ref_base)
    return q == r and r in (65, 67, 71, 84)


def md_nm(read: bytes, reference: bytes, query_start: int, ref_start: int, ops):
    """sam.rs:76-121 on letters; ops are BAM CIGAR words (len << 4 | op)."""
    md, nm, run = [], 0, 0
    i, j = query_start, ref_start
    for w in ops:
        op, n = int(w) & 0xf, int(w) >> 4
        if op == 0:
            for _ in range(n):
                if calmd_match(read[i], reference[j]):
                    run += 1
                else:
                    md.append(str(run))
                    md.append(chr(reference[j]).upper())
                    run = 0
                    nm += 1
                i += 1
                j += 1
        elif op == 1:
            i += n
            nm += n
        else:
            md.append(str(run))
            md.append("^")
            md.extend(chr(reference[j + k]).upper() for k in range(n))
            run = 0
            j += n
            nm += n
    md.append(str(run))
    return "".join(md), nm


def revcomp_letters(seq: bytes) -> bytes:
    """alphabet.rs:66-80: upper case, U to A, other letters N."""
    comp = {65: 84, 67: 71, 71: 67, 84: 65}
    return bytes(comp.get(_norm(b), 78) for b in reversed(seq))


def map_reads(reads, refs, scoring, local, min_score=0, max_ties=None, both_strands=False,
              threads=0):
    """Aligner::map_reads_scored (mapper.rs:400-552) with the scalar scores:
    `reads` and `refs` are letters (bytes/str).  Returns one dict per read:
    best_score, n_tied, suboptimal, hits [reference, reverse, score,
    coordinates, cigar, md, nm]."""
    reads = [r.encode() if isinstance(r, str) else bytes(r) for r in reads]
    refs = [r.encode() if isinstance(r, str) else bytes(r) for r in refs]
    rcodes = [encode(r) for r in refs]
    fwd = [encode(r) if len(r) else np.zeros(0, np.uint8) for r in reads]
    nonempty = [k for k in range(len(reads)) if len(reads[k])]
    qs = [fwd[k] for k in nonempty]
    if both_strands:
        qs += [revcomp(fwd[k]) for k in nonempty]
    m = score_matrix(qs, rcodes, scoring, local, threads) if qs else np.zeros((0, len(refs)))
    row_of = {k: i for i, k in enumerate(nonempty)}
    out = []
    for k, read in enumerate(reads):
        if not len(read):
            out.append({"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []})
            continue
        i = row_of[k]
        cands = []
        for r in range(len(refs)):
            cands.append((r, False, int(m[i, r])))
            if both_strands:
                cands.append((r, True, int(m[len(nonempty) + i, r])))
        best = max(s for _, _, s in cands)
        ties = [(r, rv) for r, rv, s in cands if s == best]
        others = [s for _, _, s in cands if s != best]
        sub = max(others) if others else None
        n_tied = len(ties)
        if best < min_score:
            take = []
        else:
            kk = n_tied if max_ties is None else min(n_tied, max_ties + 1)
            take = ties[:kk]
        rec = {"best_score": best, "n_tied": n_tied, "suboptimal": sub, "hits": []}
        traced = []
        for r, rv in take:
            q = revcomp(fwd[k]) if rv else fwd[k]
            a, ops = align(q, rcodes[r], scoring, local)
            traced.append((r, rv, a, ops))
        if not take or not any((int(w) & 0xf) == 0 for w in traced[0][3]):
            out.append(rec)
            continue
        letters_rev = revcomp_letters(read) if any(rv for _, rv in take) else b""
        for r, rv, a, ops in traced:
            md, nm = md_nm(letters_rev if rv else read, refs[r], int(a["query_start"]),
                           int(a["ref_start"]), ops)
            rec["hits"].append({"reference": r, "reverse": rv, "score": int(a["score"]),
                                "query_start": int(a["query_start"]),
                                "query_end": int(a["query_end"]),
                                "ref_start": int(a["ref_start"]), "ref_end": int(a["ref_end"]),
                                "cigar": cigar_string(ops), "md": md, "nm": nm})
        out.append(rec)
    return out


def _aligned_any(ops) -> bool:
    """Alignment::is_empty's negation (scalar.rs:80-85)."""
    return any((int(w) & 0xf) == 0 for w in ops)


def pair_ok(al, ops, template_reverse: bool, max_insert: int) -> bool:
    """Aligner::pair_ok (pair.rs:392-410): both mates aligned, no outie, the
    insert within max_insert."""
    if not _aligned_any(ops[0]) or not _aligned_any(ops[1]):
        return False
    fwd, rev = (al[1], al[0]) if template_reverse else (al[0], al[1])
    if int(fwd["ref_start"]) >= int(rev["ref_end"]):
        return False
    lo = min(int(al[0]["ref_start"]), int(al[1]["ref_start"]))
    hi = max(int(al[0]["ref_end"]), int(al[1]["ref_end"]))
    return hi - lo <= max_insert


def map_pairs(pairs, refs, scoring, local, min_score=0, max_ties=None, max_insert=500,
              both_strands=False, threads=0):
    """Aligner::map_pairs_scored (pair.rs:157-390) with the scalar scores:
    `pairs` is a list of (mate 1, mate 2) letters, `refs` letters.  One dict
    per pair: {"proper": True, score, n_tied, suboptimal [2], hits [{reference,
    reverse, insert, mates [hit, hit]}]} or {"proper": False, "mates": [two
    map_reads dicts]}."""
    refs = [r.encode() if isinstance(r, str) else bytes(r) for r in refs]
    pairs = [tuple(m.encode() if isinstance(m, str) else bytes(m) for m in p) for p in pairs]
    rcodes = [encode(r) for r in refs]
    n_refs = len(refs)
    strands = (False, True) if both_strands else (False,)
    mr = lambda m, t: t ^ (m == 1)  # noqa: E731  (PairState::mate_reverse)
    # all four mate rows of every pair with two non-empty mates
    live = [p for p, (a, b) in enumerate(pairs) if len(a) and len(b)]
    qs = []
    for p in live:
        for m in range(2):
            c = encode(pairs[p][m])
            qs += [c, revcomp(c)]
    mat = score_matrix(qs, rcodes, scoring, local, threads) if qs else None
    out = [None] * len(pairs)
    separate = []
    for i, p in enumerate(live):
        rows = [[mat[4 * i + 2 * m + rv] for rv in range(2)] for m in range(2)]
        codes = [[encode(pairs[p][m]), revcomp(encode(pairs[p][m]))] for m in range(2)]
        cands = []
        for t in strands:
            r0, r1 = rows[0][mr(0, t)], rows[1][mr(1, t)]
            for r in range(n_refs):
                a, b = int(r0[r]), int(r1[r])
                if a >= min_score and b >= min_score:
                    cands.append((a + b, r, t, a, b))
        cands.sort(key=lambda c: (-c[0], c[1], c[2]))
        found = []
        k = 0
        while k < len(cands) and not found:
            e = k
            while e < len(cands) and cands[e][0] == cands[k][0]:
                e += 1
            for c in cands[k:e]:
                als = [align(codes[m][int(mr(m, c[2]))], rcodes[c[1]], scoring, local)
                       for m in range(2)]
                if pair_ok([als[0][0], als[1][0]], [als[0][1], als[1][1]], c[2], max_insert):
                    found.append((c, als))
            k = e
        if not found:
            separate.append(p)
            continue
        in_set = {(c[1], c[2]) for c, _ in found}
        sub = [None, None]
        for t in strands:
            for r in range(n_refs):
                if (r, t) in in_set:
                    continue
                for m in range(2):
                    s = int(rows[m][mr(m, t)][r])
                    sub[m] = s if sub[m] is None else max(sub[m], s)
        keep = len(found) if max_ties is None else min(len(found), max_ties + 1)
        hits = []
        for c, als in found[:keep]:
            mates = []
            for m in range(2):
                rv = bool(mr(m, c[2]))
                a, ops = als[m]
                letters = revcomp_letters(pairs[p][m]) if rv else pairs[p][m]
                md, nm = md_nm(letters, refs[c[1]], int(a["query_start"]), int(a["ref_start"]),
                               ops)
                mates.append({"reference": c[1], "reverse": rv, "score": int(a["score"]),
                              "query_start": int(a["query_start"]),
                              "query_end": int(a["query_end"]),
                              "ref_start": int(a["ref_start"]), "ref_end": int(a["ref_end"]),
                              "cigar": cigar_string(ops), "md": md, "nm": nm})
            lo = min(mates[0]["ref_start"], mates[1]["ref_start"])
            hi = max(mates[0]["ref_end"], mates[1]["ref_end"])
            hits.append({"reference": c[1], "reverse": bool(c[2]), "insert": hi - lo,
                         "mates": mates})
        out[p] = {"proper": True, "score": found[0][0][0], "n_tied": len(found),
                  "suboptimal": sub, "hits": hits}
    separate += [p for p in range(len(pairs)) if p not in set(live)]
    separate.sort()
    if separate:
        flat = [pairs[p][m] for p in separate for m in range(2)]
        mapped = map_reads(flat, refs, scoring, local, min_score=min_score, max_ties=max_ties,
                           both_strands=True, threads=threads)
        for i, p in enumerate(separate):
            out[p] = {"proper": False, "mates": [mapped[2 * i], mapped[2 * i + 1]]}
    return out


def md_nm_codes(q, reverse, ref_codes, ref_letters, a, ops):
    """eo_md_nm: md_nm (sam.rs:76-121) on codes, reference letters optional."""
    q = np.ascontiguousarray(q, dtype=np.uint8)
    rc = np.ascontiguousarray(ref_codes, dtype=np.uint8)
    rl = None if ref_letters is None else np.frombuffer(bytes(ref_letters), dtype=np.uint8)
    rec = np.zeros(1, dtype=ALIGN_DTYPE)
    rec[0] = a
    ops = np.ascontiguousarray(ops, dtype=np.uint32)
    cap = 4 * (q.size + rc.size) + 16
    buf = C.create_string_buffer(cap)
    nm = C.c_uint32()
    w = lib().eo_md_nm(_p(q, C.c_uint8), q.size, int(bool(reverse)), _p(rc, C.c_uint8),
                       _p(rl, C.c_uint8) if rl is not None else None, rec.ctypes.data,
                       _p(ops, C.c_uint32), buf, cap, C.byref(nm))
    if w < 0:
        raise RuntimeError("eo_md_nm: MD buffer too small")
    return buf.raw[:w].decode(), nm.value


def cpu_map_reads(codes, off, lens, refs, scoring, local, min_score=0, max_ties=None,
                  both_strands=False, ref_letters=None, cap=32, threads=0, profile=None):
    """map_reads_scored on the host the way the reference's CPU path runs
    it, every stage in C on all threads: AVX-512 scores and the tie set
    (eo_cpu_map_batch; reads whose ties outrun `cap` take their list from
    full rows), the scalar traceback of the taken ties (eo_align_batch),
    MD / NM (eo_md_nm_batch).  Returns (results, jobs [read, ref, reverse],
    alignments, ops [n_jobs, stride], md strings, nm, threads used); the
    per-read dicts of map_reads come from cpu_mappings()."""
    prof = profile or Profile(refs, scoring)
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    off = np.ascontiguousarray(off, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    n = int(lens.size)
    res, ties, _, used = prof.map_batch(codes, off, lens, local, both_strands, cap=cap,
                                        threads=threads)
    take = np.zeros(n, dtype=np.int64)
    live = (res["flags"] & RESULT_EMPTY) == 0
    ok = live & (res["best"] >= min_score)
    nt = res["n_tied"].astype(np.int64)
    take[ok] = nt[ok] if max_ties is None else np.minimum(nt[ok], max_ties + 1)
    lists = {}
    redo = np.nonzero(take > np.minimum(nt, cap))[0]
    if redo.size:
        sub_off = off[redo]
        sub_len = lens[redo]
        r2, _, rows, _ = prof.map_batch(codes, sub_off, sub_len, local, both_strands, cap=1,
                                        threads=threads, rows=True)
        m = redo.size
        for i, k in enumerate(redo):
            best = int(res["best"][k])
            lst = []
            for r in range(len(refs)):
                if rows[i, r] == best:
                    lst.append(r << 1)
                if both_strands and rows[m + i, r] == best:
                    lst.append((r << 1) | 1)
            lists[int(k)] = lst
    jr, jf, jv = [], [], []
    for k in np.nonzero(take)[0]:
        lst = lists.get(int(k))
        t = int(take[k])
        cand = lst[:t] if lst is not None else ties[k, :t].tolist()
        for c in cand:
            jr.append(k)
            jf.append(int(c) >> 1)
            jv.append(int(c) & 1)
    jobs = np.stack([np.array(jr, np.uint32), np.array(jf, np.uint32),
                     np.array(jv, np.uint32)], 1) if jr else np.zeros((0, 3), np.uint32)
    al, ops, _ = align_batch(codes, off, lens, refs, jobs, scoring, local, threads=threads)
    rc_, ro, rl_ = pack(refs)
    letters = None
    if ref_letters is not None:
        letters = np.frombuffer(b"".join(bytes(x) for x in ref_letters), dtype=np.uint8)
    stride = ops.shape[1] if ops.ndim == 2 else 1
    md_stride = 4 * stride + 16
    nj = jobs.shape[0]
    md = np.zeros((max(nj, 1), md_stride), dtype=np.uint8)
    md_len = np.zeros(max(nj, 1), dtype=np.uint32)
    nm = np.zeros(max(nj, 1), dtype=np.uint32)
    jr_ = np.ascontiguousarray(jobs[:, 0])
    jf_ = np.ascontiguousarray(jobs[:, 1])
    jv_ = np.ascontiguousarray(jobs[:, 2].astype(np.uint8))
    if nj:
        w = lib().eo_md_nm_batch(_p(codes, C.c_uint8), _p(off, C.c_uint64), _p(lens, C.c_uint32),
                                 _p(rc_, C.c_uint8), _p(ro, C.c_uint64),
                                 _p(letters, C.c_uint8) if letters is not None else None,
                                 _p(jr_, C.c_uint32), _p(jf_, C.c_uint32), _p(jv_, C.c_uint8),
                                 al.ctypes.data, _p(ops, C.c_uint32), stride, nj, threads,
                                 md.ctypes.data, md_stride, _p(md_len, C.c_uint32),
                                 _p(nm, C.c_uint32))
        if w < 0:
            raise RuntimeError("eo_md_nm_batch: MD stride too small")
    mds = [md[k, :md_len[k]].tobytes().decode() for k in range(nj)]
    return res, jobs, al, ops, mds, nm[:nj], used


def cpu_mappings(res, jobs, al, ops, mds, nm):
    """cpu_map_reads' output as map_reads' per-read dicts (mapper.rs:497-552)."""
    out = []
    by = {}
    for i, k in enumerate(jobs[:, 0].tolist()):
        by.setdefault(k, []).append(i)
    for k in range(res.size):
        r = res[k]
        if r["flags"] & RESULT_EMPTY:
            out.append({"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []})
            continue
        rec = {"best_score": int(r["best"]), "n_tied": int(r["n_tied"]),
               "suboptimal": None if r["suboptimal"] == NO_SCORE else int(r["suboptimal"]),
               "hits": []}
        js = by.get(k, [])
        if js and _aligned_any(ops[js[0], :int(al[js[0]]["n_ops"])]):
            for i in js:
                a = al[i]
                w = ops[i, :int(a["n_ops"])]
                rec["hits"].append({"reference": int(jobs[i, 1]), "reverse": bool(jobs[i, 2]),
                                    "score": int(a["score"]),
                                    "query_start": int(a["query_start"]),
                                    "query_end": int(a["query_end"]),
                                    "ref_start": int(a["ref_start"]),
                                    "ref_end": int(a["ref_end"]), "cigar": cigar_string(w),
                                    "md": mds[i], "nm": int(nm[i])})
        out.append(rec)
    return out


def _code_letters(c) -> bytes:
    return bytes(b"ACGTN"[min(int(x), 4)] for x in c)


def cpu_map_pairs(codes, off, lens, refs, scoring, local, min_score=0, max_ties=None,
                  max_insert=500, both_strands=False, ref_letters=None, cap=32, threads=0,
                  profile=None, trim=False):
    """map_pairs_scored on the host cores, the stages in C on all threads:
    the candidate ranking from AVX-512 rows (eo_cpu_map_pairs, no trimming:
    the mates come trimmed), the scalar traceback of every pair's first tier
    (eo_align_batch), the pair constraints on the traced tier, MD / NM
    (eo_md_nm_batch), and cpu_map_reads for the Separate mates.  Pairs whose
    first tier all fails or outruns `cap` take the Python restatement
    (map_pairs).  With `trim` the mates are untrimmed and the ranking call
    trims them first (TruSeq adapters, adapter.rs:68-110, as the CLI does).
    Returns (map_pairs' per-pair dicts, threads used)."""
    prof = profile or Profile(refs, scoring)
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    off = np.ascontiguousarray(off, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    n = int(lens.size) // 2
    letters = ref_letters if ref_letters is not None else [_code_letters(r) for r in refs]
    if trim:
        res, ties, _, _, ads, used = prof.map_pairs(codes, off, lens, local, both_strands,
                                                    min_score, cap, threads)
        lens = np.ascontiguousarray(lens - ads, dtype=np.uint32)
    else:
        res, ties, _, _, _, used = prof.map_pairs(codes, off, lens, local, both_strands,
                                                  min_score, cap, threads, a1=b"", a2=b"")
    # --- the first tiers, traced together
    tier = [p for p in range(n) if not res["flags"][p] & RESULT_EMPTY and res["n_tied"][p] <= cap]
    jr, jf, jv, owner = [], [], [], []
    for p in tier:
        for i in range(int(res["n_tied"][p])):
            c = int(ties[p, i])
            for m in range(2):
                jr.append(2 * p + m)
                jf.append(c >> 1)
                jv.append((c & 1) ^ (m == 1))
            owner.append((p, c))
    jobs = (np.stack([np.array(jr, np.uint32), np.array(jf, np.uint32),
                      np.array(jv, np.uint32)], 1) if jr else np.zeros((0, 3), np.uint32))
    al, ops, _ = align_batch(codes, off, lens, refs, jobs, scoring, local, threads=threads)
    nc = len(owner)
    ok = np.zeros(nc, dtype=bool)
    if nc:
        a0, a1 = al[0::2], al[1::2]
        cols = np.arange(ops.shape[1])[None, :]
        matched = ((ops & 0xf) == 0) & (cols < al["n_ops"][:, None].astype(np.int64))
        aligned = matched.any(axis=1)
        t = np.array([c & 1 for _, c in owner], dtype=bool)
        fs = np.where(t, a1["ref_start"], a0["ref_start"]).astype(np.int64)
        re_ = np.where(t, a0["ref_end"], a1["ref_end"]).astype(np.int64)
        lo = np.minimum(a0["ref_start"], a1["ref_start"]).astype(np.int64)
        hi = np.maximum(a0["ref_end"], a1["ref_end"]).astype(np.int64)
        ok = aligned[0::2] & aligned[1::2] & (fs < re_) & (hi - lo <= max_insert)
    # --- MD / NM of every traced mate (only the kept ones are read)
    md_stride = 4 * ops.shape[1] + 16
    nj = jobs.shape[0]
    md = np.zeros((max(nj, 1), md_stride), dtype=np.uint8)
    md_len = np.zeros(max(nj, 1), dtype=np.uint32)
    nm = np.zeros(max(nj, 1), dtype=np.uint32)
    if nj:
        rc_, ro, _ = pack(refs)
        lt = np.frombuffer(b"".join(bytes(x) for x in letters), dtype=np.uint8)
        jr_ = np.ascontiguousarray(jobs[:, 0])
        jf_ = np.ascontiguousarray(jobs[:, 1])
        jv_ = np.ascontiguousarray(jobs[:, 2].astype(np.uint8))
        if lib().eo_md_nm_batch(_p(codes, C.c_uint8), _p(off, C.c_uint64), _p(lens, C.c_uint32),
                                _p(rc_, C.c_uint8), _p(ro, C.c_uint64), _p(lt, C.c_uint8),
                                _p(jr_, C.c_uint32), _p(jf_, C.c_uint32), _p(jv_, C.c_uint8),
                                al.ctypes.data, _p(ops, C.c_uint32), ops.shape[1], nj, threads,
                                md.ctypes.data, md_stride, _p(md_len, C.c_uint32),
                                _p(nm, C.c_uint32)) < 0:
            raise RuntimeError("eo_md_nm_batch: MD stride too small")

    def hit(j):
        a = al[j]
        w = ops[j, :int(a["n_ops"])]
        return {"reference": int(jobs[j, 1]), "reverse": bool(jobs[j, 2]),
                "score": int(a["score"]), "query_start": int(a["query_start"]),
                "query_end": int(a["query_end"]), "ref_start": int(a["ref_start"]),
                "ref_end": int(a["ref_end"]), "cigar": cigar_string(w),
                "md": md[j, :md_len[j]].tobytes().decode(), "nm": int(nm[j])}

    out = [None] * n
    slow, separate = [], []
    k = 0
    for p in range(n):
        if res["flags"][p] & RESULT_EMPTY:
            separate.append(p)
            continue
        if res["n_tied"][p] > cap:
            slow.append(p)
            continue
        m = int(res["n_tied"][p])
        idx = list(range(k, k + m))
        k += m
        found = [i for i in idx if ok[i]]
        if not found:
            slow.append(p)
            continue
        sub = [None if res["xs"][p][q] == NO_SCORE else int(res["xs"][p][q]) for q in range(2)]
        for i in idx:
            if not ok[i]:
                for q in range(2):
                    s = int(al[2 * i + q]["score"])
                    sub[q] = s if sub[q] is None else max(sub[q], s)
        keep = len(found) if max_ties is None else min(len(found), max_ties + 1)
        hits = []
        for i in found[:keep]:
            mates = [hit(2 * i), hit(2 * i + 1)]
            lo = min(mates[0]["ref_start"], mates[1]["ref_start"])
            hi = max(mates[0]["ref_end"], mates[1]["ref_end"])
            hits.append({"reference": int(owner[i][1] >> 1), "reverse": bool(owner[i][1] & 1),
                         "insert": hi - lo, "mates": mates})
        out[p] = {"proper": True, "score": int(res["best"][p]), "n_tied": len(found),
                  "suboptimal": sub, "hits": hits}
    if slow:
        pl = [(_code_letters(codes[off[2 * p]:off[2 * p] + lens[2 * p]]),
               _code_letters(codes[off[2 * p + 1]:off[2 * p + 1] + lens[2 * p + 1]]))
              for p in slow]
        for p, r in zip(slow, map_pairs(pl, letters, scoring, local, min_score=min_score,
                                        max_ties=max_ties, max_insert=max_insert,
                                        both_strands=both_strands, threads=threads)):
            out[p] = r
    if separate:
        so = np.array([off[2 * p + q] for p in separate for q in range(2)], dtype=np.uint64)
        sl = np.array([lens[2 * p + q] for p in separate for q in range(2)], dtype=np.uint32)
        mapped = cpu_mappings(*cpu_map_reads(codes, so, sl, refs, scoring, local,
                                             min_score=min_score, max_ties=max_ties,
                                             both_strands=True, ref_letters=letters, cap=cap,
                                             threads=threads, profile=prof)[:6])
        for i, p in enumerate(separate):
            out[p] = {"proper": False, "mates": [mapped[2 * i], mapped[2 * i + 1]]}
    return out, used
