"""ctypes view of the CPU checker (oracle/_build/libesg_oracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference legs, never by the product package.

* :func:`score` -- scalar Gotoh, crates/eschalign/src/scalar.rs:120-163;
* :func:`select` -- tie set / XS, crates/eschalign/src/mapper.rs:444-472;
* :class:`Profile` -- the AVX-512BW inter-sequence kernels,
  crates/eschalign/src/simd/avx512.rs:43-107 and :278-354, with the
  reference's dispatch (mapper.rs:216-222).
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


def build() -> str:
    """Compile the checker with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


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
