"""3' adapter read-through settings (crates/eschalign/src/adapter.rs:38-54).

The search itself runs inside the library when a paired batch is prepared
(esg_prepare_pairs): ``find`` (adapter.rs:68-91) on each mate and the
two-mate reconciliation of ``detect_pair`` (adapter.rs:95-110), with the
CLI's rule for mates over ``--max-read-len`` (align.rs:934-949).
"""
from __future__ import annotations

from .alphabet import encode

TRUSEQ_R1 = b"AGATCGGAAGAGCACACGTCTGAACTCCAGTCA"  # adapter.rs:40
TRUSEQ_R2 = b"AGATCGGAAGAGCGTCGTGTAGGGAAAGAGTGT"  # adapter.rs:42
DEFAULT_MIN_OVERLAP = 5                           # adapter.rs:44


def config(r1=TRUSEQ_R1, r2=TRUSEQ_R2, min_overlap=DEFAULT_MIN_OVERLAP, max_read_len=0) -> dict:
    """AdapterConfig (adapter.rs:46-54) as GpuScorer.prepare_pairs takes it:
    adapter letters encoded, and the CLI's read-length limit (0 = none)."""
    return {"r1": encode(r1), "r2": encode(r2), "min_overlap": int(min_overlap),
            "max_read_len": int(max_read_len)}


def pair_adapters(mates, cfg: dict | None = None):
    """pair_adapters (align.rs:934-949) over a batch of mates (2p, 2p + 1),
    in the library (esg_pair_adapters, host threads, no device).  Returns
    (adapter bases per mate, bases left to align per mate)."""
    import ctypes as C

    import numpy as np

    from . import _native
    from .scorer import _check, _inputs_of, _ptr

    lib = _native.load()
    codes, off, lens = _inputs_of(mates)
    if lens.size % 2:
        raise ValueError("mates come in pairs: an even number of reads is needed")
    cfg = config() if cfg is None else cfg
    r1 = np.ascontiguousarray(cfg.get("r1", np.zeros(0)), dtype=np.uint8)
    r2 = np.ascontiguousarray(cfg.get("r2", np.zeros(0)), dtype=np.uint8)
    c = _native.EsgAdapterConfig(r1.ctypes.data if r1.size else None, r1.size,
                                 r2.ctypes.data if r2.size else None, r2.size,
                                 int(cfg.get("min_overlap", DEFAULT_MIN_OVERLAP)),
                                 int(cfg.get("max_read_len", 0)))
    ads = np.zeros(lens.size, dtype=np.uint32)
    aligned = np.zeros(lens.size, dtype=np.uint32)
    _check(lib, lib.esg_pair_adapters(_ptr(codes, C.c_uint8), _ptr(off, C.c_uint64),
                                      _ptr(lens, C.c_uint32), lens.size // 2, C.byref(c),
                                      _ptr(ads, C.c_uint32), _ptr(aligned, C.c_uint32)))
    return ads, aligned
