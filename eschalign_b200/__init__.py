"""eschalign_b200 -- eschalign's panel-scoring hot path, B200-native.

Every read of a batch against every reference of a panel (Gotoh affine
gaps, local or semi-global, forward and reverse complement), reduced on the
device to each read's best score, suboptimal score and tie set.  The host
side mirrors eschalign's ``GpuScorer`` (crates/eschalign/src/cuda/mod.rs);
the device side is ``libeschalign_b200.so`` (CUDA, sm_100a), whose C ABI is
include/eschalign_b200.h.
"""
from . import adapter
from ._native import build, load
from .alphabet import WILDCARD, encode, reverse_complement_codes
from .panel import Panel, PanelError, read_fasta
from .scorer import (BOTH_STRANDS, FULL_ROWS, KERNEL_AUTO, KERNEL_INT32, KERNEL_PLAIN32, NO_SCORE,
                     BatchResult, GpuError, GpuScorer, PairBatchResult, PairScores, ReadScores,
                     ScoreMatrix, device_visible, fits_i16, pack_reads, select_hits)
from .scoring import Mode, Scoring, ScoringError

__all__ = [
    "adapter", "build", "load", "WILDCARD", "encode", "reverse_complement_codes", "Panel", "PanelError",
    "read_fasta", "BOTH_STRANDS", "FULL_ROWS", "KERNEL_AUTO", "KERNEL_INT32", "KERNEL_PLAIN32", "NO_SCORE",
    "BatchResult", "GpuError", "GpuScorer", "PairBatchResult", "PairScores", "ReadScores", "ScoreMatrix", "device_visible",
    "fits_i16", "pack_reads", "select_hits", "Mode", "Scoring", "ScoringError",
]
