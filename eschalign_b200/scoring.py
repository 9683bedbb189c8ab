"""Scoring scheme and alignment modes (crates/eschalign/src/scoring.rs).

A gap of k bases scores ``gap_open + (k - 1) * gap_extend``
(scoring.rs:18-25); a match is two equal codes or either one the wildcard
(scoring.rs:105-111).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass

MAX_SCORE_MAGNITUDE = 1000  # scoring.rs:14


class ScoringError(ValueError):
    """AlignError::ScoringSyntax / ScoringInvalid (error.rs:9-11)."""


@dataclass(frozen=True)
class Scoring:
    match_score: int = 2
    mismatch: int = -1
    gap_open: int = -10
    gap_extend: int = -1

    def __post_init__(self):
        self.validate()

    def validate(self) -> None:
        """scoring.rs:70-100."""
        if self.match_score <= 0:
            raise ScoringError(f"match must be positive, got {self.match_score}")
        if self.mismatch >= self.match_score:
            raise ScoringError(f"mismatch ({self.mismatch}) must score below match "
                               f"({self.match_score})")
        if self.gap_open > 0 or self.gap_extend > 0:
            raise ScoringError("gap scores are penalties and must be zero or negative, got "
                               f"open {self.gap_open} extend {self.gap_extend}")
        for v in self.astuple():
            if abs(v) > MAX_SCORE_MAGNITUDE:
                raise ScoringError(f"|{v}| exceeds the supported magnitude {MAX_SCORE_MAGNITUDE}")

    @classmethod
    def parse(cls, s: str) -> "Scoring":
        """scoring.rs:120-137: ``MATCH,MISMATCH,GAP_OPEN,GAP_EXTEND``."""
        parts = [p.strip() for p in s.split(",")]
        if len(parts) != 4:
            raise ScoringError(f"scoring {s!r} is not MATCH,MISMATCH,GAP_OPEN,GAP_EXTEND")
        try:
            v = [int(p) for p in parts]
        except ValueError:
            raise ScoringError(f"scoring {s!r} is not MATCH,MISMATCH,GAP_OPEN,GAP_EXTEND") from None
        return cls(*v)

    def substitution(self, a: int, b: int) -> int:
        return self.match_score if (a == b or a == 4 or b == 4) else self.mismatch

    def gap(self, length: int) -> int:
        return self.gap_open + (length - 1) * self.gap_extend

    def astuple(self):
        return (self.match_score, self.mismatch, self.gap_open, self.gap_extend)

    def __str__(self):
        return ",".join(str(v) for v in self.astuple())


class Mode(enum.IntEnum):
    """scoring.rs:149-186."""
    LOCAL = 0
    SEMIGLOBAL = 1

    @classmethod
    def parse(cls, s: str) -> "Mode":
        if s == "local":
            return cls.LOCAL
        if s in ("semiglobal", "semi-global", "overlap"):
            return cls.SEMIGLOBAL
        raise ValueError(f"unknown mode {s!r}, expected local|semiglobal")

    @property
    def label(self) -> str:
        return "local" if self is Mode.LOCAL else "semiglobal"
