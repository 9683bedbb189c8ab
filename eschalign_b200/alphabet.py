"""The scoring alphabet (crates/eschalign/src/alphabet.rs:7-64).

A/C/G/T encode to 0-3, U folds to T, case is ignored, and every other byte
encodes to WILDCARD (4), which pairs with any code as a match.
"""
from __future__ import annotations

import numpy as np

A, C, G, T, WILDCARD = 0, 1, 2, 3, 4
N_CODES = 5

_TABLE = np.full(256, WILDCARD, dtype=np.uint8)
for _ch, _c in (("A", A), ("C", C), ("G", G), ("T", T), ("U", T)):
    _TABLE[ord(_ch)] = _c
    _TABLE[ord(_ch.lower())] = _c


def encode(letters) -> np.ndarray:
    """alphabet.rs:48-55 -- letters (str, bytes or uint8 array) to codes."""
    if isinstance(letters, str):
        letters = letters.encode()
    return _TABLE[np.frombuffer(bytes(letters), dtype=np.uint8)] if not isinstance(
        letters, np.ndarray) else _TABLE[letters.astype(np.uint8, copy=False)]


def encode_base(b: int) -> int:
    return int(_TABLE[b])


def reverse_complement_codes(codes) -> np.ndarray:
    """alphabet.rs:58-64 -- reversed, c -> 3 - c, the wildcard stays."""
    c = np.asarray(codes, dtype=np.uint8)[::-1]
    return np.where(c >= WILDCARD, WILDCARD, 3 - c).astype(np.uint8)
