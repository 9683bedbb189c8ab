"""The reference panel (crates/eschalign/src/panel.rs) and a FASTA reader
(crates/eschalign/src/fasta.rs:42-88, first word of the header as the name,
duplicates refused)."""
from __future__ import annotations

import numpy as np

from .alphabet import encode


class PanelError(ValueError):
    """AlignError::EmptyPanel / EmptyReference / DuplicateReferenceName."""


class Panel:
    """References in the order given; order is the @SQ order and ties break
    toward the lowest index (panel.rs:234-237)."""

    def __init__(self, refs):
        self.names, self.seqs, self.codes = [], [], []
        for name, seq in refs:
            if isinstance(seq, str):
                seq = seq.encode()
            if len(seq) == 0:
                raise PanelError(f"reference {name!r} has no bases")
            self.names.append(str(name))
            self.seqs.append(bytes(seq))
            self.codes.append(encode(seq))
        if not self.codes:
            raise PanelError("the reference panel is empty")

    @classmethod
    def from_codes(cls, codes_list, names=None):
        p = cls.__new__(cls)
        p.codes = [np.asarray(c, dtype=np.uint8) for c in codes_list]
        if not p.codes:
            raise PanelError("the reference panel is empty")
        for k, c in enumerate(p.codes):
            if c.size == 0:
                raise PanelError(f"reference {k} has no bases")
        p.names = list(names) if names else [f"r{k}" for k in range(len(p.codes))]
        letters = np.frombuffer(b"ACGTN", dtype=np.uint8)
        p.seqs = [letters[np.minimum(c, 4)].tobytes() for c in p.codes]
        return p

    def __len__(self):
        return len(self.codes)

    def max_len(self) -> int:
        return max(c.size for c in self.codes)

    def total_len(self) -> int:
        return int(sum(c.size for c in self.codes))

    def packed(self):
        """(codes, off u64, len u32) as the C ABI takes them."""
        lens = np.array([c.size for c in self.codes], dtype=np.uint32)
        off = np.zeros(len(self.codes), dtype=np.uint64)
        off[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
        return np.ascontiguousarray(np.concatenate(self.codes)), off, lens


def read_fasta(path):
    recs, seen, name, seq = [], set(), None, []
    with open(path, "rb") as fh:
        for raw in fh:
            line = raw.rstrip(b"\r\n")
            if line.startswith(b">"):
                if name is not None:
                    recs.append((name, b"".join(seq)))
                words = line[1:].split()
                if not words:
                    raise PanelError("empty reference name")
                name = words[0].decode()
                if name in seen:
                    raise PanelError(f"duplicate reference name {name!r}")
                seen.add(name)
                seq = []
            elif name is not None:
                seq.append(b"".join(line.split()))
            elif line.strip():
                raise PanelError("sequence data before the first '>' header")
    if name is not None:
        recs.append((name, b"".join(seq)))
    return recs
