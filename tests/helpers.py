"""Generators of the reference's own tests, restated: xorshift64* and the
read / panel builders of crates/eschalign/tests/gpu_parity.rs:32-126 and
crates/eschalign/src/simd/mod.rs:685-740."""
import json
import os

import numpy as np

from eschalign_b200 import encode

MASK = (1 << 64) - 1
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class Rng:
    """xorshift64* (gpu_parity.rs:34-48)."""

    def __init__(self, seed):
        self.s = seed & MASK

    def next(self):
        x = self.s
        x ^= x >> 12
        x ^= (x << 25) & MASK
        x ^= x >> 27
        self.s = x
        return (x * 0x2545F4914F6CDD1D) & MASK

    def below(self, n):
        return self.next() % n

    def chance(self, p):
        return (self.next() >> 11) / float(1 << 53) <= p


def random_seq(rng, n, n_rate):
    out = bytearray()
    for _ in range(n):
        out.append(ord("N") if rng.chance(n_rate) else b"ACGT"[rng.below(4)])
    return bytes(out)


def mutate(rng, s):
    """gpu_parity.rs:62-79."""
    out = bytearray()
    for b in s:
        if rng.chance(0.04):
            continue
        out.append(b"ACGT"[rng.below(4)] if rng.chance(0.05) else b)
        if rng.chance(0.03):
            out.append(b"ACGT"[rng.below(4)])
    return bytes(out)


def random_panel(rng, n_refs, min_len, spread):
    """gpu_parity.rs:81-87 -> list of letter strings."""
    return [random_seq(rng, min_len + rng.below(spread), 0.01) for _ in range(n_refs)]


def reads_for(rng, panel, n):
    """gpu_parity.rs:107-126: every length 1..40, then reads drawn from the
    panel (mutated) and unrelated random reads.  Returns code arrays."""
    reads = [random_seq(rng, ln, 0.02) for ln in range(1, 41)]
    for t in range(n):
        if t % 4 == 3:
            reads.append(random_seq(rng, 1 + rng.below(300), 0.02))
        else:
            r = panel[rng.below(len(panel))]
            a = rng.below(len(r) // 3 + 1)
            b = len(r) - rng.below(len(r) // 3 + 1)
            lead, tail = rng.below(30), rng.below(30)
            read = random_seq(rng, lead, 0.0) + mutate(rng, r[a:max(b, a)]) + random_seq(rng, tail, 0.0)
            reads.append(read)
    return [encode(r) for r in reads]


SCHEMES = [(2, -1, -10, -1), (1, -1, -2, -1), (3, -2, -5, -2), (3, 1, -5, -2), (2, -1, 0, 0)]


def golden():
    with open(os.path.join(GOLDEN, "align_golden_scores.json")) as fh:
        return json.load(fh)


def fixture_panel(tag):
    with open(os.path.join(GOLDEN, f"panel_{tag}.json")) as fh:
        d = json.load(fh)
    return [encode(r["seq"]) for r in d["references"]]


def fixture_reads():
    return [encode(s) for s in golden()["fixture_reads"]]


def revcomp(c):
    c = np.asarray(c, dtype=np.uint8)[::-1]
    return np.where(c >= 4, 4, 3 - c).astype(np.uint8)


def pairs_fixture():
    """The reference's paired fixture (crates/eschalign-cli/tests/fixtures/pairs,
    via tests/golden/make_golden.py): reference names, reference codes, and
    {pair name: (mate 1 codes, mate 2 codes)} in file order."""
    with open(os.path.join(GOLDEN, "pairs_fixture.json")) as fh:
        d = json.load(fh)
    names = [r["name"] for r in d["references"]]
    refs = [encode(r["seq"]) for r in d["references"]]
    pairs = {p["name"]: (encode(p["r1"]), encode(p["r2"])) for p in d["pairs"]}
    return names, refs, pairs


def brute_pair_select(f0, r0, f1, r1, both, min_score, cap):
    """pair.rs:195-234 spelled out: every candidate, sorted by (-sum, r, t)."""
    cands = []
    for r in range(len(f0)):
        for t in ((0, 1) if both else (0,)):
            a, b = (int(r0[r]), int(f1[r])) if t else (int(f0[r]), int(r1[r]))
            cands.append((a, b, r, t))
    elig = sorted([c for c in cands if c[0] >= min_score and c[1] >= min_score],
                  key=lambda c: (-(c[0] + c[1]), c[2], c[3]))
    if not elig:
        best = None
        tier = []
    else:
        best = elig[0][0] + elig[0][1]
        tier = [c for c in elig if c[0] + c[1] == best]
    rest = [c for c in elig if c[0] + c[1] != best]
    nxt = rest[0][0] + rest[0][1] if rest else None
    in_tier = {(c[2], c[3]) for c in tier}
    outside = [c for c in cands if (c[2], c[3]) not in in_tier]
    xs = (max((c[0] for c in outside), default=None), max((c[1] for c in outside), default=None))
    prim = (tier[0][0], tier[0][1]) if tier else (None, None)
    return best, nxt, len(tier), [(c[2] << 1) | c[3] for c in tier[:cap]], xs, prim
