"""Seeded synthetic panels and reads with the shapes of the benchmark configs.

They stand in for the reference's real samples (tRNA reads M1/M4 and the
sacCer3 panel of benchmarks/README.md), which are not shipped: uniform ACGT
references, reads cut from a random reference and mutated with the stated
substitution / insertion / deletion rates (indel lengths geometric), plus a
share of unrelated random reads.  Everything is vectorised numpy (PCG64 from
a named seed), so a million reads take about a second and every machine
builds the same bytes.

Sizes:
* ``panel_tiles``   164 references, lengths uniform 70-180 (C1, C2, C4)
* ``reads_c1``      10 000 reads, 90 % cut from a reference (start 0-20,
                    length 60-200 with a random 0-30 nt 3' tail), 8 % subs,
                    2 % insertions, 1 % deletions; 10 % random of 60-200 nt
* ``reads_c2``      1 000 000 reads, lengths lognormal (median 110, sigma
                    0.4) clipped to 20-1000, same mutation model
* ``panel_c3``      10 000 references of 300-1000 nt (GC 0.5)
* ``reads_c3``      200 000 reads of 50-1000 nt, 70 % derived (10 % subs,
                    3 % indels), 30 % random
* ``pairs_c4``      2 x 150 nt mates, inserts lognormal (median 90) clipped
                    to 40-600, adapter read-through past short inserts
"""
from __future__ import annotations

import numpy as np

from .adapter import TRUSEQ_R1, TRUSEQ_R2

SEED_PANEL = 0x5EED_C1C2
SEED_C1 = 0x5EED_0C01
SEED_C2 = 0x5EED_0C02
SEED_C3_PANEL = 0x5EED_C3A0
SEED_C3 = 0x5EED_0C03
SEED_C4 = 0x5EED_0C04


class Packed:
    """Reads as the C ABI takes them: contiguous codes, u64 offsets, u32 lengths."""

    def __init__(self, codes, off, lens):
        self.codes = np.ascontiguousarray(codes, dtype=np.uint8)
        self.off = np.ascontiguousarray(off, dtype=np.uint64)
        self.lens = np.ascontiguousarray(lens, dtype=np.uint32)

    def __len__(self):
        return int(self.lens.size)

    def tuple(self):
        return self.codes, self.off, self.lens

    def read(self, k):
        o = int(self.off[k])
        return self.codes[o:o + int(self.lens[k])]

    def list(self):
        return [self.read(k) for k in range(len(self))]

    def slice(self, k0, k1):
        """Reads k0..k1-1 as a view (reads are stored in order)."""
        k1 = min(k1, len(self))
        if k1 <= k0:
            return Packed(np.zeros(1, np.uint8), np.zeros(0, np.uint64), np.zeros(0, np.uint32))
        o0 = int(self.off[k0])
        o1 = int(self.off[k1 - 1]) + int(self.lens[k1 - 1])
        return Packed(self.codes[o0:max(o1, o0 + 1)], self.off[k0:k1] - np.uint64(o0),
                      self.lens[k0:k1])

    def subset(self, idx):
        idx = np.asarray(idx)
        parts = [self.read(int(k)) for k in idx]
        lens = self.lens[idx].astype(np.uint32)
        off = np.zeros(idx.size, dtype=np.uint64)
        if idx.size > 1:
            off[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
        codes = np.concatenate(parts) if lens.sum() else np.zeros(1, np.uint8)
        return Packed(codes, off, lens)

    def bases(self) -> int:
        return int(self.lens.sum(dtype=np.uint64))


def _offsets(lens):
    off = np.zeros(lens.size, dtype=np.uint64)
    if lens.size > 1:
        off[1:] = np.cumsum(lens[:-1].astype(np.uint64))
    return off


def random_bases(rng, n, gc=0.5):
    if gc == 0.5:
        return rng.integers(0, 4, n, dtype=np.uint8)
    u = rng.random(n)
    at = (1 - gc) / 2
    return np.searchsorted(np.cumsum([at, gc / 2, gc / 2]), u).astype(np.uint8)


def panel(n_refs, lo, hi, seed, gc=0.5):
    """n_refs uniform references with lengths uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, n_refs)
    return [random_bases(rng, int(m), gc) for m in lens]


def panel_tiles(seed=SEED_PANEL):
    return panel(164, 70, 180, seed)


def panel_c3(seed=SEED_C3_PANEL, n_refs=10_000):
    return panel(n_refs, 300, 1000, seed)


def mutate(rng, codes, lens, p_sub, p_ins, p_del, p_geom=0.6):
    """Mutate concatenated sequences (segment lengths `lens`): per base a
    deletion starts with p_del (geometric length), the base is substituted
    with p_sub (by a different base), and an insertion (geometric length of
    random bases) follows it with p_ins.  Returns (codes, lens)."""
    n = codes.size
    if n == 0:
        return codes, lens
    lens = np.asarray(lens, dtype=np.int64)
    bounds = np.cumsum(lens)
    keep = np.ones(n, dtype=np.int8)
    starts = np.nonzero(rng.random(n) < p_del)[0]
    if starts.size:
        dl = rng.geometric(p_geom, starts.size)
        seg_end = bounds[np.searchsorted(bounds, starts, side="right")]
        ends = np.minimum(starts + dl, seg_end)
        diff = np.zeros(n + 1, dtype=np.int32)
        np.add.at(diff, starts, 1)
        np.add.at(diff, ends, -1)
        keep[np.cumsum(diff[:-1]) > 0] = 0
    out = codes.copy()
    sub = np.nonzero(rng.random(n) < p_sub)[0]
    if sub.size:
        out[sub] = (out[sub] + rng.integers(1, 4, sub.size)) % 4
    reps = keep.astype(np.int32)
    ii = np.nonzero(rng.random(n) < p_ins)[0]
    if ii.size:
        reps[ii] += rng.geometric(p_geom, ii.size).astype(np.int32)
    idx_t = np.int32 if n < (1 << 31) else np.int64
    src = np.repeat(np.arange(n, dtype=idx_t), reps)
    new = out[src]
    # inserted copies (all but the first of a kept base, all of a deleted one)
    cs = np.cumsum(reps, dtype=np.int64)
    first = np.zeros(src.size, dtype=bool)
    starts_out = cs - reps
    first[starts_out[reps > 0]] = True
    is_ins = ~first | (keep[src] == 0)
    new[is_ins] = rng.integers(0, 4, int(is_ins.sum()), dtype=np.uint8)
    cs0 = np.concatenate(([0], cs))
    new_lens = cs0[bounds] - cs0[bounds - lens]
    return new, new_lens


def _ranges(starts, lens):
    """Concatenated index ranges [starts[i], starts[i] + lens[i])."""
    lens = np.asarray(lens, dtype=np.int64)
    total = int(lens.sum())
    base = np.repeat(np.asarray(starts, dtype=np.int64) - (np.cumsum(lens) - lens), lens)
    return base + np.arange(total, dtype=np.int64)


def derived_reads(rng, refs, target, p_sub, p_ins, p_del, start_max=20, tail_max=30):
    """Reads of exactly `target` bases cut from random references: a body
    starting 0..start_max into the reference, mutated, then a random 3'
    tail of 0..tail_max bases (more when the reference runs out)."""
    target = np.asarray(target, dtype=np.int64)
    ref_lens = np.array([r.size for r in refs], dtype=np.int64)
    ref_off = _offsets(ref_lens).astype(np.int64)
    cat = np.concatenate(refs)
    n = target.size
    which = rng.integers(0, len(refs), n)
    start = np.minimum(rng.integers(0, start_max + 1, n), ref_lens[which] - 1)
    tail = rng.integers(0, tail_max + 1, n)
    body = np.minimum(np.clip(target - tail, 1, None), ref_lens[which] - start)
    codes = cat[_ranges(ref_off[which] + start, body)]
    codes, lens = mutate(rng, codes, body, p_sub, p_ins, p_del)
    take = np.minimum(lens, target)
    pad = target - take
    out = np.empty(int(target.sum()), dtype=np.uint8)
    o_off = np.cumsum(target) - target
    src_off = np.cumsum(lens) - lens
    out[_ranges(o_off, take)] = codes[_ranges(src_off, take)]
    out[_ranges(o_off + take, pad)] = random_bases(rng, int(pad.sum()))
    return out, target


def mixed_reads(rng, refs, lens, frac_derived, p_sub, p_ins, p_del):
    n = lens.size
    derived = rng.random(n) < frac_derived
    d_codes, d_lens = derived_reads(rng, refs, lens[derived], p_sub, p_ins, p_del)
    r_lens = lens[~derived]
    r_codes = random_bases(rng, int(r_lens.sum()))
    # stitch back in read order
    all_lens = np.zeros(n, dtype=np.int64)
    all_lens[derived] = d_lens
    all_lens[~derived] = r_lens
    off = _offsets(all_lens)
    codes = np.empty(int(all_lens.sum()), dtype=np.uint8)
    di = np.nonzero(derived)[0]
    ri = np.nonzero(~derived)[0]
    for idx_set, src, src_lens in ((di, d_codes, d_lens), (ri, r_codes, r_lens)):
        if idx_set.size == 0:
            continue
        codes[_ranges(off[idx_set], src_lens)] = src
    return Packed(codes, off, all_lens.astype(np.uint32))


def reads_c1(refs, n=10_000, seed=SEED_C1):
    rng = np.random.default_rng(seed)
    lens = rng.integers(60, 201, n)
    return mixed_reads(rng, refs, lens, 0.9, 0.08, 0.02, 0.01)


def lognormal_lengths(rng, n, median, sigma, lo, hi):
    return np.clip(np.round(median * np.exp(sigma * rng.standard_normal(n))), lo, hi).astype(np.int64)


def reads_c2(refs, n=1_000_000, seed=SEED_C2):
    rng = np.random.default_rng(seed)
    lens = lognormal_lengths(rng, n, 110, 0.4, 20, 1000)
    return mixed_reads(rng, refs, lens, 0.9, 0.08, 0.02, 0.01)


def reads_c3(refs, n=200_000, seed=SEED_C3):
    rng = np.random.default_rng(seed)
    lens = rng.integers(50, 1001, n)
    return mixed_reads(rng, refs, lens, 0.7, 0.10, 0.015, 0.015)


def _seg_revcomp(codes, off, lens):
    """Reverse-complement every segment of a concatenation (wildcard stays)."""
    lens = np.asarray(lens, dtype=np.int64)
    off = np.asarray(off, dtype=np.int64)
    k = np.arange(int(lens.sum()), dtype=np.int64) - np.repeat(np.cumsum(lens) - lens, lens)
    src = np.repeat(off + lens - 1, lens) - k
    c = codes[src]
    return np.where(c == 4, 4, 3 - c).astype(np.uint8)


def _fix_length(rng, codes, lens, target):
    """Cut or pad (random bases) each segment to `target` bases."""
    lens = np.asarray(lens, dtype=np.int64)
    n = lens.size
    take = np.minimum(lens, target)
    out = random_bases(rng, n * target)
    o_off = np.arange(n, dtype=np.int64) * target
    out[_ranges(o_off, take)] = codes[_ranges(np.cumsum(lens) - lens, take)]
    return out


def pairs_c4(refs, n=2_000_000, seed=SEED_C4, read_len=150, median=90, sigma=0.5,
             insert_lo=40, insert_hi=600, p_adapter=0.01, p_sub=0.01, p_ins=0.001,
             p_del=0.001, chunk=8192):
    """Read pairs of 2 x read_len: a fragment (the insert, lognormal around
    `median`, clipped to [insert_lo, insert_hi]) from a random reference on
    a random template strand; mate 1 reads the fragment from its 5' end,
    mate 2 its reverse complement.  A mate longer than the insert reads on
    into its adapter (TRUSEQ_R1 / _R2 with p_adapter substitutions, random
    bases past the adapter's end).  A fragment longer than its reference
    gets random flanks.  Each mate then takes p_sub substitutions and
    p_ins + p_del indels and is cut or padded back to read_len.  Built in
    chunks of `chunk` pairs (generator seeded by (seed, chunk index)).
    Returns a Packed of 2n reads, mate 1 of pair p at 2p, mate 2 at 2p + 1,
    and the inserts."""
    codes, inserts = [], []
    for c0 in range(0, n, chunk):
        rng = np.random.default_rng([seed, c0 // chunk])
        cc, ins = _pairs_chunk(rng, refs, min(chunk, n - c0), read_len, median, sigma,
                               insert_lo, insert_hi, p_adapter, p_sub, p_ins, p_del)
        codes.append(cc)
        inserts.append(ins)
    codes = np.concatenate(codes) if codes else np.zeros(0, np.uint8)
    ins = np.concatenate(inserts) if inserts else np.zeros(0, np.int64)
    lens = np.full(2 * n, read_len, dtype=np.uint32)
    return Packed(codes, _offsets(lens), lens), ins


def _pairs_chunk(rng, refs, n, read_len, median, sigma, insert_lo, insert_hi, p_adapter, p_sub,
                 p_ins, p_del):
    from .alphabet import encode

    ref_lens = np.array([r.size for r in refs], dtype=np.int64)
    ref_off = _offsets(ref_lens).astype(np.int64)
    cat = np.concatenate(refs)
    which = rng.integers(0, len(refs), n)
    rev = rng.random(n) < 0.5
    ins = lognormal_lengths(rng, n, median, sigma, insert_lo, insert_hi)
    rl = ref_lens[which]
    # fragment: a window of the reference, or the reference inside random flanks
    span = np.minimum(ins, rl)
    s_ref = rng.integers(0, np.maximum(rl - ins, 0) + 1)
    s_dst = rng.integers(0, np.maximum(ins - rl, 0) + 1)
    frag_off = _offsets(ins).astype(np.int64)
    frag = random_bases(rng, int(ins.sum()))
    frag[_ranges(frag_off + s_dst, span)] = cat[_ranges(ref_off[which] + s_ref, span)]
    # template strand
    if rev.any():
        idx = np.nonzero(rev)[0]
        sel = _ranges(frag_off[idx], ins[idx])
        frag[sel] = _seg_revcomp(frag, frag_off[idx], ins[idx])
    frag_rc = _seg_revcomp(frag, frag_off, ins)
    mates = []
    for src, adapter in ((frag, TRUSEQ_R1), (frag_rc, TRUSEQ_R2)):
        m = random_bases(rng, n * read_len)
        m_off = np.arange(n, dtype=np.int64) * read_len
        body = np.minimum(ins, read_len)
        m[_ranges(m_off, body)] = src[_ranges(frag_off, body)]
        ad = encode(adapter)
        short = np.nonzero(ins < read_len)[0]
        if short.size:
            k = np.minimum(read_len - ins[short], ad.size)
            pos = _ranges(m_off[short] + ins[short], k)
            a = ad[_ranges(np.zeros(short.size, dtype=np.int64), k)].copy()
            err = rng.random(a.size) < p_adapter
            a[err] = (a[err] + rng.integers(1, 4, int(err.sum()))) % 4
            m[pos] = a
        mc, ml = mutate(rng, m, np.full(n, read_len, dtype=np.int64), p_sub, p_ins, p_del)
        mates.append(_fix_length(rng, mc, ml, read_len).reshape(n, read_len))
    return np.stack(mates, axis=1).reshape(-1), ins
