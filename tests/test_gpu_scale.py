"""Parity at the sizes that are timed.

The reference's own harness compares every pair it scores
(crates/eschalign/tests/gpu_parity.rs:151-192).  Here the whole C2 workload
-- all 1 000 000 reads, both strands, against the 164-reference panel -- is
scored on the GPU and every read's best score, XS, tie count and tie list is
compared with the reference's CPU path (the AVX-512BW restatement with its
scalar fallback, itself equal to the scalar oracle by test), for the
headline local scheme and for semi-global.  The uneven C3 panel (10 000
references of 300-1000 nt, read through L2 in panel chunks) gets a sample of
its reads on both strands, and a large-score scheme on a slice of it that
drives long reads past int16 so the re-score path runs at that shape."""
import numpy as np
import pytest

from eschalign_b200 import GpuScorer, Mode, Scoring, synth

pytestmark = pytest.mark.gpu

CAP = 8


@pytest.fixture(scope="module")
def c2():
    refs = synth.panel_tiles()
    return refs, synth.reads_c2(refs, n=1_000_000)


@pytest.fixture(scope="module")
def c3_panel():
    return synth.panel_c3()


def assert_same(got, got_ties, want, want_ties, cap, what):
    for f in ("best", "suboptimal", "n_tied"):
        bad = np.nonzero(got[f] != want[f])[0]
        assert bad.size == 0, (f"{what}: {f} differs on {bad.size} reads, first read "
                               f"{bad[0]}: got {got[f][bad[0]]} want {want[f][bad[0]]}")
    assert ((got["flags"] & 3) == (want["flags"] & 3)).all(), what
    n_l = np.minimum(want["n_tied"], cap)
    mask = np.arange(cap)[None, :] < n_l[:, None]
    bad = np.nonzero((got_ties != want_ties) & mask)[0]
    assert bad.size == 0, f"{what}: tie lists differ on {np.unique(bad).size} reads"


@pytest.mark.parametrize("mode", [Mode.LOCAL, Mode.SEMIGLOBAL])
def test_gpu_c2_every_read_equals_cpu_path(oracle, c2, mode):
    """All 1 000 000 C2 reads, both strands, 2,-1,-10,-1: the GPU's per-read
    results equal the CPU path's, read for read."""
    refs, reads = c2
    local = mode == Mode.LOCAL
    scoring = (2, -1, -10, -1)
    with GpuScorer(refs, Scoring(*scoring), mode) as g:
        g.autotune()
        res = g.score_batch(reads.tuple(), both_strands=True)
    assert res.stats["queries_batched"] == 2 * len(reads)
    want, want_t, _, _ = oracle.Profile(refs, scoring).map_batch(
        *reads.tuple(), local=local, both_strands=True, cap=CAP)
    assert_same(res.results, res.ties, want, want_t, CAP, f"C2 1M {mode.label}")


def test_gpu_c3_sample_on_the_full_panel(oracle, c3_panel):
    """200 C3 reads (50-1000 nt) against all 10 000 references, local
    2,-1,-10,-1, both strands: the panel is read through L2 and a small
    batch is cut into panel chunks whose states are merged."""
    refs = c3_panel
    reads = synth.reads_c3(refs, n=200)
    scoring = (2, -1, -10, -1)
    with GpuScorer(refs, Scoring(*scoring), Mode.LOCAL) as g:
        info = g.info()
        res = g.score_batch(reads.tuple(), both_strands=True)
    assert info["panel_bytes"] == 0  # too large for shared memory
    assert res.stats["panel_chunks"] > 1
    want, want_t, _, _ = oracle.Profile(refs, scoring).map_batch(
        *reads.tuple(), local=True, both_strands=True, cap=CAP)
    assert_same(res.results, res.ties, want, want_t, CAP, "C3 sample")


@pytest.mark.parametrize("mode", [Mode.LOCAL, Mode.SEMIGLOBAL])
def test_gpu_c3_shape_saturating_scheme(oracle, c3_panel, mode):
    """The C3 shape with a scheme whose long exact matches leave int16
    (100,-100,-27,-27: a 500-nt match scores 50 000): the batched kernel
    takes the queries, flags those that may have wrapped, the int32 lanes
    re-score them, and every result equals the scalar oracle's."""
    refs = c3_panel[:400]
    reads = synth.reads_c3(refs, n=24, seed=0x5EED_0C3F)
    scoring = (100, -100, -27, -27)
    with GpuScorer(refs, Scoring(*scoring), mode) as g:
        res = g.score_batch(reads.tuple(), both_strands=True)
    if mode == Mode.LOCAL:
        assert res.stats["queries_batched"] == 2 * len(reads)
    else:  # reads past the semi-global gap floor's bound go to the int32 lanes
        assert 0 < res.stats["queries_batched"] < 2 * len(reads)
    assert res.stats["queries_rescored"] > 0
    want, want_t, _ = oracle.scalar_map_batch(reads.list(), refs, scoring, mode == Mode.LOCAL,
                                              True, cap=CAP)
    assert_same(res.results, res.ties, want, want_t, CAP, f"C3 saturating {mode.label}")


def test_bam_run_at_scale_equals_the_oracle(c2, tmp_path):
    """The unpaired BAM run on 100 000 C2 reads (an unaligned BAM in, both
    strands, every tie traced, MD from the panel's letters, two scorers)
    against the oracle's: the CPU mapping stage (AVX-512 scores and ties,
    scalar traceback, MD / NM, all in C) and its restatement of the CLI's
    record building -- the output record stream byte for byte."""
    from eschalign_b200 import bam as EB
    from oracle import bam as B
    from oracle import oracle as O
    from tests.test_bam_pairs import bgzf
    refs, reads = c2
    sub = reads.slice(0, 100_000)
    names = [f"ref{k}" for k in range(len(refs))]
    letters = [bytes(b"ACGTN"[int(c)] for c in r) for r in refs]
    rng = np.random.default_rng(5)
    recs = []
    for k in range(len(sub)):
        seq = bytes(b"ACGTN"[int(c)] for c in sub.read(k))
        qual = rng.integers(2, 41, len(seq), dtype=np.uint8).tobytes()
        recs.append(B.encode_record(-1, -1, 0, [], 4, b"r%06d" % k, seq, qual,
                                    [B.str_field(b"RG", "grp1")]))
    src, dst = str(tmp_path / "in.bam"), str(tmp_path / "out.bam")
    with open(src, "wb") as fh:
        fh.write(bgzf(b"BAM\1" + bytes(8) + b"".join(recs)))
    srt = str(tmp_path / "sorted.bam")
    gs = [GpuScorer(refs, Scoring(2, -1, -10, -1), Mode.LOCAL) for _ in range(2)]
    try:
        n = EB.align_bam(gs, src, dst, names, letters, both_strands=True, secondary=True)
        EB.align_bam(gs, src, srt, names, letters, both_strands=True, secondary=True,
                     sort_coordinate=True)
    finally:
        for g in gs:
            g.close()
    from tests.test_bam_fastx import split_records
    from tests.test_bam_native import record_stream
    got = record_stream(dst)
    res, jobs, al, ops, mds, nm, _ = O.cpu_map_reads(
        *sub.tuple(), refs, (2, -1, -10, -1), True, both_strands=True,
        ref_letters=letters)
    maps = O.cpu_mappings(res, jobs, al, ops, mds, nm)
    _, _, inputs = B.read_bam(open(src, "rb").read())
    want = b"".join(x for r, m in zip(inputs, maps) for x in B.build_records(r, m, names, True))
    assert n["reads"] == len(sub)
    assert got == want
    # and coordinate-sorted: the CLI's stable sort (align.rs:2406-2450)
    assert record_stream(srt) == b"".join(B.coordinate_order(split_records(want)))


def test_paired_bam_run_at_scale_equals_the_oracle(tmp_path):
    """The paired BAM run on 20 000 C4 pairs (two FASTQ files, TruSeq
    adapters trimmed, semi-global, --min-score 40, two scorers) against the
    oracle's: its pair reader and adapter search, its C-composed paired
    mapping stage and its restatement of build_pair_records -- the output
    record stream byte for byte."""
    from eschalign_b200 import bam as EB
    from oracle import bam as B
    from oracle import oracle as O
    from tests.test_bam_native import record_stream
    refs = synth.panel_tiles()
    pairs, _ = synth.pairs_c4(refs, n=20_000, seed=0x5EED_0912)
    names = [f"ref{k}" for k in range(len(refs))]
    letters = [bytes(b"ACGTN"[int(c)] for c in r) for r in refs]
    rng = np.random.default_rng(6)
    texts = [[], []]
    for p in range(len(pairs) // 2):
        for m in range(2):
            seq = bytes(b"ACGTN"[int(c)] for c in pairs.read(2 * p + m)).decode()
            q = "".join(chr(33 + int(x)) for x in rng.integers(2, 41, len(seq)))
            texts[m].append(f"@p{p}\n{seq}\n+\n{q}\n")
    t1, t2 = "".join(texts[0]).encode(), "".join(texts[1]).encode()
    p1, p2, dst = str(tmp_path / "r1.fq"), str(tmp_path / "r2.fq"), str(tmp_path / "o.bam")
    open(p1, "wb").write(t1)
    open(p2, "wb").write(t2)
    scoring = (2, -1, -10, -1)
    gs = [GpuScorer(refs, Scoring(*scoring), Mode.SEMIGLOBAL) for _ in range(2)]
    try:
        n = EB.align_pairs_bam(gs, p1, p2, dst, names, letters, min_score=40, secondary=True)
    finally:
        for g in gs:
            g.close()
    got = record_stream(dst)
    recs = B.read_pairs(t1, t2)
    ads, mates = [], []
    for a, b in recs:
        ad = O.pair_adapters(a["seq"], b["seq"], max_read_len=1000)
        ads.append(ad)
        mates += [a["seq"][:len(a["seq"]) - ad[0]], b["seq"][:len(b["seq"]) - ad[1]]]
    from eschalign_b200 import pack_reads, encode
    codes, off, lens = pack_reads([encode(m) for m in mates])
    pms, _ = O.cpu_map_pairs(codes, off, lens, refs, scoring, False, min_score=40,
                             ref_letters=letters)
    want = b"".join(x for (a, b), pm, ad in zip(recs, pms, ads)
                    for x in B.build_pair_records([a, b], pm, ad, names, True))
    assert n["reads"] == len(pairs) and got == want
