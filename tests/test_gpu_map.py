"""Mapping on the CUDA path (esg_map_reads) against the oracle's
map_reads_scored restatement (crates/eschalign/src/mapper.rs:400-552 with
sam.rs:55-121's MD / NM): per read the best score, tie count, XS and every
traced hit -- reference, strand, score, coordinates, CIGAR, MD, NM -- equal
field for field."""
import json
import os

import numpy as np
import pytest

from eschalign_b200 import GpuScorer, Mode, Scoring, encode, synth
from tests.helpers import GOLDEN, Rng, golden, mutate, random_seq

pytestmark = pytest.mark.gpu

SCHEME = (2, -1, -10, -1)
# the panel and reads of mapper.rs's unit tests (556-620)
UNIT_PANEL = [b"GGGGACGTACGTACGTTTTT", b"CCCCACGTACGTACGTAAAA", b"TTTTTTTTTTTTTTTTTTTT"]
UNIT_READS = [b"ACGTACGTACGT", b"CCCCACGTACGTACGTAAAA", b"TTTTTTTTTTTT", b"",
              b"GGGGACGTACGTACGTTTTT", b"NNNN"]


def code_letters(codes):
    return bytes(b"ACGTN"[min(int(c), 4)] for c in codes)


def panel_letters(tag):
    with open(os.path.join(GOLDEN, f"panel_{tag}.json")) as fh:
        return [r["seq"].encode() for r in json.load(fh)["references"]]


def run(oracle, panel, reads, scoring, mode, cap=8, give_letters=True, **opts):
    codes = [encode(p) for p in panel]
    with GpuScorer(codes, Scoring(*scoring), mode, tie_capacity=cap) as g:
        got = g.map_reads([encode(r) if len(r) else np.zeros(0, np.uint8) for r in reads],
                          ref_letters=panel if give_letters else None, **opts)
    want = oracle.map_reads(reads, panel if give_letters else [code_letters(c) for c in codes],
                            scoring, mode == Mode.LOCAL, **opts)
    assert len(got) == len(want)
    for k, w in enumerate(want):
        assert got.mapping(k) == w, (k, reads[k], opts, cap)
    return got, want


@pytest.mark.parametrize("mode", [Mode.LOCAL, Mode.SEMIGLOBAL])
def test_map_unit_panel(oracle, mode):
    for both in (False, True):
        for max_ties in (None, 0, 1):
            for min_score in (0, 20, 1000):
                run(oracle, UNIT_PANEL, UNIT_READS, SCHEME, mode, both_strands=both,
                    max_ties=max_ties, min_score=min_score)


def test_map_unit_answers(oracle):
    """mapper.rs:569-590, 739-758 through the CUDA path."""
    got, _ = run(oracle, UNIT_PANEL, [b"ACGTACGTACGT"], SCHEME, Mode.LOCAL)
    m = got.mapping(0)
    assert m["best_score"] == 24 and m["n_tied"] == 2
    assert [h["reference"] for h in m["hits"]] == [0, 1]
    read = oracle.revcomp_letters(b"CGTACGTAAAA")
    got, _ = run(oracle, UNIT_PANEL, [read], SCHEME, Mode.LOCAL, both_strands=True)
    h = got.mapping(0)["hits"][0]
    assert h["reference"] == 1 and h["reverse"] and h["md"] == "11"


@pytest.mark.parametrize("tag", ["trna", "trna_ambiguous"])
@pytest.mark.parametrize("mode", [Mode.LOCAL, Mode.SEMIGLOBAL])
def test_map_trna_panels(oracle, tag, mode):
    """The 47-reference tRNA panels (near-identical isodecoders: large tie
    sets; the ambiguous one carries N, an MD mismatch the scorer calls a
    match), the golden fixture reads and reads cut from the panel."""
    panel = panel_letters(tag)
    rng = Rng(0x5EED_0901)
    reads = [s.encode() for s in golden()["fixture_reads"]]
    for _ in range(120):
        r = panel[rng.below(len(panel))]
        a = rng.below(len(r) // 4 + 1)
        b = len(r) - rng.below(len(r) // 4 + 1)
        reads.append(random_seq(rng, rng.below(8), 0.0) + mutate(rng, r[a:max(b, a)]))
    reads.append(b"")
    for cap, max_ties, min_score, both in ((8, None, 0, True), (1, None, 0, True),
                                           (2, 3, 40, False), (32, 0, 0, True)):
        for give in (True, False):
            run(oracle, panel, reads, SCHEME, mode, cap=cap, give_letters=give,
                max_ties=max_ties, min_score=min_score, both_strands=both)


def test_map_letters_verbatim(oracle):
    """Reference letters in lower case, U and IUPAC codes: MD writes them
    upper-cased but otherwise verbatim, and counts each non-ACGT as a
    mismatch (sam.rs:17-27)."""
    panel = [b"ggggACGUACGTACGTRTTT", b"CCCCacgtacgtNCGTAAAA", b"TTTTTTTTYTTTTTTTTTTT"]
    reads = [b"ACGTACGTACGT", b"GGGGACGTACGTACGTATTT", b"CCCCACGTACGTACGTAAAA", b"TTTTTTTTTT",
             b"acgtNcgt"]
    for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
        got, want = run(oracle, panel, reads, SCHEME, mode, both_strands=True)
        assert any("R" in h["md"] or "N" in h["md"] or "U" in h["md"]
                   for w in want for h in w["hits"])


def test_map_c1_sample(oracle):
    """2000 reads of the C1 workload on the 164-reference panel, local,
    forward strand: a batch of the size the reference's feeder sends."""
    refs = synth.panel_tiles()
    data = synth.reads_c1(refs)
    reads = [code_letters(data.read(k)) for k in range(2000)]
    panel = [code_letters(r) for r in refs]
    got, want = run(oracle, panel, reads, SCHEME, Mode.LOCAL)
    assert sum(1 for w in want if w["hits"]) > 1500


def test_map_bad_arguments(oracle):
    codes = [encode(p) for p in UNIT_PANEL]
    with GpuScorer(codes, Scoring(*SCHEME), Mode.LOCAL) as g:
        with pytest.raises(ValueError):
            g.map_reads([encode(b"ACGT")], ref_letters=UNIT_PANEL[:2])
        with pytest.raises(ValueError):
            g.map_reads([encode(b"ACGT")], ref_letters=[b"ACGT"] * 3)
        m = g.map_reads([])
        assert len(m) == 0


def test_map_large_batch_equals_small_ones(oracle):
    """All 10 000 C1 reads in one call (the hits assembled on several host
    threads) equal the same reads mapped 2000 at a time, both strands."""
    refs = synth.panel_tiles()
    data = synth.reads_c1(refs)
    with GpuScorer(refs, Scoring(*SCHEME), Mode.LOCAL) as g:
        whole = g.map_reads(data.tuple(), both_strands=True)
        assert len(whole) == len(data)
        for k0 in range(0, len(data), 2000):
            part = g.map_reads(data.slice(k0, k0 + 2000).tuple(), both_strands=True)
            for k in range(len(part)):
                assert whole.mapping(k0 + k) == part.mapping(k), k0 + k


# ---------------------------------------------------------------- pairs
def fixture_pairs(oracle):
    """The reference's paired fixture, mates trimmed as the CLI trims them."""
    from tests.helpers import pairs_fixture
    names, refs, pairs = pairs_fixture()
    trimmed, _ = oracle.trim_pairs([m for p in pairs.values() for m in p])
    return ([code_letters(r) for r in refs],
            [(code_letters(trimmed[2 * i]), code_letters(trimmed[2 * i + 1]))
             for i in range(len(pairs))])


def run_pairs(oracle, panel, pairs, scoring, mode, cap=8, give_letters=True, **opts):
    codes = [encode(p) for p in panel]
    mates = [encode(m) if len(m) else np.zeros(0, np.uint8) for p in pairs for m in p]
    with GpuScorer(codes, Scoring(*scoring), mode, tie_capacity=cap) as g:
        got = g.map_pairs(mates, ref_letters=panel if give_letters else None, **opts)
    want = oracle.map_pairs(pairs, panel if give_letters else [code_letters(c) for c in codes],
                            scoring, mode == Mode.LOCAL, **opts)
    assert len(got) == len(want)
    for p, w in enumerate(want):
        assert got.pair_mapping(p) == w, (p, opts, cap)
    return got, want


@pytest.mark.parametrize("mode", [Mode.SEMIGLOBAL, Mode.LOCAL])
def test_map_pairs_fixture(oracle, mode):
    """The paired fixture under the options tests/align_paired.rs uses
    (--min-score 40, --max-insert 120 and the default 500) and more."""
    panel, pairs = fixture_pairs(oracle)
    for min_score, max_insert, both, cap, max_ties in ((40, 500, False, 8, None),
                                                       (40, 120, False, 8, None),
                                                       (0, 500, True, 1, None),
                                                       (40, 60, True, 2, 0)):
        run_pairs(oracle, panel, pairs, SCHEME, mode, cap=cap, min_score=min_score,
                  max_insert=max_insert, both_strands=both, max_ties=max_ties)


def test_map_pairs_fixture_answers(oracle):
    """What align_paired.rs pins, through the CUDA path."""
    from tests.helpers import pairs_fixture
    names, _, named = pairs_fixture()
    panel, pairs = fixture_pairs(oracle)
    by = dict(zip(named, range(len(pairs))))
    got, _ = run_pairs(oracle, panel, pairs, SCHEME, Mode.SEMIGLOBAL, min_score=40)
    p = got.pair_mapping(by["paralog"])
    assert p["proper"] and names[p["hits"][0]["reference"]] == "P1"
    assert p["suboptimal"][0] == p["hits"][0]["mates"][0]["score"]
    assert [names[h["reference"]] for h in got.pair_mapping(by["pair_tie"])["hits"]] == ["P1", "P2"]
    got, _ = run_pairs(oracle, panel, pairs, SCHEME, Mode.SEMIGLOBAL, min_score=40,
                       max_insert=120)
    o = got.pair_mapping(by["over_max_insert"])
    assert not o["proper"] and [m["hits"][0]["reverse"] for m in o["mates"]] == [False, True]


@pytest.mark.parametrize("mode", [Mode.SEMIGLOBAL, Mode.LOCAL])
def test_map_pairs_synthetic(oracle, mode):
    """C4-style pairs on the 164-reference panel (adapters trimmed): a tight
    max_insert makes first tiers fail and the pairs walk deeper tiers from
    full rows; a tie capacity of 1 sends every tied first tier there too."""
    refs = synth.panel_tiles()
    P, _ = synth.pairs_c4(refs, n=250, seed=0x5EED_0A01)
    trimmed, _ = oracle.trim_pairs([P.read(k) for k in range(len(P))])
    pairs = [(code_letters(trimmed[2 * i]), code_letters(trimmed[2 * i + 1]))
             for i in range(len(P) // 2)]
    pairs += [(b"", b"ACGTACGTAC"), (b"ACGT", b"")]
    panel = [code_letters(r) for r in refs]
    for max_insert, cap, both in ((500, 8, True), (70, 8, True), (45, 1, False)):
        run_pairs(oracle, panel, pairs, SCHEME, mode, cap=cap, min_score=20,
                  max_insert=max_insert, both_strands=both)


def test_map_zero_score_ties_and_saturation(oracle):
    """A read that matches nothing scores 0 locally against every candidate:
    all 2 x 20 candidates tie (more than the tie capacity, so the list comes
    from full rows), every trace is empty, and the read is unmapped with its
    best and tie count kept (mapper.rs:508-512).  Then scores far past int16
    (re-scored in int32 before tracing) under a large scheme."""
    panel = [b"A" * (20 + k) for k in range(20)]
    reads = [b"CCCCCCCC", b"AAAAAAAAAA", b""]
    for max_ties in (None, 3):
        got, want = run(oracle, panel, reads, SCHEME, Mode.LOCAL, both_strands=True,
                        max_ties=max_ties)
        m = got.mapping(0)
        assert m["best_score"] == 0 and m["n_tied"] == 40 and m["hits"] == []
    rng = Rng(0x5EED_0903)
    big = [random_seq(rng, 600 + 50 * k, 0.0) for k in range(6)]
    reads = [mutate(rng, r[50:]) for r in big] + [r[::-1] for r in big[:2]]
    for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
        got, want = run(oracle, big, reads, (100, -100, -27, -27), mode, both_strands=True)
        assert max(w["best_score"] for w in want) > 32767


def test_map_pipelined_call_equals_single_batches():
    """300 000 C2 reads in one call (scored in batches, each batch traced on
    its own stream while the next is scored) equal three single-batch calls
    of 100 000, array for array."""
    refs = synth.panel_tiles()
    data = synth.reads_c2(refs, n=300_000, seed=0x5EED_0907)
    with GpuScorer(refs, Scoring(*SCHEME), Mode.LOCAL) as g:
        whole = g.map_reads(data.tuple(), both_strands=True)
        parts = [g.map_reads(data.slice(k, k + 100_000).tuple(), both_strands=True)
                 for k in range(0, 300_000, 100_000)]
    fields = ("best_score", "suboptimal", "n_tied", "flags", "n_hits")
    for f in fields:
        assert (whole.reads[f] == np.concatenate([p.reads[f] for p in parts])).all(), f
    hf = ("reference", "reverse", "score", "query_start", "query_end", "ref_start", "ref_end",
          "n_ops", "nm", "md_len")
    for f in hf:
        assert (whole.hits[f] == np.concatenate([p.hits[f] for p in parts])).all(), f
    assert (whole.ops == np.concatenate([p.ops for p in parts])).all()
    assert whole.md_bytes == b"".join(p.md_bytes for p in parts)
    # offsets are consistent: each read's hits start where the previous ended
    fh = whole.reads["first_hit"].astype(np.int64)
    nh = whole.reads["n_hits"].astype(np.int64)
    assert (fh[1:] == fh[:-1] + nh[:-1]).all()


def test_map_pairs_large_batch_equals_small_ones():
    """20 000 trimmed C4 pairs in one call (the Proper pairs' hits assembled
    on several host threads) equal the same pairs mapped 2000 at a time."""
    from eschalign_b200 import adapter
    refs = synth.panel_tiles()
    P, _ = synth.pairs_c4(refs, n=20_000, seed=0x5EED_0A04)
    codes, off, _ = P.tuple()
    _, aligned = adapter.pair_adapters(P.tuple())
    with GpuScorer(refs, Scoring(*SCHEME), Mode.SEMIGLOBAL) as g:
        whole = g.map_pairs((codes, off, aligned), min_score=40, both_strands=True)
        assert len(whole) == 20_000
        for p0 in range(0, 20_000, 2000):
            part = g.map_pairs((codes, off[2 * p0:2 * p0 + 4000], aligned[2 * p0:2 * p0 + 4000]),
                               min_score=40, both_strands=True)
            for p in range(len(part)):
                assert whole.pair_mapping(p0 + p) == part.pair_mapping(p), p0 + p


def test_map_mid_sized_call_equals_small_ones():
    """50 000 C2 reads (the CLI's batch size) in one call equal five calls
    of 10 000, array for array."""
    refs = synth.panel_tiles()
    data = synth.reads_c2(refs, n=50_000, seed=0x5EED_0908)
    with GpuScorer(refs, Scoring(*SCHEME), Mode.LOCAL) as g:
        whole = g.map_reads(data.tuple(), both_strands=True)
        parts = [g.map_reads(data.slice(k, k + 10_000).tuple(), both_strands=True)
                 for k in range(0, 50_000, 10_000)]
    for f in ("best_score", "suboptimal", "n_tied", "flags", "n_hits"):
        assert (whole.reads[f] == np.concatenate([p.reads[f] for p in parts])).all(), f
    for f in ("reference", "reverse", "score", "query_start", "query_end", "ref_start",
              "ref_end", "n_ops", "nm", "md_len"):
        assert (whole.hits[f] == np.concatenate([p.hits[f] for p in parts])).all(), f
    assert (whole.ops == np.concatenate([p.ops for p in parts])).all()
    assert whole.md_bytes == b"".join(p.md_bytes for p in parts)


def test_map_two_scorers_on_two_threads():
    """align_bam's several mapping threads: two scorers over one panel, each
    mapping on its own thread at once, give what one thread gives, call for
    call."""
    from concurrent.futures import ThreadPoolExecutor
    refs = synth.panel_tiles()
    data = synth.reads_c2(refs, n=20_000, seed=0x5EED_0909)
    letters = [code_letters(r) for r in refs]
    chunks = [data.slice(k, k + 1000) for k in range(0, 20_000, 1000)]
    gs = [GpuScorer(refs, Scoring(*SCHEME), Mode.LOCAL) for _ in range(2)]
    try:
        want = [gs[0].map_reads(c.tuple(), both_strands=True, ref_letters=letters)
                for c in chunks]
        for _ in range(2):
            with ThreadPoolExecutor(2) as ex:
                got = list(ex.map(lambda k: gs[k % 2].map_reads(
                    chunks[k].tuple(), both_strands=True, ref_letters=letters),
                    range(len(chunks))))
            for g, w in zip(got, want):
                assert np.array_equal(g.reads, w.reads) and np.array_equal(g.hits, w.hits)
                assert np.array_equal(g.ops, w.ops) and g.md_bytes == w.md_bytes
    finally:
        for g in gs:
            g.close()
