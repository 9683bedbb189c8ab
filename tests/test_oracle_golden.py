"""The CPU oracle pinned against the reference's golden vectors and known
answers, and the AVX-512 baseline against the scalar oracle."""
import numpy as np
import pytest

from tests.helpers import SCHEMES, Rng, fixture_panel, fixture_reads, golden, random_panel, reads_for

D = (2, -1, -10, -1)


def test_scalar_matches_parasail_golden(oracle):
    """parasail_golden.rs:48-77: the 192 parasail 1.3.4 scores."""
    g = golden()
    assert len(g["cases"]) == 192
    for c in g["cases"]:
        q, r = oracle.encode(c["query"]), oracle.encode(c["reference"])
        got = oracle.score(q, r, c["scheme"], c["mode"] == "local")
        assert got == c["score"], (c["name"], c["mode"], c["scheme"])


def test_scalar_known_answers(oracle):
    """scalar.rs:378-430."""
    E = oracle.encode
    assert oracle.score(E("ACGTACGT"), E("TTACGTACGTTT"), D, True) == 16
    assert oracle.score(E("ACGTA"), E("ACNTA"), D, True) == 10
    assert oracle.score(E("AAAACCCGGGGTTTT"), E("AAAACCCCGGGGTTTT"), (2, -4, -3, -1), True) == 27
    assert oracle.score(E("ACGTACGTCCCCC"), E("GGGGGACGTACGT"), D, False) == 16
    assert oracle.score(E("AAAA"), E("CCCC"), D, True) == 0
    assert oracle.score(E(""), E("ACGT"), D, True) == 0


def test_alphabet_and_scoring(oracle):
    """alphabet.rs:513-537, scoring.rs:192-213."""
    assert list(oracle.encode("ACGTUacgtu")) == [0, 1, 2, 3, 3, 0, 1, 2, 3, 3]
    assert all(v == 4 for v in oracle.encode("NnRYKMSWBDHV-*.X"))
    assert list(oracle.revcomp(oracle.encode("ACGTN"))) == list(oracle.encode("NACGT"))
    assert oracle.validate(D) == 0
    assert oracle.validate((0, -1, -10, -1)) != 0
    assert oracle.validate((2, 3, -10, -1)) != 0
    assert oracle.validate((2, -1, 10, -1)) != 0
    assert oracle.validate((2, -1, -1001, -1)) != 0
    assert oracle.fits_i16(5000, 200, D)
    assert not oracle.fits_i16(20000, 20000, D)


def test_gap_convention(oracle):
    """scoring.rs:199-204: gap(1) = -10, gap(3) = -12 at 2,-1,-10,-1 -- seen
    through the score of a read that is its reference less 1 or 3 bases:
    matches * 2 + open + (k - 1) * extend, end to end."""
    from tests.helpers import Rng, random_seq
    ref = oracle.encode(random_seq(Rng(0x5EED_6A9), 60, 0.0))
    for k, gap in ((1, -10), (3, -12)):
        q = np.concatenate([ref[:30], ref[30 + k:]])
        assert oracle.score(q, ref, D, local=False) == 2 * (60 - k) + gap


def test_tie_selection_known_answers(oracle):
    """mapper.rs:570-589: two ties in reference order, XS below the best."""
    E = oracle.encode
    panel = [E("GGGGACGTACGTACGTTTTT"), E("CCCCACGTACGTACGTAAAA"), E("TTTTTTTTTTTTTTTTTTTT")]
    q = E("ACGTACGTACGT")
    fwd = [oracle.score(q, r, D, True) for r in panel]
    best, sub, n_tied, flags, ties = oracle.select(fwd, None, cap=8)
    assert best == 24 and n_tied == 2 and ties == [0 << 1, 1 << 1] and sub < 24
    # mapper.rs:722-739: the reverse strand wins when it scores higher
    read = oracle.revcomp(E("CGTACGTAAAA"))
    f = [oracle.score(read, r, D, True) for r in panel]
    rv = [oracle.score(oracle.revcomp(read), r, D, True) for r in panel]
    b2, _, n2, _, t2 = oracle.select(f, rv)
    assert b2 > max(f) and t2[0] == (1 << 1) | 1
    # every candidate tied: no suboptimal
    b3, s3, n3, fl3, t3 = oracle.select([5, 5, 5], [5, 5, 5], cap=2)
    assert (b3, s3, n3) == (5, oracle.NO_SCORE, 6) and fl3 & oracle.RESULT_TIES_TRUNCATED
    assert t3 == [0, 1]


@pytest.mark.parametrize("scoring", SCHEMES)
def test_avx512_equals_scalar(oracle, scoring):
    """simd/mod.rs:752-810 / 917-1002: both loop orders and the dispatch,
    by equality, on a ragged 37-reference panel."""
    rng = Rng(0x5EED_0002)
    letters = random_panel(rng, 37, 20, 280)
    panel = [oracle.encode(s) for s in letters]
    reads = reads_for(rng, letters, 16)
    reads.append(oracle.encode(b"ACGT" * 80))  # >= 256 nt: the transposed kernel
    prof = oracle.Profile(panel, scoring)
    for local in (True, False):
        want = oracle.score_matrix(reads, panel, scoring, local)
        for k, q in enumerate(reads):
            for kernel in (0, 1, 2):
                got = prof.score_all(q, local, kernel)
                assert (got == want[k]).all(), (scoring, local, kernel, len(q))


def test_avx512_on_fixture_panels(oracle):
    """simd/mod.rs:817-863: the tRNA fixture reads against both panels."""
    reads = fixture_reads()
    assert len(reads) >= 5
    for tag in ("trna", "trna_ambiguous"):
        panel = fixture_panel(tag)
        assert len(panel) == 47
        for scoring in SCHEMES:
            prof = oracle.Profile(panel, scoring)
            for local in (True, False):
                want = oracle.score_matrix(reads, panel, scoring, local)
                for k, q in enumerate(reads):
                    assert (prof.score_all(q, local) == want[k]).all()


def test_cpu_batch_equals_scalar_batch(oracle):
    rng = Rng(0x5EED_0101)
    letters = random_panel(rng, 37, 20, 280)
    panel = [oracle.encode(s) for s in letters]
    reads = reads_for(rng, letters, 30) + [np.zeros(0, np.uint8)]
    prof = oracle.Profile(panel, D)
    codes, off, lens = oracle.pack(reads)
    for local in (True, False):
        for both in (False, True):
            a, ta, ra, _ = prof.map_batch(codes, off, lens, local, both, cap=4, rows=True)
            b, tb, rb = oracle.scalar_map_batch(reads, panel, D, local, both, cap=4, rows=True)
            assert (a == b).all() and (ta == tb).all() and (ra == rb).all()


def test_align_matches_parasail_golden(oracle):
    """parasail_golden.rs:48-110 on the oracle's traceback: the 192 golden
    cases' scores and coordinates (query_start, query_end, ref_start,
    ref_end), and ops that re-score to the score, span the coordinates and
    start and end with M."""
    for c in golden()["cases"]:
        q, r = oracle.encode(c["query"]), oracle.encode(c["reference"])
        local = c["mode"] == "local"
        a, ops = oracle.align(q, r, tuple(c["scheme"]), local)
        label = (c["name"], c["mode"], c["scheme"])
        assert int(a["score"]) == c["score"], label
        assert oracle.score(q, r, tuple(c["scheme"]), local) == c["score"], label
        assert (int(a["query_start"]), int(a["query_end"]), int(a["ref_start"]),
                int(a["ref_end"])) == (c["query_start"], c["query_end"], c["ref_start"],
                                       c["ref_end"]), label
        assert oracle.rescore(q, r, a, ops, tuple(c["scheme"])) == c["score"], label
        qs = sum(int(w) >> 4 for w in ops if int(w) & 0xf in (0, 1))
        rs = sum(int(w) >> 4 for w in ops if int(w) & 0xf in (0, 2))
        assert qs == a["query_end"] - a["query_start"] and rs == a["ref_end"] - a["ref_start"]
        if len(ops):
            assert int(ops[0]) & 0xf == 0 and int(ops[-1]) & 0xf == 0, label


def test_align_known_answers(oracle):
    """scalar.rs:378-430."""
    E = oracle.encode
    a, ops = oracle.align(E("ACGTACGT"), E("TTACGTACGTTT"), D, True)
    assert (a["score"], a["query_start"], a["query_end"], a["ref_start"], a["ref_end"]) == \
        (16, 0, 8, 2, 10) and oracle.cigar_string(ops) == "8M"
    s = (2, -4, -3, -1)
    a, ops = oracle.align(E("AAAACCCGGGGTTTT"), E("AAAACCCCGGGGTTTT"), s, True)
    assert a["score"] == 15 * 2 - 3 and "1D" in oracle.cigar_string(ops)
    a, ops = oracle.align(E("ACGTACGTCCCCC"), E("GGGGGACGTACGT"), D, False)
    assert (a["score"], a["ref_start"], a["ref_end"], a["query_start"], a["query_end"]) == \
        (16, 5, 13, 0, 8)
    a, ops = oracle.align(E("AAAA"), E("CCCC"), D, True)
    assert a["score"] == 0 and len(ops) == 0
