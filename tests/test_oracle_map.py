"""The oracle's mapping stage pinned on the reference's own answers:
MD / NM against the samtools calmd records of calmd_golden.json (checked in
the reference by tests/sam_fields.rs) and sam.rs's unit case, and
map_reads against the known answers of mapper.rs's unit tests (556-760)."""
import json
import os
import re

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "calmd_golden.json")
SCHEME = (2, -1, -10, -1)  # Scoring::default (scoring.rs:38-49)
PANEL = [b"GGGGACGTACGTACGTTTTT", b"CCCCACGTACGTACGTAAAA", b"TTTTTTTTTTTTTTTTTTTT"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    O.build()


def parse_cigar(s):
    """A SAM CIGAR into (leading clip, BAM words, trailing clip)."""
    lead = tail = 0
    words = []
    for n, op in re.findall(r"(\d+)([MIDS])", s):
        n = int(n)
        if op == "S":
            if words:
                tail = n
            else:
                lead = n
        else:
            words.append((n << 4) | "MID".index(op))
    return lead, words, tail


def test_md_nm_matches_samtools_calmd():
    g = json.load(open(GOLDEN))
    ref = g["reference"].encode()
    names = {r["name"] for r in g["records"]}
    assert {"n_under_read_base", "n_under_read_n", "n_inside_deletion"} <= names
    for r in g["records"]:
        lead, words, _ = parse_cigar(r["cigar"])
        md, nm = O.md_nm(r["seq"].encode(), ref, lead, r["pos"] - 1, words)
        assert (md, nm) == (r["md"], r["nm"]), r["name"]


def test_md_nm_reference_n_is_a_mismatch():
    # sam.rs:134-140
    assert O.md_nm(b"ACGTAACGTA", b"ACGTANCGTA", 0, 0, [10 << 4]) == ("5N4", 1)


def test_ties_in_reference_order():
    # mapper.rs:569-590
    m = O.map_reads([b"ACGTACGTACGT"], PANEL, SCHEME, True)[0]
    assert m["best_score"] == 24 and m["n_tied"] == 2
    assert [h["reference"] for h in m["hits"]] == [0, 1]
    assert m["suboptimal"] < 24
    c = O.map_reads([b"ACGTACGTACGT"], PANEL, SCHEME, True, max_ties=0)[0]
    assert c["n_tied"] == 2 and len(c["hits"]) == 1


def test_min_score_unmaps():
    # mapper.rs:725-737
    m = O.map_reads([b"ACGTACGTACGT"], PANEL, SCHEME, True, min_score=1000)[0]
    assert m["hits"] == [] and m["best_score"] == 24


def test_reverse_strand_found_when_asked():
    # mapper.rs:739-758
    read = O.revcomp_letters(b"CGTACGTAAAA")
    fwd = O.map_reads([read], PANEL, SCHEME, True)[0]
    both = O.map_reads([read], PANEL, SCHEME, True, both_strands=True)[0]
    assert both["best_score"] > fwd["best_score"]
    h = both["hits"][0]
    assert h["reference"] == 1 and h["reverse"] and h["md"] == "11"


def test_empty_and_wildcard_reads():
    # the reads of mapper.rs:593-617: an empty read has no best; NNNN scores
    # (wildcards match) but its MD counts every base a mismatch
    ms = O.map_reads([b"", b"NNNN"], PANEL, SCHEME, True, both_strands=True)
    assert ms[0] == {"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []}
    assert ms[1]["best_score"] == 8 and ms[1]["hits"]
    assert ms[1]["hits"][0]["nm"] == 4


def _fixture_pairs():
    """The reference's paired fixture, mates trimmed of their adapters as the
    CLI does before map_pairs_scored (align.rs:2844-2863)."""
    from tests.helpers import pairs_fixture
    names, refs, pairs = pairs_fixture()
    mates = [m for p in pairs.values() for m in p]
    trimmed, _ = O.trim_pairs(mates)
    L = lambda c: bytes(b"ACGTN"[min(int(x), 4)] for x in c)  # noqa: E731
    return (names, [L(r) for r in refs], list(pairs),
            [(L(trimmed[2 * i]), L(trimmed[2 * i + 1])) for i in range(len(pairs))])


def test_map_pairs_fixture_answers():
    """What the reference's tests/align_paired.rs pins for the fixture with
    --min-score 40, semi-global (the paired default)."""
    names, refs, pnames, pairs = _fixture_pairs()
    by = lambda res: dict(zip(pnames, res))  # noqa: E731
    roomy = by(O.map_pairs(pairs, refs, SCHEME, False, min_score=40))
    wide = by(O.map_pairs(pairs, refs, SCHEME, False, min_score=40, max_insert=120))
    p = roomy["paralog"]  # unique on P1, mate-1 XS equal to its AS
    assert p["proper"] and p["n_tied"] == 1 and names[p["hits"][0]["reference"]] == "P1"
    assert p["suboptimal"][0] == p["hits"][0]["mates"][0]["score"]
    t = roomy["pair_tie"]  # the P1 / P2 tie
    assert t["proper"] and [names[h["reference"]] for h in t["hits"]] == ["P1", "P2"]
    tm = roomy["terminal_mismatch"]  # kept end to end, 117 + 117
    assert [m["score"] for m in tm["hits"][0]["mates"]] == [117, 117]
    assert roomy["over_max_insert"]["proper"] and roomy["over_max_insert"]["hits"][0]["insert"] == 150
    o = wide["over_max_insert"]  # each mate at its own best (U1), mate 2 reversed
    assert not o["proper"]
    assert [(names[m["hits"][0]["reference"]], m["hits"][0]["reverse"]) for m in o["mates"]] == \
        [("U1", False), ("U1", True)]
    w = roomy["wrong_orientation"]  # both forward on U2, not proper
    assert not w["proper"]
    assert [(names[m["hits"][0]["reference"]], m["hits"][0]["reverse"]) for m in w["mates"]] == \
        [("U2", False), ("U2", False)]
    u = roomy["one_unmapped"]  # the junk mate is unmapped
    assert not u["proper"] and u["mates"][0]["hits"] and not u["mates"][1]["hits"]


def test_md_nm_in_c_matches_samtools_calmd():
    """eo_md_nm (the C restatement the CPU mapping baseline runs) on codes,
    with the reference letters, against the same calmd records."""
    g = json.load(open(GOLDEN))
    ref = g["reference"].encode()
    rc = O.encode(ref)
    for r in g["records"]:
        lead, words, _ = parse_cigar(r["cigar"])
        q = O.encode(r["seq"])
        n_q = sum(w >> 4 for w in words if w & 0xf in (0, 1))
        n_r = sum(w >> 4 for w in words if w & 0xf in (0, 2))
        a = (0, lead, lead + n_q, r["pos"] - 1, r["pos"] - 1 + n_r, len(words))
        assert O.md_nm_codes(q, False, rc, ref, a, words) == (r["md"], r["nm"]), r["name"]


@pytest.mark.parametrize("local", [True, False])
def test_cpu_mapper_equals_the_restatement(local):
    """The C-composed CPU mapper (AVX-512 scores, scalar traceback, C MD/NM)
    gives map_reads' dicts exactly, tie lists from full rows included."""
    if not O.lib().eo_cpu_has_avx512bw():
        pytest.skip("no AVX-512BW on this host")
    from tests.helpers import Rng, mutate, random_seq
    panel = [b"GGGGACGTACGTACGTTTTT", b"CCCCACGTACGTACGTAAAA", b"TTTTTTTTTTTTTTTTTTTT"]
    panel += [b"A" * (20 + k) for k in range(12)] + [b"ACGTNACGTRACGU" * 3]
    rng = Rng(0x5EED_0905)
    reads = [b"ACGTACGTACGT", b"", b"NNNN", b"CCCCCCCC", b"AAAAAAAAAAAA"]
    reads += [mutate(rng, p[2:]) for p in panel] + [random_seq(rng, 30, 0.05) for _ in range(10)]
    codes, off, lens = O.pack([O.encode(r) if len(r) else np.zeros(0, np.uint8) for r in reads])
    refs = [O.encode(p) for p in panel]
    for both, max_ties, min_score, cap in ((True, None, 0, 2), (False, 0, 10, 8),
                                           (True, 3, 0, 32)):
        got = O.cpu_mappings(*O.cpu_map_reads(codes, off, lens, refs, SCHEME, local,
                                              min_score=min_score, max_ties=max_ties,
                                              both_strands=both, ref_letters=panel,
                                              cap=cap)[:6])
        want = O.map_reads(reads, panel, SCHEME, local, min_score=min_score,
                           max_ties=max_ties, both_strands=both)
        assert got == want


@pytest.mark.parametrize("local", [False, True])
def test_cpu_pair_mapper_equals_the_restatement(local):
    """The C-composed CPU paired mapper gives map_pairs' dicts exactly: the
    paired fixture under align_paired.rs's options and synthetic pairs whose
    first tiers fail (tight max insert) or outrun a small capacity."""
    if not O.lib().eo_cpu_has_avx512bw():
        pytest.skip("no AVX-512BW on this host")
    from eschalign_b200 import synth
    names, refs, pnames, pairs = _fixture_pairs()
    cases = [(refs, pairs)]
    panel = synth.panel_tiles()
    P, _ = synth.pairs_c4(panel, n=120, seed=0x5EED_0A02)
    trimmed, _ = O.trim_pairs([P.read(k) for k in range(len(P))])
    L = lambda c: bytes(b"ACGTN"[min(int(x), 4)] for x in c)  # noqa: E731
    cases.append(([L(r) for r in panel],
                  [(L(trimmed[2 * i]), L(trimmed[2 * i + 1])) for i in range(len(P) // 2)]
                  + [(b"", b"ACGTACGT")]))
    for letters, prs in cases:
        rc = [O.encode(x) for x in letters]
        codes, off, lens = O.pack([O.encode(m) if len(m) else np.zeros(0, np.uint8)
                                   for p in prs for m in p])
        for min_score, max_insert, both, cap in ((40, 500, False, 8), (40, 120, True, 2),
                                                 (20, 45, True, 1), (0, 500, True, 32)):
            got, _ = O.cpu_map_pairs(codes, off, lens, rc, SCHEME, local, min_score=min_score,
                                     max_insert=max_insert, both_strands=both,
                                     ref_letters=letters, cap=cap)
            want = O.map_pairs(prs, letters, SCHEME, local, min_score=min_score,
                               max_insert=max_insert, both_strands=both)
            assert got == want, (min_score, max_insert, both, cap)


def test_cpu_pair_mapper_trims_like_the_cli():
    """trim=True (adapters found by the C ranking call) maps the same pairs
    as trimming first with the restated pair_adapters."""
    if not O.lib().eo_cpu_has_avx512bw():
        pytest.skip("no AVX-512BW on this host")
    from eschalign_b200 import synth
    panel = synth.panel_tiles()
    P, _ = synth.pairs_c4(panel, n=300, seed=0x5EED_0A03)
    raw = [P.read(k) for k in range(len(P))]
    trimmed, _ = O.trim_pairs(raw)
    a, _ = O.cpu_map_pairs(*O.pack(raw), panel, SCHEME, False, min_score=40, both_strands=True,
                           trim=True)
    b, _ = O.cpu_map_pairs(*O.pack(trimmed), panel, SCHEME, False, min_score=40,
                           both_strands=True)
    assert a == b
