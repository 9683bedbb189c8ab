"""Paired-end inputs and candidate ranking, on the CPU.

* The oracle's adapter search against the reference's own known answers
  (crates/eschalign/src/adapter.rs:117-197) and the paired fixture's adapter
  counts (crates/eschalign-cli/tests/align_paired.rs:303-340).
* The library's host-side trimming (esg_pair_adapters, the code
  esg_prepare_pairs runs) against the oracle on synthetic read-through pairs.
* The oracle's pair ranking (pair.rs:195-234, :297-314) against a spelled-out
  sort, and on the paired fixture against what align_paired.rs pins.
"""
import numpy as np
import pytest

from eschalign_b200 import adapter, synth
from tests.helpers import Rng, brute_pair_select, pairs_fixture

R1, R2 = adapter.TRUSEQ_R1, adapter.TRUSEQ_R2
SG = (2, -1, -10, -1)


def test_adapter_find_known_answers(oracle):
    """adapter.rs:117-165."""
    f = oracle.adapter_find
    assert f(b"ACGTACGTAC" + R1[:20]) == 20
    assert f(b"ACGTACGTAC" + R1[:6]) == 6
    assert f(b"ACGTACGTAC" + R1 + b"TTTT") == len(R1) + 4
    a = bytearray(R1[:20])
    a[5], a[12] = ord("T"), ord("T")
    assert f(b"G" * 12 + bytes(a)) == 20
    a[15] = ord("C")
    assert f(b"G" * 12 + bytes(a)) == 0
    assert f(b"G" * 12 + b"AGATCGGAT") == 0
    assert f(b"G" * 12 + b"AGAT") == 0
    assert f(b"G" * 12 + b"AGAT", min_overlap=4) == 4
    assert f(b"AG") == 0 and f(b"") == 0
    assert f(b"G" * 12 + b"AGATNGGAAGAG") == 12


def test_adapter_detect_pair_known_answers(oracle):
    """adapter.rs:168-197."""
    ins = b"GGGGCCCCGGGGCCCCGGGG"
    mk = lambda ad, x: ins + ad[:x]  # noqa: E731
    sh = lambda ad, x: ins + b"CC" + ad[:x]  # noqa: E731
    d = oracle.adapter_detect_pair
    assert d(mk(R1, 12), mk(R2, 12)) == [12, 12]
    assert d(mk(R1, 12), sh(R2, 9)) == [12, 0]
    assert d(sh(R1, 7), mk(R2, 12)) == [0, 12]
    assert d(mk(R1, 8), sh(R2, 8)) == [0, 0]
    assert d(mk(R1, 12), ins) == [12, 0]


def _fixture_mates(pairs, names):
    return [m for n in names for m in pairs[n]]


def test_fixture_adapter_counts(oracle):
    """align_paired.rs:303-340 (the `ad` tag of each mate), in the oracle and
    in the library."""
    _, _, pairs = pairs_fixture()
    names = list(pairs)
    want = {"short_insert": [20, 20], "one_mate_reads_through": [15, 0], "plain": [0, 0]}
    for n, w in want.items():
        assert oracle.pair_adapters(*pairs[n]) == w, n
    mates = _fixture_mates(pairs, names)
    ads, aligned = adapter.pair_adapters(mates)
    got = {n: ads[2 * i:2 * i + 2].tolist() for i, n in enumerate(names)}
    for n, w in want.items():
        assert got[n] == w, n
    for i, n in enumerate(names):
        assert got[n] == oracle.pair_adapters(*pairs[n]), n
        assert aligned[2 * i] == pairs[n][0].size - got[n][0]
    # an adapter that is not in the data finds nothing (align_paired.rs:323-333)
    t16 = adapter.config(b"T" * 16, b"T" * 16)
    ads, _ = adapter.pair_adapters(mates, t16)
    assert ads[2 * names.index("short_insert")] == 0
    # a raised minimum overlap hides the 15-base read-through (:335-338)
    ads, _ = adapter.pair_adapters(mates, adapter.config(min_overlap=16))
    assert ads[2 * names.index("one_mate_reads_through")] == 0
    # no adapters: nothing trimmed
    ads, aligned = adapter.pair_adapters(mates, {})
    assert not ads.any() and np.array_equal(aligned, [m.size for m in mates])


@pytest.mark.parametrize("max_read_len", [0, 60, 149])
def test_library_trimming_matches_oracle(oracle, max_read_len):
    """esg_pair_adapters on synthetic read-through pairs (insert median 90,
    1 % adapter errors, indels) and over-length mates, against the oracle."""
    refs = synth.panel_tiles()
    P, _ = synth.pairs_c4(refs, n=3000, seed=77)
    if max_read_len:
        # ragged mates: cut some mates so both sides of the limit occur
        mates = []
        rng = np.random.default_rng(max_read_len)
        for k in range(len(P)):
            m = P.read(k)
            mates.append(m[:rng.integers(max_read_len - 20, 151)])
    else:
        mates = P.list()
    cfg = adapter.config(max_read_len=max_read_len)
    ads, aligned = adapter.pair_adapters(mates, cfg)
    for p in range(len(mates) // 2):
        want = oracle.pair_adapters(mates[2 * p], mates[2 * p + 1], max_read_len=max_read_len)
        assert ads[2 * p:2 * p + 2].tolist() == want, p
    trimmed, want_ads = oracle.trim_pairs(mates, max_read_len=max_read_len)
    assert np.array_equal(ads, want_ads)
    assert np.array_equal(aligned, [t.size for t in trimmed])
    if not max_read_len:
        assert (ads > 0).mean() > 0.3  # the workload does read through
    else:
        assert (aligned == 0).any() and (aligned > 0).any()


def test_pair_select_against_sort(oracle):
    """The oracle's single-pass ranking equals pair.rs's sort of every
    candidate, with ties, ineligible mates and both strand settings."""
    rng = Rng(2024)
    for case in range(400):
        n = 1 + rng.below(40)
        span = 1 + rng.below(12)
        rows = [np.array([rng.below(span) - 3 for _ in range(n)]) for _ in range(4)]
        both = bool(rng.below(2))
        ms = rng.below(5) - 2
        cap = 1 + rng.below(6)
        res, ties = oracle.pair_select(*rows, both_strands=both, min_score=ms, cap=cap)
        best, nxt, n_tied, bt, xs, prim = brute_pair_select(*rows, both, ms, cap)
        NO = oracle.NO_SCORE
        opt = lambda v: NO if v is None else v  # noqa: E731
        assert int(res["best"]) == opt(best), case
        assert int(res["next"]) == opt(nxt), case
        assert int(res["n_tied"]) == n_tied, case
        assert ties == bt, case
        assert tuple(int(v) for v in res["xs"]) == tuple(opt(v) for v in xs), case
        assert tuple(int(v) for v in res["primary"]) == tuple(opt(v) for v in prim), case
        assert bool(res["flags"] & oracle.RESULT_EMPTY) == (best is None)
        assert bool(res["flags"] & oracle.RESULT_TIES_TRUNCATED) == (n_tied > cap)


def test_fixture_pair_ranking(oracle):
    """What align_paired.rs pins, at the ranking stage (semi-global,
    2,-1,-10,-1, --min-score 40, forward template strand: the CLI's paired
    defaults, align.rs:1921-1926 and align_paired.rs:31)."""
    names, refs, pairs = pairs_fixture()
    order = list(pairs)
    trimmed, _ = oracle.trim_pairs(_fixture_mates(pairs, order))
    res, ties = oracle.scalar_map_pairs(trimmed, refs, SG, local=False, both_strands=False,
                                        min_score=40, cap=8)
    got = {n: (res[i], ties[i, :min(int(res[i]["n_tied"]), 8)].tolist())
           for i, n in enumerate(order)}
    ref = {n: i for i, n in enumerate(names)}
    # paralog: the pair is unique on P1 (:199-206) while mate 1 alone ties
    # P1/P2, so mate 1's XS equals its score (:224)
    r, t = got["paralog"]
    assert t == [ref["P1"] << 1] and r["n_tied"] == 1
    assert r["xs"][0] == r["primary"][0]
    # pair_tie: tie between P1 and P2, P1 first (:255-263)
    r, t = got["pair_tie"]
    assert t == [ref["P1"] << 1, ref["P2"] << 1] and r["n_tied"] == 2
    # terminal mismatch kept end to end (:342-356): 59 matches, 1 mismatch
    r, t = got["terminal_mismatch"]
    assert t == [ref["U1"] << 1] and tuple(r["primary"]) == (117, 117)
    # short insert, one mate reading through, plain, over max insert: all on
    # their reference (:282-300, :303-318, :365-380)
    for n, want in (("short_insert", "U1"), ("one_mate_reads_through", "U2"), ("plain", "U2"),
                    ("over_max_insert", "U1")):
        r, t = got[n]
        assert t[:1] == [ref[want] << 1], n
    # the junk mate leaves no eligible candidate (:390-397): Separate
    r, _ = got["one_unmapped"]
    assert r["flags"] & oracle.RESULT_EMPTY and r["n_tied"] == 0
    # each mate of the FF pair on its own, both strands, forward on U2 (:383-388)
    a, b = pairs["wrong_orientation"]
    for m in (a, b):
        fwd = [oracle.score(m, x, SG, False) for x in refs]
        rev = [oracle.score(oracle.revcomp(m), x, SG, False) for x in refs]
        best, _, _, _, tl = oracle.select(fwd, rev, cap=8)
        assert tl[0] == ref["U2"] << 1
