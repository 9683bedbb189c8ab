"""Paired-end batches on the CUDA path against the CPU oracle, by equality.

A paired batch trims each mate's 3' adapter on the host (adapter.rs:68-110,
align.rs:934-949), scores all four mate queries per pair on the device and
ranks the (reference, template strand) candidates there (pair.rs:195-234,
:297-314).  Each check compares the adapters, every mate's row, each mate's
own both-strand result (the Separate fallback, pair.rs:366-387) and each
pair's ranking with the oracle, on both kernels."""
import numpy as np
import pytest

from eschalign_b200 import KERNEL_AUTO, KERNEL_INT32, KERNEL_PLAIN32, GpuScorer, Mode, Scoring, adapter, synth
from tests.helpers import pairs_fixture

pytestmark = pytest.mark.gpu

SG = (2, -1, -10, -1)
NO_TIE = 0xFFFFFFFF
CONFIGS = ((KERNEL_AUTO, 512, 64), (KERNEL_AUTO, 0, 1), (KERNEL_INT32, 256, 64),
           (KERNEL_PLAIN32, 256, 64))


def expected(O, mates, refs, scoring, local, both, min_score, cap, max_read_len=0,
             adapters=True):
    if adapters:
        trimmed, ads = O.trim_pairs(mates, max_read_len=max_read_len)
    else:
        trimmed, ads = list(mates), np.zeros(len(mates), dtype=np.uint32)
    lens = np.array([t.size for t in trimmed], dtype=np.uint32)
    rc = [O.revcomp(t) for t in trimmed]
    rows = O.score_matrix(list(trimmed) + rc, refs, scoring, local)
    mres, mties, _ = O.scalar_map_batch(trimmed, refs, scoring, local, True, cap=cap)
    pres, pties = O.pairs_from_rows(rows, lens, len(refs), both, min_score, cap)
    return ads, rows, mres, mties, pres, pties


def compare(got, want, cap, what):
    ads, rows, mres, mties, pres, pties = want
    assert np.array_equal(got.adapters, ads), f"{what}: adapters"
    bad = np.argwhere(got.mates.rows != rows)
    assert bad.size == 0, f"{what}: row {bad[0]} got {got.mates.rows[tuple(bad[0])]} want {rows[tuple(bad[0])]}"
    for f in ("best", "suboptimal", "n_tied"):
        assert np.array_equal(got.mates.results[f], mres[f]), f"{what}: mate {f}"
    assert np.array_equal(got.mates.results["flags"] & 3, mres["flags"]), f"{what}: mate flags"
    for k in range(len(mres)):
        n = min(int(mres["n_tied"][k]), cap)
        assert np.array_equal(got.mates.ties[k, :n], mties[k, :n]), f"{what}: mate {k} ties"
    for f in ("best", "next", "n_tied"):
        bad = np.nonzero(got.pairs[f] != pres[f])[0]
        assert bad.size == 0, f"{what}: pair {bad[0]} {f} got {got.pairs[bad[0]]} want {pres[bad[0]]}"
    for f in ("xs", "primary"):
        assert np.array_equal(got.pairs[f], pres[f]), f"{what}: pair {f}"
    assert np.array_equal(got.pairs["flags"] & 3, pres["flags"]), f"{what}: pair flags"
    for p in range(len(pres)):
        n = min(int(pres["n_tied"][p]), cap)
        assert np.array_equal(got.pair_ties[p, :n], pties[p, :n]), f"{what}: pair {p} ties"
        assert (got.pair_ties[p, n:] == NO_TIE).all(), f"{what}: pair {p} unused tie slots"


def test_fixture_pairs(oracle):
    """The reference's paired fixture (align_paired.rs), CLI paired defaults:
    semi-global, 2,-1,-10,-1, --min-score 40, forward template strand."""
    names, refs, pairs = pairs_fixture()
    order = list(pairs)
    mates = [m for n in order for m in pairs[n]]
    want = expected(oracle, mates, refs, SG, False, False, 40, 8)
    with GpuScorer(refs, Scoring(*SG), Mode.SEMIGLOBAL, tie_capacity=8) as g:
        for kernel, split, chunks in CONFIGS:
            g.set_kernel(kernel)
            g.set_split(split)
            g.set_chunking(chunks)
            got = g.score_pairs(mates, adapters=adapter.config(), min_score=40,
                                both_strands=False, full_rows=True)
            compare(got, want, 8, f"fixture kernel {kernel}/{split}")
            ix = {n: i for i, n in enumerate(order)}
            ref = {n: i for i, n in enumerate(names)}
            assert got.pair(ix["paralog"]).ties == [(ref["P1"], False)]
            assert got.pair(ix["pair_tie"]).ties == [(ref["P1"], False), (ref["P2"], False)]
            assert got.pair(ix["terminal_mismatch"]).primary == (117, 117)
            assert got.pair(ix["one_unmapped"]).best is None
            i = ix["short_insert"]
            assert got.adapters[2 * i:2 * i + 2].tolist() == [20, 20]
            i = ix["one_mate_reads_through"]
            assert got.adapters[2 * i:2 * i + 2].tolist() == [15, 0]


def _panel_with_paralogs():
    refs = synth.panel_tiles()[:40]
    # exact copies and a one-base paralog give pair and mate ties
    para = refs[3].copy()
    para[para.size // 2] = (para[para.size // 2] + 1) % 4
    return refs + [refs[7].copy(), refs[11].copy(), para]


def _edge_mates(refs):
    """Empty mates, one-base mates, a mate that is all adapter."""
    a = refs[0][10:90]
    r = [a, np.zeros(0, np.uint8), np.zeros(0, np.uint8), np.zeros(0, np.uint8),
         refs[1][:1], refs[1][5:6], adapter.encode(adapter.TRUSEQ_R1), a[::-1].copy()]
    return r


@pytest.mark.parametrize("mode", [Mode.SEMIGLOBAL, Mode.LOCAL])
@pytest.mark.parametrize("both,min_score,cap", [(True, 0, 8), (False, 40, 8), (True, -5, 2)])
def test_synthetic_pairs(oracle, mode, both, min_score, cap):
    """Read-through pairs of 2 x 150 (insert median 90) plus edge mates."""
    refs = _panel_with_paralogs()
    P, _ = synth.pairs_c4(refs, n=300, seed=4242)
    mates = P.list() + _edge_mates(refs)
    local = mode == Mode.LOCAL
    want = expected(oracle, mates, refs, SG, local, both, min_score, cap)
    with GpuScorer(refs, Scoring(*SG), mode, tie_capacity=cap) as g:
        for kernel, split, chunks in CONFIGS:
            g.set_kernel(kernel)
            g.set_split(split)
            g.set_chunking(chunks)
            got = g.score_pairs(mates, adapters=adapter.config(), min_score=min_score,
                                both_strands=both, full_rows=True)
            compare(got, want, cap, f"{mode.label} both={both} min={min_score} kernel {kernel}")
            assert got.stats["n_pairs"] == len(mates) // 2
            assert got.stats["mates_trimmed"] == int((want[0] > 0).sum())
    # ties were exercised, and truncated at the small capacity
    pres = want[4]
    assert (pres["n_tied"] > 1).any()
    if cap == 2:
        assert (pres["n_tied"] > 2).any() or both is False


def test_pairs_max_read_len_and_no_trimming(oracle):
    """align.rs:934-949: a mate over --max-read-len is neither searched nor
    aligned; without adapters nothing is trimmed."""
    refs = _panel_with_paralogs()
    P, _ = synth.pairs_c4(refs, n=200, seed=99)
    rng = np.random.default_rng(5)
    mates = [m[:rng.integers(100, 151)] for m in P.list()]
    with GpuScorer(refs, Scoring(*SG), Mode.SEMIGLOBAL, tie_capacity=4) as g:
        want = expected(oracle, mates, refs, SG, False, True, 0, 4, max_read_len=130)
        got = g.score_pairs(mates, adapters=adapter.config(max_read_len=130), full_rows=True)
        compare(got, want, 4, "max_read_len 130")
        want = expected(oracle, mates, refs, SG, False, True, 0, 4, adapters=False)
        got = g.score_pairs(mates, adapters=None, full_rows=True)
        compare(got, want, 4, "no trimming")


def test_pairs_without_rows_and_overlapped(oracle):
    """The ranking does not depend on returning rows, and paired batches
    pipeline like any batch (prepare while the previous one runs)."""
    refs = _panel_with_paralogs()
    P, _ = synth.pairs_c4(refs, n=400, seed=7)
    mates = P.list()
    with GpuScorer(refs, Scoring(*SG), Mode.SEMIGLOBAL, tie_capacity=8) as g:
        full = g.score_pairs(mates, adapters=adapter.config(), full_rows=True)
        a = g.submit(g.prepare_pairs(mates[:400], adapters=adapter.config()))
        b = g.prepare_pairs(mates[400:], adapters=adapter.config())
        ra = g.finish_pairs(a)
        rb = g.finish_pairs(g.submit(b))
        for f in full.pairs.dtype.names:
            assert np.array_equal(np.concatenate([ra.pairs[f], rb.pairs[f]]), full.pairs[f]), f
        assert np.array_equal(np.vstack([ra.pair_ties, rb.pair_ties]), full.pair_ties)
        assert ra.mates.rows is None
