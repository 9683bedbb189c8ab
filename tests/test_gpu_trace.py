"""Traceback of winners on the CUDA path (esg_align_*) against the oracle.

Every job's score, coordinates and CIGAR must equal scalar::align
(crates/eschalign/src/scalar.rs:182-364, restated in oracle/esg_align.c):
the same end cell (first maximum of a column-major scan) and the same path
(diagonal, then insertion, then deletion; extending inside a gap; local mode
stopping at the first zero cell) -- not merely an optimal one."""
import numpy as np
import pytest

from eschalign_b200 import GpuScorer, Mode, Scoring, encode, synth
from tests.helpers import SCHEMES, Rng, fixture_panel, fixture_reads, golden, random_panel, \
    random_seq, reads_for, revcomp

pytestmark = pytest.mark.gpu


def check(oracle, g, reads, panel, jobs, scoring, local, what):
    got = g.align(reads, jobs)
    for k, (rd, ref, rev) in enumerate(jobs):
        q = revcomp(reads[rd]) if rev else reads[rd]
        want, wops = oracle.align(q, panel[ref], scoring, local)
        r = got.records[k]
        fields = ("score", "query_start", "query_end", "ref_start", "ref_end")
        assert tuple(int(r[f]) for f in fields) == tuple(int(want[f]) for f in fields), \
            (what, k, rd, ref, rev, r, want)
        assert list(got.ops_of(k)) == list(wops), (what, k, got.cigar(k), oracle.cigar_string(wops))
    return got


def test_trace_golden_cases(oracle):
    """The 192 parasail golden cases, each read against its own reference."""
    by = {}
    for c in golden()["cases"]:
        by.setdefault((c["mode"], tuple(c["scheme"])), []).append(c)
    for (mode, scheme), cases in by.items():
        for c in cases:
            q, r = encode(c["query"]), encode(c["reference"])
            with GpuScorer([r], Scoring(*scheme), Mode.LOCAL if mode == "local"
                           else Mode.SEMIGLOBAL) as g:
                got = check(oracle, g, [q], [r], [(0, 0, 0)], scheme, mode == "local",
                            c["name"])
                rec = got.records[0]
                assert (int(rec["query_start"]), int(rec["query_end"]), int(rec["ref_start"]),
                        int(rec["ref_end"])) == (c["query_start"], c["query_end"],
                                                 c["ref_start"], c["ref_end"])


@pytest.mark.parametrize("mode", [Mode.LOCAL, Mode.SEMIGLOBAL])
def test_trace_random_panel_all_jobs(oracle, mode):
    """Every (read, reference, strand) of a ragged 30-ref panel, five
    schemes: tiles of many jobs, each on its own reference."""
    rng = Rng(0x5EED_0701)
    letters = random_panel(rng, 30, 20, 260)
    panel = [encode(s) for s in letters]
    reads = reads_for(rng, letters, 25) + [np.zeros(0, np.uint8), encode("A")]
    jobs = [(i, r, v) for i in range(len(reads)) for r in range(len(panel)) for v in (0, 1)]
    for scoring in SCHEMES:
        with GpuScorer(panel, Scoring(*scoring), mode) as g:
            got = check(oracle, g, reads, panel, jobs, scoring, mode == Mode.LOCAL,
                        f"{mode.label} {scoring}")
            empty = [k for k, (i, _, _) in enumerate(jobs) if reads[i].size == 0]
            assert all(got.records[k]["score"] == 0 and got.records[k]["n_ops"] == 0
                       for k in empty)


def test_trace_long_reads_in_passes(oracle):
    """Reads over 32 stripes (512 nt) run alone in passes; up to 2500 nt
    against 700-900 nt references, both modes."""
    rng = Rng(0x5EED_0702)
    letters = random_panel(rng, 4, 700, 200)
    panel = [encode(s) for s in letters]
    reads = []
    for n in (513, 700, 1024, 1600, 2500):
        body = letters[n % 4]
        s = (body * 4)[:n]
        reads.append(encode(s))
    reads.append(encode(random_seq(rng, 900, 0.0)))
    jobs = [(i, r, v) for i in range(len(reads)) for r in (0, 3) for v in (0, 1)]
    for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
        with GpuScorer(panel, Scoring(2, -1, -10, -1), mode) as g:
            check(oracle, g, reads, panel, jobs, (2, -1, -10, -1), mode == Mode.LOCAL,
                  f"long {mode.label}")


def test_trace_wildcards_on_fixture_panel(oracle):
    """The ambiguous tRNA panel (wildcards in the references) and the
    fixture reads."""
    panel = fixture_panel("trna_ambiguous")
    reads = fixture_reads()
    jobs = [(i, r, 0) for i in range(len(reads)) for r in range(0, len(panel), 3)]
    for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
        with GpuScorer(panel, Scoring(), mode) as g:
            check(oracle, g, reads, panel, jobs, (2, -1, -10, -1), mode == Mode.LOCAL,
                  f"trna {mode.label}")


def test_trace_winners_of_a_scored_batch(oracle):
    """The flow of map_reads_scored: score a C2 sample, then trace each
    read's first tie straight from the batch's reads on the device."""
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=1500)
    with GpuScorer(refs, Scoring(), Mode.LOCAL) as g:
        b = g.submit(g.prepare(reads.tuple(), both_strands=True))
        res = g.finish(b, keep=True)
        jobs = [(k, int(res.ties[k, 0]) >> 1, int(res.ties[k, 0]) & 1)
                for k in range(len(reads)) if res.results["n_tied"][k] > 0]
        got = g.align_batch(b, jobs)
        b.free()
    rl = reads.list()
    for k, (rd, ref, rev) in enumerate(jobs):
        q = revcomp(rl[rd]) if rev else rl[rd]
        want, wops = oracle.align(q, refs[ref], (2, -1, -10, -1), True)
        rec = got.records[k]
        assert int(rec["score"]) == int(res.results["best"][rd]) == int(want["score"])
        assert (int(rec["query_start"]), int(rec["ref_start"]), int(rec["ref_end"])) == \
            (int(want["query_start"]), int(want["ref_start"]), int(want["ref_end"]))
        assert list(got.ops_of(k)) == list(wops)


def test_trace_pair_winners_on_trimmed_mates(oracle):
    """A paired batch's reads on the device are the trimmed mates: trace the
    first tie of each pair (mate 1 on the template strand, mate 2 on the
    other, pair.rs:135-137) against the oracle on the trimmed codes."""
    from eschalign_b200 import adapter
    refs = synth.panel_tiles()[:40]
    P, _ = synth.pairs_c4(refs, n=200, seed=21)
    mates = P.list()
    trimmed, _ = oracle.trim_pairs(mates)
    with GpuScorer(refs, Scoring(), Mode.SEMIGLOBAL) as g:
        b = g.submit(g.prepare_pairs(mates, adapters=adapter.config()))
        got = g.finish_pairs(b, keep=True)
        jobs = []
        for p in range(len(mates) // 2):
            if got.pairs["n_tied"][p] == 0:
                continue
            c = int(got.pair_ties[p, 0])
            ref, t = c >> 1, c & 1
            jobs += [(2 * p, ref, t), (2 * p + 1, ref, 1 - t)]
        al = g.align_batch(b, jobs)
        b.free()
    for k, (rd, ref, rev) in enumerate(jobs):
        q = revcomp(trimmed[rd]) if rev else trimmed[rd]
        want, wops = oracle.align(q, refs[ref], (2, -1, -10, -1), False)
        rec = al.records[k]
        assert int(rec["score"]) == int(want["score"]), k
        assert (int(rec["query_start"]), int(rec["query_end"]), int(rec["ref_start"]),
                int(rec["ref_end"])) == (int(want["query_start"]), int(want["query_end"]),
                                         int(want["ref_start"]), int(want["ref_end"])), k
        assert list(al.ops_of(k)) == list(wops), k
    # each pair's two traced mates add up to the ranked sum
    for p in range(0, len(jobs), 2):
        pi = jobs[p][0] // 2
        assert int(al.records[p]["score"]) + int(al.records[p + 1]["score"]) == \
            int(got.pairs["best"][pi])
