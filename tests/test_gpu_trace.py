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
