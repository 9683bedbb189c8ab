"""The CUDA path against the CPU oracle, by equality (no tolerance: integer
scores).  Mirrors crates/eschalign/tests/gpu_parity.rs: every check runs on
every kernel setting (the batched int16x2 kernel with int32 lanes for what
it cannot take, every query on the int32 lanes, and int32 one thread per
(query, reference)), reverse complements included, and compares
every query's full row with the scalar oracle and every read's reduced
result (best, XS, tie count, tie list) with the oracle's selection
(mapper.rs:444-472)."""
import numpy as np
import pytest

from eschalign_b200 import (KERNEL_AUTO, KERNEL_INT32, KERNEL_PLAIN32, GpuError, GpuScorer, Mode,
                            Scoring, encode, pack_reads, synth)
from tests.helpers import (SCHEMES, Rng, fixture_panel, fixture_reads, golden, random_panel,
                           random_seq, reads_for)

pytestmark = pytest.mark.gpu

CAP = 8


def cpu_results(O, refs, packed, scoring, local, both):
    """Per-read results of the reference's CPU path: the AVX-512 restatement
    where the host has AVX-512BW, else the scalar oracle (equal by test)."""
    if O.lib().eo_cpu_has_avx512bw():
        r, t, _, _ = O.Profile(refs, scoring).map_batch(*packed.tuple(), local=local,
                                                       both_strands=both, cap=CAP)
        return r, t
    r, t, _ = O.scalar_map_batch(packed.list(), refs, scoring, local, both, cap=CAP)
    return r, t


def oracle_rows(O, reads, panel, scoring, local):
    """Forward rows then reverse-complement rows, scalar oracle."""
    rc = [O.revcomp(r) for r in reads]
    return O.score_matrix(list(reads) + rc, panel, scoring, local)


# (kernel, 16/32-row split, panel chunks at most): 16-row stripes up to
# 512 nt with the panel chunked or whole, every query on 32-row stripes
# chunked or whole, every query on the int32 lanes, and in int32 one thread
# per (query, reference)
CONFIGS = ((KERNEL_AUTO, 512, 64), (KERNEL_AUTO, 512, 1), (KERNEL_AUTO, 0, 64),
           (KERNEL_AUTO, 0, 1), (KERNEL_INT32, 256, 64), (KERNEL_PLAIN32, 256, 64))


def check(O, panel, reads, scoring, mode, what, kernels=CONFIGS, tie_capacity=CAP):
    """gpu_parity.rs:132-192."""
    local = mode == Mode.LOCAL
    want_rows = oracle_rows(O, reads, panel, scoring, local)
    want_res, want_ties, _ = O.scalar_map_batch(reads, panel, scoring, local, True,
                                               cap=tie_capacity)
    n = len(reads)
    stats = {}
    with GpuScorer(panel, Scoring(*scoring), mode, tie_capacity=tie_capacity) as g:
        for kernel, split, chunks in kernels:
            g.set_kernel(kernel)
            g.set_split(split)
            g.set_chunking(chunks)
            res = g.score_batch(reads, both_strands=True, full_rows=True)
            got = res.rows
            assert got.shape == want_rows.shape
            bad = np.argwhere(got != want_rows)
            assert bad.size == 0, (f"{what} {mode.label} {scoring} kernel {kernel}: query "
                                   f"{bad[0][0]} ref {bad[0][1]} got {got[tuple(bad[0])]} "
                                   f"want {want_rows[tuple(bad[0])]}")
            for field in ("best", "suboptimal", "n_tied"):
                assert (res.results[field] == want_res[field]).all(), (what, field, kernel)
            assert ((res.results["flags"] & 3) == (want_res["flags"] & 3)).all(), (what, kernel)
            for k in range(n):
                nl = min(int(want_res["n_tied"][k]), tie_capacity)
                assert (res.ties[k, :nl] == want_ties[k, :nl]).all(), (what, k, kernel)
            stats[(kernel, split, chunks)] = res.stats
            stats.setdefault(kernel, res.stats)
    return stats


def test_gpu_scores_equal_scalar_random_panel(oracle):
    """gpu_parity.rs:217-232: 37 references, ragged, five schemes."""
    rng = Rng(0x5EED_0101)
    letters = random_panel(rng, 37, 20, 280)
    panel = [encode(s) for s in letters]
    reads = reads_for(rng, letters, 60)
    for scoring in SCHEMES:
        for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
            st = check(oracle, panel, reads, scoring, mode, "random 37-ref panel")
            assert st[KERNEL_AUTO]["queries_batched"] == 2 * len(reads)
            # a small batch cuts the panel into chunks, unless told not to
            assert st[(KERNEL_AUTO, 512, 64)]["panel_chunks"] > 1
            assert st[(KERNEL_AUTO, 512, 1)]["panel_chunks"] == 1


def test_gpu_gap_open_cheaper_than_extend(oracle):
    """Schemes whose gap open costs less than an extension (|o| < |e|; valid
    for the reference, scoring.rs:70-100), where a gap of one base can beat
    the extension of an open one: short and long (multi-pass) reads, both
    modes, every kernel setting."""
    rng = Rng(0x5EED_0101 + 3)
    letters = random_panel(rng, 37, 20, 280)
    panel = [encode(s) for s in letters]
    reads = reads_for(rng, letters, 40)
    reads += [encode(random_seq(rng, 1100 + 150 * k, 0.01)) for k in range(3)]
    for scoring in ((2, -3, -1, -5), (1, -1, 0, -2), (3, -2, -2, -4)):
        for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
            check(oracle, panel, reads, scoring, mode, "open below extend")


def test_gpu_scores_equal_scalar_wide_panel(oracle):
    """gpu_parity.rs:234-247: 300 references up to 620 nt -- too big for the
    shared-memory panel, so the batched kernel reads it through L2."""
    rng = Rng(0x5EED_0101 + 7)
    letters = random_panel(rng, 300, 20, 600)
    panel = [encode(s) for s in letters]
    reads = reads_for(rng, letters, 6)
    for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
        check(oracle, panel, reads, (2, -1, -10, -1), mode, "random 300-ref panel")


@pytest.mark.parametrize("tag", ["trna", "trna_ambiguous"])
def test_gpu_fixture_reads_on_trna_panels(oracle, tag):
    """gpu_parity.rs:249-260: the real tRNA reads against both 47-reference
    fixture panels (the ambiguous one carries wildcards)."""
    panel = fixture_panel(tag)
    reads = fixture_reads()
    assert len(panel) == 47 and len(reads) >= 5
    for scoring in SCHEMES:
        for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
            check(oracle, panel, reads, scoring, mode, tag)


def test_gpu_golden_pairs(oracle):
    """The 192 parasail golden pairs, each read against its own reference."""
    g = golden()
    for c in g["cases"]:
        q, r = encode(c["query"]), encode(c["reference"])
        mode = Mode.LOCAL if c["mode"] == "local" else Mode.SEMIGLOBAL
        with GpuScorer([r], Scoring(*c["scheme"]), mode) as s:
            for kernel, split, chunks in CONFIGS:
                s.set_kernel(kernel)
                s.set_split(split)
                s.set_chunking(chunks)
                res = s.score_batch([q], full_rows=True)
                assert res.rows[0, 0] == c["score"], (c["name"], c["mode"], kernel, split)


def test_gpu_long_and_straddling_reads(oracle):
    """gpu_parity.rs:269-321 in spirit: reads either side of the batched
    kernel's 512-row limit, against references of 900-1000 nt."""
    rng = Rng(0x5EED_0103)
    letters = random_panel(rng, 21, 900, 100)
    panel = [encode(s) for s in letters]
    reads = []
    for t in range(24):
        ln = 440 + 12 * t
        r = letters[rng.below(len(letters))]
        read = random_seq(rng, ln, 0.01) if t % 3 == 2 else mutate_trunc(rng, r, ln)
        reads.append(encode(read))
    for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
        st = check(oracle, panel, reads, (3, -2, -5, -2), mode, "straddling batch")
        a = st[KERNEL_AUTO]
        # reads over 512 nt run on the batched kernel in several passes
        assert a["queries_batched"] == 2 * len(reads) and a["queries_plain"] == 0


@pytest.mark.parametrize("tag", ["trna_ambiguous", "random"])
def test_gpu_multipass_reads(oracle, tag):
    """Reads either side of every pass boundary of the batched kernel's long
    path (32 stripes of 16 rows per pass): 511-513, 527-529, 1023-1025 nt,
    and 2000 / 5000 nt (4 and 10 passes), on a tRNA panel with wildcards
    and on a random panel, both modes, two schemes."""
    rng = Rng(0x5EED_0106)
    if tag == "random":
        letters = random_panel(rng, 11, 60, 200)
        panel = [encode(s) for s in letters]
    else:
        panel = fixture_panel(tag)[:13]
        letters = [bytes(np.frombuffer(b"ACGTN", np.uint8)[p]) for p in panel]
    reads = []
    for ln in (511, 512, 513, 527, 528, 529, 1023, 1024, 1025, 2000, 5000):
        r = letters[rng.below(len(letters))]
        body = b"".join(mutate_trunc(rng, r, len(r)) for _ in range(ln // 60 + 2))
        reads.append(encode((random_seq(rng, 7, 0.01) + body)[:ln]))
    reads.append(encode(random_seq(rng, 700, 0.02)))
    for scoring in ((2, -1, -10, -1), (3, 1, -5, -2)):
        for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
            st = check(oracle, panel, reads, scoring, mode, f"multipass {tag}")
            assert st[KERNEL_AUTO]["queries_plain"] == 0


def mutate_trunc(rng, r, ln):
    from tests.helpers import mutate
    return mutate(rng, r[:ln])[:ln]


def test_gpu_scores_everything_it_is_given(oracle):
    """gpu_parity.rs:355-378, inverted: empty reads come back empty, and a
    read over the reference GPU's 4096 nt limit is scored here too."""
    rng = Rng(0x5EED_0102)
    letters = random_panel(rng, 20, 50, 100)
    panel = [encode(s) for s in letters]
    long = encode(random_seq(rng, 4097, 0.0))
    ok = encode(random_seq(rng, 120, 0.0))
    edge = encode(random_seq(rng, 4096, 0.0))
    reads = [ok, np.zeros(0, np.uint8), long, edge, ok]
    with GpuScorer(panel, Scoring(), Mode.LOCAL) as g:
        res = g.score_batch(reads, full_rows=True)
        assert res.read(1).best is None and res.results["flags"][1] & 1
        assert not res.rows[1].any()  # an empty query scores 0 against everything
        for k in (0, 2, 3, 4):
            for r, ref in enumerate(panel):
                assert res.rows[k, r] == oracle.score(reads[k], ref, (2, -1, -10, -1), True)
        assert len(g.score_batch([])) == 0


def test_gpu_refuses_a_reference_it_cannot_hold():
    """gpu_parity.rs:380-389."""
    with pytest.raises(GpuError) as ei:
        GpuScorer([np.zeros(32769, np.uint8)], Scoring(), Mode.LOCAL)
    assert ei.value.kind == "ReferenceTooLong"


def test_gpu_int16_saturation_is_rescored_in_int32(oracle):
    """Scores past int16: 100,-100,-27,-27 on 400-500 nt exact matches reach
    40 000-50 000.  The batched kernel flags them and the int32 kernel
    re-scores them; results equal the oracle's int32 scores."""
    rng = Rng(0x5EED_0105)
    letters = random_panel(rng, 40, 480, 40)
    panel = [encode(s) for s in letters]
    reads = [encode(letters[k][:400 + 10 * k]) for k in range(9)]
    reads += [encode(random_seq(rng, 300, 0.0)) for _ in range(5)]
    scoring = (100, -100, -27, -27)
    st = check(oracle, panel, reads, scoring, Mode.LOCAL, "saturating")
    for key in ((KERNEL_AUTO, 512, 64), (KERNEL_AUTO, 512, 1), (KERNEL_AUTO, 0, 64)):
        assert st[key]["queries_rescored"] >= 9, key
    # the re-score requests also come through the panel-chunk merge
    assert st[(KERNEL_AUTO, 512, 64)]["panel_chunks"] > 1
    assert st[KERNEL_AUTO]["queries_batched"] == 2 * len(reads)
    # semi-global: the checked batched kernel takes every query (the gap
    # floor stays inside int16) and flags those whose cells pass 16384
    st = check(oracle, panel, reads, scoring, Mode.SEMIGLOBAL, "saturating semi-global")
    assert st[KERNEL_AUTO]["queries_batched"] == 2 * len(reads)
    assert st[KERNEL_AUTO]["queries_plain"] == 0
    for key in ((KERNEL_AUTO, 512, 64), (KERNEL_AUTO, 512, 1), (KERNEL_AUTO, 0, 64),
                (KERNEL_AUTO, 0, 1)):
        assert st[key]["queries_rescored"] >= 9, key


def test_gpu_ties_truncated_and_counted_in_full(oracle):
    """A panel of identical references: every candidate ties; the count is
    complete and the list holds the first tie_capacity in candidate order."""
    ref = encode(b"ACGTTGCAACGTAGCTAGCTAGGATCCA")
    panel = [ref] * 12 + [encode(b"TTTTTTTTTTTT")]
    reads = [ref, encode(b"ACGTTGCAACG"), encode(b"GGGG")]
    for cap in (1, 3, 8, 32):
        check(oracle, panel, reads, (2, -1, -10, -1), Mode.LOCAL, f"ties cap {cap}",
              tie_capacity=cap)


def test_gpu_config1_reads_equal_avx512(oracle):
    """Config C1 at full size: 10 000 reads vs the 164-reference panel,
    local 2,-1,-10,-1, forward strand -- every read's result equal to the
    AVX-512 baseline's (itself equal to the scalar oracle by test)."""
    refs = synth.panel_tiles()
    reads = synth.reads_c1(refs)
    want, want_t = cpu_results(oracle, refs, reads, (2, -1, -10, -1), True, False)
    with GpuScorer(refs, Scoring(), Mode.LOCAL) as g:
        for kernel in (KERNEL_AUTO, KERNEL_INT32, KERNEL_PLAIN32):
            g.set_kernel(kernel)
            res = g.score_batch(reads.tuple())
            assert (res.results["best"] == want["best"]).all()
            assert (res.results["suboptimal"] == want["suboptimal"]).all()
            assert (res.results["n_tied"] == want["n_tied"]).all()
            n_l = np.minimum(want["n_tied"], CAP)
            mask = np.arange(CAP)[None, :] < n_l[:, None]
            assert (res.ties[mask] == want_t[mask]).all()


@pytest.mark.parametrize("mode", [Mode.LOCAL, Mode.SEMIGLOBAL])
@pytest.mark.parametrize("scoring", [(2, -1, -10, -1), (1, -1, -2, -1)])
def test_gpu_config2_sample_both_strands(oracle, mode, scoring):
    """Config C2 shape (lognormal lengths, both strands, both modes, both
    schemes) on a 20 000-read sample, against the AVX-512 baseline."""
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=20_000)
    local = mode == Mode.LOCAL
    want, want_t = cpu_results(oracle, refs, reads, scoring, local, True)
    with GpuScorer(refs, Scoring(*scoring), mode) as g:
        res = g.score_batch(reads.tuple(), both_strands=True)
        for f in ("best", "suboptimal", "n_tied"):
            assert (res.results[f] == want[f]).all(), f
        n_l = np.minimum(want["n_tied"], CAP)
        mask = np.arange(CAP)[None, :] < n_l[:, None]
        assert (res.ties[mask] == want_t[mask]).all()


def test_gpu_prepare_submit_finish_overlap(oracle):
    """cuda/mod.rs:520-528 / align.rs:2817-2887: batch k+1 prepared while k
    runs, results identical to score_batch one at a time."""
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=6000)
    chunks = [reads.subset(np.arange(k, min(k + 1500, len(reads)))) for k in range(0, 6000, 1500)]
    with GpuScorer(refs, Scoring(), Mode.LOCAL) as g:
        one = [g.score_batch(c.tuple(), both_strands=True) for c in chunks]
        pending = None
        got = []
        for c in chunks + [None]:
            prepared = g.prepare(c.tuple(), both_strands=True) if c is not None else None
            if pending is not None:
                got.append(g.finish(pending))
            pending = g.submit(prepared) if prepared is not None else None
        for a, b in zip(one, got):
            assert (a.results == b.results).all() and (a.ties == b.ties).all()
            # slots past the listed ties hold ESG_NO_TIE
            n_l = np.minimum(a.results["n_tied"], CAP)
            unused = np.arange(CAP)[None, :] >= n_l[:, None]
            assert (a.ties[unused] == 0xFFFFFFFF).all()


def test_gpu_strand_swap_property():
    """Scoring the reverse complements with both strands swaps every
    candidate's strand: best, XS and tie counts are unchanged, tie
    candidates flip their strand bit."""
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=4000)
    rc = [np.where(r[::-1] >= 4, 4, 3 - r[::-1]).astype(np.uint8) for r in reads.list()]
    with GpuScorer(refs, Scoring(), Mode.SEMIGLOBAL) as g:
        a = g.score_batch(reads.tuple(), both_strands=True)
        b = g.score_batch(pack_reads(rc), both_strands=True)
    for f in ("best", "suboptimal", "n_tied"):
        assert (a.results[f] == b.results[f]).all()
    for k in range(len(reads)):
        n = min(int(a.results["n_tied"][k]), CAP)
        assert sorted(a.ties[k, :n] ^ 1) == sorted(b.ties[k, :n]) or a.results["n_tied"][k] > CAP


def test_gpu_autotune_measures_and_keeps_results(oracle):
    """The tile-shape autotuner times 16- and 32-row stripes on this panel,
    picks a split, and the scores do not change with it."""
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=3000)
    with GpuScorer(refs, Scoring(), Mode.LOCAL) as g:
        before = g.score_batch(reads.tuple(), both_strands=True)
        rep = g.autotune()
        assert len(rep["lengths"]) == 7 and all(
            t > 0 for t in rep["ms_rows16"] + rep["ms_rows32"] + rep["ms_int32"])
        assert rep["split_len"] in (0, 48, 80, 112, 160, 224, 320, 512)
        # int16x2 lanes beat int32 lanes on this scheme at every length
        assert rep["int32_from"] == 0
        for knob in ("ctas16", "ctas32", "chunk_target"):
            assert rep[knob]["chosen"] in rep[knob]["tried"] and all(t > 0 for t in rep[knob]["ms"])
        # on the workload's length histogram: every split timed on one batch
        rep = g.autotune(reads.lens)
        hs = rep["split_on_histogram"]
        assert len(hs["tried"]) == 8 and rep["split_len"] in hs["tried"]
        best = min(hs["ms"])
        assert hs["ms"][hs["tried"].index(rep["split_len"])] <= 1.01 * best
        info = g.info()
        assert info["tuned"] == 1 and info["split_len"] == rep["split_len"]
        after = g.score_batch(reads.tuple(), both_strands=True)
        assert (before.results == after.results).all() and (before.ties == after.ties).all()


def test_gpu_half2_lever_and_introspection(oracle):
    """cuda/mod.rs:446-514 mirrored: set_half2 moves every query between the
    fast (batched) kernel and the int32 kernel, half2_scores_len says where a
    length goes, the two geometries / register counts are reported, and the
    scores do not change."""
    rng = Rng(0x5EED_0107)
    letters = random_panel(rng, 20, 60, 100)
    panel = [encode(s) for s in letters]
    reads = reads_for(rng, letters, 30)
    with GpuScorer(panel, Scoring(), Mode.SEMIGLOBAL) as g:
        assert g.half2() and g.half2_scores_len(120) and not g.half2_scores_len(0)
        assert g.geometry()[0] > 0 and g.geometry_h2()[0] > 0
        assert g.registers() > 0 and g.registers_h2() > 0
        fast = g.score_batch(reads, both_strands=True, full_rows=True)
        assert fast.stats["queries_batched"] == 2 * len(reads)
        g.set_half2(False)
        assert not g.half2() and not g.half2_scores_len(120)
        slow = g.score_batch(reads, both_strands=True, full_rows=True)
        assert slow.stats["queries_plain"] == 2 * len(reads)
        assert np.array_equal(fast.rows, slow.rows)
    # semi-global queries whose gap floor 2 |o| + (min(read, reference) - 1)
    # |e| leaves the int16 lanes' range go to int32; inside it the batched
    # kernel takes them (checked when their scores may pass int16)
    assert max(len(p) for p in panel) >= 125
    with GpuScorer(panel, Scoring(100, -100, -27, -127), Mode.SEMIGLOBAL) as g:
        assert g.half2_scores_len(10) and not g.half2_scores_len(400)
    with GpuScorer(panel, Scoring(100, -100, -27, -27), Mode.SEMIGLOBAL) as g:
        assert g.half2_scores_len(10) and g.half2_scores_len(400)


def test_gpu_panel_shards_merge_to_the_whole_panel(oracle):
    """Panel shards on one GPU (the multi-GPU path's scoring and merge, no
    exchange): three shard scorers over a 300-ref panel with copies across
    the cuts, merged, equal the whole-panel scorer."""
    from eschalign_b200 import shards
    rng = Rng(0x5EED_0109)
    letters = random_panel(rng, 300, 200, 300)
    panel = [encode(s) for s in letters]
    panel += [panel[3].copy(), panel[150].copy(), panel[3].copy()]
    reads = reads_for(rng, letters, 40)
    cap = 4
    ranges = shards.shard_ranges([len(p) for p in panel], 3)
    parts = []
    for lo, hi in ranges:
        with GpuScorer(panel[lo:hi], Scoring(), Mode.LOCAL, tie_capacity=cap) as g:
            r = g.score_batch(reads, both_strands=True)
            parts.append((r.results, shards.globalize_ties(r.ties, lo)))
    got_r, got_t = shards.merge(parts, cap)
    with GpuScorer(panel, Scoring(), Mode.LOCAL, tie_capacity=cap) as g:
        want = g.score_batch(reads, both_strands=True)
    for f in ("best", "suboptimal", "n_tied", "flags"):
        assert np.array_equal(got_r[f], want.results[f]), f
    assert np.array_equal(got_t, want.ties)


def test_gpu_graph_launches_equal_direct_launches(oracle):
    """A batch's device work launched as one CUDA graph (the default) and
    kernel by kernel give the same results; relaunching a submitted batch
    through its graph leaves them unchanged; batches of other shapes in
    between (long reads, a chunked small batch) update or add graphs without
    disturbing the others."""
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=5000)
    small = synth.reads_c2(refs, n=40, seed=99)
    rng = Rng(0x5EED_0A12)
    longs = [encode(random_seq(rng, 1500 + 100 * k, 0.0)) for k in range(3)]
    for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
        with GpuScorer(refs, Scoring(), mode) as g:
            got = [g.score_batch(x, both_strands=True)
                   for x in (reads.tuple(), longs, small.tuple(), reads.tuple())]
            g.set_graphs(False)
            want = [g.score_batch(x, both_strands=True)
                    for x in (reads.tuple(), longs, small.tuple(), reads.tuple())]
            for a, b in zip(got, want):
                assert (a.results == b.results).all() and (a.ties == b.ties).all()
            assert got[1].stats["queries_batched"] == 2 * len(longs)
            assert got[2].stats["panel_chunks"] > 1
            g.set_graphs(True)
            pb = g.submit(g.prepare(reads.tuple(), both_strands=True))
            first = g.finish(pb, keep=True)
            g.score_batch(small.tuple(), both_strands=True)  # another shape in between
            g.relaunch(pb)
            res, ties = g.read_results(pb)
            pb.free()
            assert (res == first.results).all() and (ties == first.ties).all()
            assert (first.results == want[0].results).all()


def test_gpu_autotune_lane_type_follows_its_measurements(oracle):
    """With a scheme whose long reads leave int16 (100,-100,-27,-27 on a
    panel of ~500-nt references) the batched kernel flags long queries for a
    second, int32 pass; the autotuner times that against every query on the
    int32 lanes and routes to the int32 lanes exactly the lengths where they
    win at that length and every longer one.  Results stay exact either way."""
    rng = Rng(0x5EED_0A13)
    letters = random_panel(rng, 60, 480, 40)
    panel = [encode(s) for s in letters]
    reads = [encode(letters[k][5:60 + 9 * k]) for k in range(50)]
    reads += [encode(random_seq(rng, 50 + 8 * k, 0.0)) for k in range(10)]
    scoring = (100, -100, -27, -27)
    with GpuScorer(panel, Scoring(*scoring), Mode.LOCAL) as g:
        rep = g.autotune()
        best_k2 = [min(a, b) for a, b in zip(rep["ms_rows16"], rep["ms_rows32"])]
        wins = [i32 < k2 for i32, k2 in zip(rep["ms_int32"], best_k2)]
        if rep["int32_from"]:
            at = rep["lengths"].index(rep["int32_from"])
            assert all(wins[at:]) and (at == 0 or not wins[at - 1])
        else:
            assert not wins[-1]
        res = g.score_batch(reads, both_strands=True, full_rows=True)
        n_int32 = sum(2 for r in reads if rep["int32_from"] and len(r) >= rep["int32_from"])
        assert res.stats["queries_plain"] == n_int32
    want_rows = oracle_rows(oracle, reads, panel, scoring, True)
    assert (res.rows == want_rows).all()
    want, want_t, _ = oracle.scalar_map_batch(reads, panel, scoring, True, True, cap=CAP)
    for f in ("best", "suboptimal", "n_tied"):
        assert (res.results[f] == want[f]).all(), f


def test_gpu_feeder_equals_single_batches():
    """GpuScorer.score_batches (the CLI's GPU feeder, two batches in flight)
    gives each chunk what score_batch gives it alone, in order; and the
    paired feeder what prepare_pairs / finish_pairs give."""
    from eschalign_b200 import adapter
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=12_000, seed=0x5EED_0911)
    chunks = [reads.slice(k, k + 2500) for k in range(0, 12_000, 2500)]
    with GpuScorer(refs, Scoring(), Mode.LOCAL) as g:
        got = list(g.score_batches((c.tuple() for c in chunks), both_strands=True))
        for c, r in zip(chunks, got):
            w = g.score_batch(c.tuple(), both_strands=True)
            assert np.array_equal(r.results, w.results) and np.array_equal(r.ties, w.ties)
    pairs, _ = synth.pairs_c4(refs, n=6000)
    pch = [pairs.slice(2 * k, 2 * (k + 1500)) for k in range(0, 6000, 1500)]
    cfg = adapter.config()
    with GpuScorer(refs, Scoring(), Mode.SEMIGLOBAL) as g:
        got = list(g.score_pair_batches((c.tuple() for c in pch), adapters=cfg))
        for c, r in zip(pch, got):
            w = g.finish_pairs(g.submit(g.prepare_pairs(c.tuple(), adapters=cfg)))
            assert np.array_equal(r.pairs, w.pairs) and np.array_equal(r.pair_ties, w.pair_ties)
