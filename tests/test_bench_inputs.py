"""The bench's synthetic inputs for the BAM runs are well-formed: the
unaligned BAM of C2 reads and the two FASTQ files of C4 pairs parse back,
through the oracle's readers, to the reads they were made from; and the
bench's CPU arm hands the library the oracle's mappings unchanged."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from eschalign_b200 import synth  # noqa: E402


def test_unmapped_bam_round_trip(tmp_path):
    from oracle import bam as B
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=1500)
    p = str(tmp_path / "in.bam")
    bench.unmapped_bam(p, reads)
    _, _, recs = B.read_bam(open(p, "rb").read())
    assert len(recs) == len(reads)
    for k in (0, 1, 700, 1499):
        r = recs[k]
        assert r["seq"] == bytes(b"ACGTN"[int(c)] for c in reads.read(k))
        assert r["name"] == b"r%07d" % k and r["flag"] == 4 and len(r["qual"]) == len(r["seq"])
        assert all(2 <= q <= 40 for q in r["qual"])


def test_fastq_files_round_trip(tmp_path):
    from oracle import bam as B
    refs = synth.panel_tiles()
    pairs, _ = synth.pairs_c4(refs, n=800)
    a, b = str(tmp_path / "1.fq"), str(tmp_path / "2.fq")
    bench.fastq_files(a, b, pairs)
    got = B.read_pairs(open(a, "rb").read(), open(b, "rb").read())
    assert len(got) == 800
    for k in (0, 399, 799):
        for m in range(2):
            assert got[k][m]["seq"] == bytes(b"ACGTN"[int(c)] for c in pairs.read(2 * k + m))
            assert got[k][m]["name"] == b"p%07d" % k


def test_cpu_arm_mappings_are_the_oracles(oracle):
    """bench's dict-to-array conversion keeps every field of every hit."""
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=300)
    letters = [bytes(b"ACGTN"[int(c)] for c in r) for r in refs]
    m = bench.CpuMapper(refs, (2, -1, -10, -1), True).map_reads(
        reads.tuple(), both_strands=True, ref_letters=letters)
    res, jobs, al, ops, mds, nm, _ = oracle.cpu_map_reads(
        *reads.tuple(), refs, (2, -1, -10, -1), True, both_strands=True, ref_letters=letters)
    want = oracle.cpu_mappings(res, jobs, al, ops, mds, nm)
    assert [m.mapping(k) for k in range(len(want))] == want
    assert np.all(m.reads["n_hits"] == [len(w["hits"]) for w in want])
