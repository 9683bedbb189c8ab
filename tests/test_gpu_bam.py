"""The CLI's unpaired run end to end on the CUDA path: the reference's fixture
BAM read by esg_bam_read_batch, mapped by esg_map_reads on the device, its
records built by esg_bam_encode and written by esg_bam_writer must hold the
record stream the reference CLI wrote -- record count and FNV-1a 64 digest
(crates/eschalign-cli/tests/align_unpaired.rs:37-62) -- for each of its six
flag sets."""
import pytest

from eschalign_b200 import GpuScorer, Mode, Scoring, encode
from eschalign_b200 import bam as EB
from tests.test_bam_golden import flag_set, golden_digests, trna_panel
from tests.test_bam_native import FIXTURE, record_stream

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("batch_size", [1000, 13])
@pytest.mark.parametrize("label", sorted(golden_digests()))
def test_align_bam_writes_the_reference_record_stream(tmp_path, label, batch_size):
    from oracle import bam as B
    want = golden_digests()[label]
    o = flag_set(label)
    names, refs = trna_panel()
    mode = Mode.LOCAL if o["local"] else Mode.SEMIGLOBAL
    path = str(tmp_path / "out.bam")
    with GpuScorer([encode(r) for r in refs], Scoring(*o["scoring"]), mode) as g:
        n = EB.align_bam(g, FIXTURE, path, names, refs, min_score=o["min_score"],
                         max_ties=o["max_ties"], both_strands=o["both"],
                         secondary=o["secondary"], sort_coordinate=o["sort"],
                         max_read_len=o["max_read_len"], batch_size=batch_size, threads=4)
    assert n["records"] == want["records"]
    assert format(B.fnv1a64(record_stream(path)), "016x") == want["fnv1a64"]


@pytest.mark.parametrize("label", ["default", "semiglobal_both_secondary", "sort_coordinate"])
def test_align_bam_fastq_gz_input(oracle, tmp_path, label):
    """The fixture's reads as gzip FASTQ through the same run: the records
    the oracle builds for the FASTQ records (read_fastx + build_records, in
    coordinate order when sorting)."""
    import gzip

    from oracle import bam as B
    from tests.test_bam_fastx import fastq_of
    from tests.test_bam_golden import input_records
    o = flag_set(label)
    names, refs = trna_panel()
    text = gzip.compress(fastq_of(input_records()))
    src, dst = str(tmp_path / "reads.fq.gz"), str(tmp_path / "out.bam")
    open(src, "wb").write(text)
    recs = B.read_fastx(text)
    ms = oracle.map_reads([r["seq"] for r in recs], refs, o["scoring"], o["local"],
                          min_score=o["min_score"], max_ties=o["max_ties"],
                          both_strands=o["both"])
    want = [x for r, m in zip(recs, ms) for x in B.build_records(r, m, names, o["secondary"])]
    if o["sort"]:
        want = B.coordinate_order(want)
    mode = Mode.LOCAL if o["local"] else Mode.SEMIGLOBAL
    with GpuScorer([encode(r) for r in refs], Scoring(*o["scoring"]), mode) as g:
        n = EB.align_bam(g, src, dst, names, refs, min_score=o["min_score"],
                         max_ties=o["max_ties"], both_strands=o["both"],
                         secondary=o["secondary"], sort_coordinate=o["sort"], batch_size=11)
    assert n["reads"] == len(recs) and n["records"] == len(want)
    assert record_stream(dst) == b"".join(want)


PAIR_CASES = [{}, {"secondary": True, "both": True}, {"max_insert": 120},
              {"trim": False, "local": True}, {"sort": True, "secondary": True}]


@pytest.mark.parametrize("extra", PAIR_CASES, ids=[str(c) for c in PAIR_CASES])
def test_align_pairs_bam_equals_the_oracle(oracle, tmp_path, extra):
    """The CLI's paired run on the CUDA path (align_pairs_bam: the mate
    files read, trimmed by esg_pair_adapters, mapped by esg_map_pairs,
    encoded and written) holds the records of the oracle's restatement,
    which pins what align_paired.rs asserts; batches of 3 pairs."""
    from oracle import bam as B
    from tests.test_bam_pairs import fastq_texts, fixture, opts, run_oracle
    extra = dict(extra)
    sort = extra.pop("sort", False)
    o = opts(**extra)
    refs, _ = fixture()
    names = [r["name"] for r in refs]
    letters = [r["seq"].encode() for r in refs]
    r1, r2 = fastq_texts()
    p1, p2, dst = str(tmp_path / "r1.fq"), str(tmp_path / "r2.fq"), str(tmp_path / "o.bam")
    open(p1, "wb").write(r1)
    open(p2, "wb").write(r2)
    want = run_oracle(oracle, o, r1, r2)
    if sort:
        want = B.coordinate_order(want)
    mode = Mode.LOCAL if o["local"] else Mode.SEMIGLOBAL
    with GpuScorer([encode(r) for r in letters], Scoring(*o["scoring"]), mode) as g:
        n = EB.align_pairs_bam(g, p1, p2, dst, names, letters, min_score=o["min_score"],
                               max_ties=o["max_ties"], max_insert=o["max_insert"],
                               both_strands=o["both"], secondary=o["secondary"],
                               sort_coordinate=sort,
                               adapters=EB.DEFAULT_ADAPTERS if o["trim"] else None,
                               batch_size=6)
    assert n["reads"] == 18 and n["records"] == len(want)
    assert record_stream(dst) == b"".join(want)
