"""The library's BAM stage (esg_bam_*) against the reference CLI's golden
record streams, on the CPU.

The reader parses the reference's 60-record fixture; the encoder builds each
read's records from its mapping (here the oracle's mappings, handed over with
esg_mapping_from_arrays, so no GPU is needed) and must give the record count
and FNV-1a 64 digest the reference CLI gave for each of its six flag sets
(crates/eschalign-cli/tests/align_unpaired.rs:37-62).  The writer's BGZF file
must decompress to the same stream, in input or coordinate order."""
import gzip
import os
import struct

import numpy as np
import pytest

from eschalign_b200 import bam as EB
from eschalign_b200.scorer import (HIT_DTYPE, MAPPING_DTYPE, MAPPING_HAS_BEST,
                                   MAPPING_HAS_SUBOPTIMAL, Mappings)
from tests.helpers import GOLDEN
from tests.test_bam_golden import flag_set, golden_digests, input_records, trna_panel

FIXTURE = os.path.join(GOLDEN, "unpaired_input.bam")
_OPS = "MIDNSHP=X"


def mappings_from_oracle(ms) -> Mappings:
    """The oracle's map_reads dicts as esg_map_reads' arrays."""
    reads = np.zeros(len(ms), MAPPING_DTYPE)
    hits, ops, md = [], [], bytearray()
    for k, m in enumerate(ms):
        r = reads[k]
        r["first_hit"] = len(hits)
        r["n_hits"] = len(m["hits"])
        r["n_tied"] = m["n_tied"]
        if m["best_score"] is not None:
            r["best_score"] = m["best_score"]
            r["flags"] |= MAPPING_HAS_BEST
        if m["suboptimal"] is not None:
            r["suboptimal"] = m["suboptimal"]
            r["flags"] |= MAPPING_HAS_SUBOPTIMAL
        for h in m["hits"]:
            e = np.zeros((), HIT_DTYPE)
            for f in ("reference", "reverse", "score", "query_start", "query_end", "ref_start",
                      "ref_end", "nm"):
                e[f] = int(h[f])
            words, n = [], ""
            for ch in h["cigar"]:
                if ch.isdigit():
                    n += ch
                else:
                    words.append(int(n) << 4 | _OPS.index(ch))
                    n = ""
            e["ops_offset"], e["n_ops"] = len(ops), len(words)
            ops += words
            e["md_offset"], e["md_len"] = len(md), len(h["md"])
            md += h["md"].encode()
            hits.append(e)
    return Mappings(reads, np.array(hits, HIT_DTYPE), np.array(ops, np.uint32), bytes(md))


def oracle_mappings(oracle, recs, o):
    names, refs = trna_panel()
    keep = [k for k, r in enumerate(recs)
            if not (o["max_read_len"] and len(r["seq"]) > o["max_read_len"])]
    ms = oracle.map_reads([recs[k]["seq"] for k in keep], refs, o["scoring"], o["local"],
                          min_score=o["min_score"], max_ties=o["max_ties"],
                          both_strands=o["both"])
    out = [{"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []} for _ in recs]
    for k, m in zip(keep, ms):
        out[k] = m
    return out


def record_stream(path):
    """The uncompressed records of a BAM file, header skipped."""
    raw = gzip.decompress(open(path, "rb").read())
    lt = struct.unpack("<I", raw[4:8])[0]
    o = 8 + lt
    n_ref = struct.unpack("<I", raw[o:o + 4])[0]
    o += 4
    for _ in range(n_ref):
        o += 8 + struct.unpack("<I", raw[o:o + 4])[0]
    return raw[o:]


def test_reader_gives_the_primary_records_as_codes():
    from eschalign_b200 import encode
    recs = input_records()
    with EB.BamReader(FIXTURE, threads=2) as rd:
        assert rd.header_text.startswith(b"@")
        batches = list(rd.batches(max_reads=17, max_read_len=1000))
    assert [len(b) for b in batches] == [17, 17, 17, len(recs) - 51]
    got = []
    for b in batches:
        codes, off, lens = b.reads()
        got += [codes[int(off[k]):int(off[k]) + int(lens[k])].tolist() for k in range(len(b))]
    assert got == [encode(r["seq"]).tolist() for r in recs]


def test_reader_leaves_long_reads_unscored():
    recs = input_records()
    with EB.BamReader(FIXTURE) as rd:
        (b,) = list(rd.batches(max_reads=1000, max_read_len=40))
    assert b.lens.tolist() == [0 if len(r["seq"]) > 40 else len(r["seq"]) for r in recs]


@pytest.mark.parametrize("label", sorted(golden_digests()))
def test_encoder_reproduces_the_reference_record_stream(oracle, label):
    from oracle import bam as B
    want = golden_digests()[label]
    o = flag_set(label)
    names, _ = trna_panel()
    recs = input_records()
    maps = mappings_from_oracle(oracle_mappings(oracle, recs, o))
    with EB.BamReader(FIXTURE) as rd:
        (b,) = list(rd.batches(max_reads=1000, max_read_len=o["max_read_len"]))
    rec = EB.encode(b, maps, names, secondary=o["secondary"], threads=3)
    stream = rec.bytes()
    if o["sort"]:
        parts, at = [], 0
        while at < len(stream):
            n = 4 + struct.unpack("<I", stream[at:at + 4])[0]
            parts.append(stream[at:at + n])
            at += n
        stream = b"".join(B.coordinate_order(parts))
    assert rec.n_records == want["records"]
    assert format(B.fnv1a64(stream), "016x") == want["fnv1a64"]


@pytest.mark.parametrize("label", ["default", "sort_coordinate", "semiglobal_both_secondary"])
def test_writer_file_holds_the_reference_record_stream(oracle, tmp_path, label):
    """Chunks pushed out of order; the file is BGZF with the end marker and
    decompresses to the golden stream (coordinate-sorted by the writer)."""
    from oracle import bam as B
    want = golden_digests()[label]
    o = flag_set(label)
    names, refs = trna_panel()
    recs = input_records()
    ms = oracle_mappings(oracle, recs, o)
    path = str(tmp_path / "out.bam")
    hdr = EB.header_text(names, [len(r) for r in refs], o["sort"])
    chunks = []
    with EB.BamReader(FIXTURE) as rd:
        for seq, b in enumerate(rd.batches(max_reads=7, max_read_len=o["max_read_len"])):
            lo = seq * 7
            chunks.append(EB.encode(b, mappings_from_oracle(ms[lo:lo + len(b)]), names,
                                    secondary=o["secondary"]))
    with EB.BamWriter(path, hdr, names, [len(r) for r in refs], o["sort"], threads=2) as wr:
        for seq in [2, 0, 1] + list(range(3, len(chunks))):
            wr.push(seq, chunks[seq])
    data = open(path, "rb").read()
    assert data[-28:] == bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")
    text, refs_out, out_recs = B.read_bam(data)
    assert text == hdr and [n.decode() for n, _ in refs_out] == names
    assert len(out_recs) == want["records"]
    assert format(B.fnv1a64(record_stream(path)), "016x") == want["fnv1a64"]


def test_writer_refuses_a_repeated_chunk(tmp_path):
    names, refs = trna_panel()
    with EB.BamReader(FIXTURE) as rd:
        (b,) = list(rd.batches(max_reads=1000))
    empty = {"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []}
    rec = EB.encode(b, mappings_from_oracle([empty] * len(b)), names)
    wr = EB.BamWriter(str(tmp_path / "x.bam"), b"", names, [len(r) for r in refs])
    wr.push(0, rec)
    with pytest.raises(RuntimeError):
        wr.push(0, rec)
    wr.close()
    assert len(record_stream(str(tmp_path / "x.bam"))) == rec.nbytes


def test_encoder_refuses_a_mapping_of_other_reads():
    names, _ = trna_panel()
    with EB.BamReader(FIXTURE) as rd:
        (b,) = list(rd.batches(max_reads=1000))
    empty = {"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []}
    with pytest.raises(RuntimeError):
        EB.encode(b, mappings_from_oracle([empty] * (len(b) - 1)), names)


def test_mapping_from_arrays_checks_its_offsets():
    m = mappings_from_oracle([{"best_score": 5, "n_tied": 1, "suboptimal": None, "hits": [
        {"reference": 0, "reverse": False, "score": 5, "query_start": 0, "query_end": 3,
         "ref_start": 0, "ref_end": 3, "cigar": "3M", "md": "3", "nm": 0}]}])
    m.hits["md_len"] = 2 ** 32 - 1
    with pytest.raises(RuntimeError):
        EB.mapping_handle(m)
    m.hits["md_len"] = 1
    m.reads["first_hit"] = 2 ** 64 - 1
    with pytest.raises(RuntimeError):
        EB.mapping_handle(m)


@pytest.mark.parametrize("field,value,why", [
    ("reverse", 2, "strand"), ("query_end", 3, "CIGAR does not span"),
    ("ref_end", 6, "CIGAR does not span"), ("query_start", 5, "start is past its end")])
def test_mapping_from_arrays_checks_each_hit(field, value, why):
    """A caller's hit must be one a traceback could give: strand 0 / 1,
    starts before ends, CIGAR words spanning its read and reference
    coordinates; anything else is refused before the encoder sees it."""
    from eschalign_b200 import _native
    # 2M1D1I1M: 4 read bases (0..4) and 4 reference bases (1..5)
    hit = {"reference": 0, "reverse": False, "score": 5, "query_start": 0, "query_end": 4,
           "ref_start": 1, "ref_end": 5, "cigar": "2M1D1I1M", "md": "2^A1", "nm": 2}

    def mapping():
        return mappings_from_oracle([{"best_score": 5, "n_tied": 1, "suboptimal": None,
                                      "hits": [dict(hit)]}])

    _native.load().esg_mapping_free(EB.mapping_handle(mapping()))  # consistent: taken
    m = mapping()
    m.hits[field] = value
    with pytest.raises(RuntimeError, match=why):
        EB.mapping_handle(m)
    m = mapping()
    m.ops[0] = (2 << 4) | 9  # no BAM op 9
    with pytest.raises(RuntimeError, match="past X"):
        EB.mapping_handle(m)


class OracleScorer:
    """A stand-in for GpuScorer.map_reads that maps with the oracle, so the
    pipeline of align_bam runs on the CPU."""

    def __init__(self, oracle, refs, scoring, local):
        self.oracle, self.refs, self.scoring, self.local = oracle, refs, scoring, local
        self.calls = 0

    def map_reads(self, reads, min_score=0, max_ties=None, both_strands=False, ref_letters=None,
                  raw=False):
        codes, off, lens = reads
        letters = [bytes(b"ACGTN"[int(c)] for c in codes[int(o):int(o) + int(n)])
                   for o, n in zip(off, lens)]
        self.calls += 1
        ms = self.oracle.map_reads(letters, self.refs, self.scoring, self.local,
                                   min_score=min_score, max_ties=max_ties,
                                   both_strands=both_strands)
        return mappings_from_oracle(ms)


@pytest.mark.parametrize("n_scorers", [1, 2])
@pytest.mark.parametrize("label", sorted(golden_digests()))
def test_align_bam_pipeline_writes_the_reference_record_stream(oracle, tmp_path, label,
                                                               n_scorers):
    """align_bam's overlapped read / map / encode / write, in batches of 13,
    with the oracle's mappings: the golden stream, input order kept."""
    from oracle import bam as B
    want = golden_digests()[label]
    o = flag_set(label)
    names, refs = trna_panel()
    scs = [OracleScorer(oracle, refs, o["scoring"], o["local"]) for _ in range(n_scorers)]
    path = str(tmp_path / "out.bam")
    st = {}
    n = EB.align_bam(scs if n_scorers > 1 else scs[0], FIXTURE, path, names, refs,
                     min_score=o["min_score"],
                     max_ties=o["max_ties"], both_strands=o["both"], secondary=o["secondary"],
                     sort_coordinate=o["sort"], max_read_len=o["max_read_len"], batch_size=13,
                     threads=3, stats=st)
    assert n["batches"] == sum(sc.calls for sc in scs) == 5 and n["reads"] == 60
    assert n["records"] == want["records"]
    assert format(B.fnv1a64(record_stream(path)), "016x") == want["fnv1a64"]
    assert set(st) == {"read", "map", "encode", "write"}
    # the run summary (Outcome, align.rs:1077-1082): from the oracle's mappings
    ms = oracle_mappings(oracle, input_records(), o)
    assert (n["unique"], n["tied"], n["unmapped"]) == (
        sum(1 for m in ms if m["hits"] and m["n_tied"] == 1),
        sum(1 for m in ms if m["hits"] and m["n_tied"] > 1),
        sum(1 for m in ms if not m["hits"]))


def test_corrupt_records_are_errors(tmp_path):
    """A record whose sequence length runs past its block, or whose B-array
    count runs past its tags, is an error status, not a read past the
    buffer."""
    import struct
    from oracle import bam as B
    from tests.test_bam_pairs import bgzf
    good = B.encode_record(-1, -1, 0, [], 4, b"r1", b"ACGT", b"IIII", [])
    bad_len = good[:20] + struct.pack("<I", 0xFFFFFFF0) + good[24:]
    p = tmp_path / "bad_len.bam"
    p.write_bytes(bgzf(b"BAM\1" + bytes(8) + bad_len))
    with pytest.raises(RuntimeError, match="malformed BAM record"):
        with EB.BamReader(str(p)) as rd:
            list(rd.batches(10, 0))
    arr = b"ZZBc" + struct.pack("<I", 0xFFFFFFF0) + b"\x01"
    bad_aux = B.encode_record(-1, -1, 0, [], 4, b"r2", b"ACGT", b"IIII", [arr])
    p = tmp_path / "bad_aux.bam"
    p.write_bytes(bgzf(b"BAM\1" + bytes(8) + bad_aux))
    names, _ = trna_panel()
    with EB.BamReader(str(p)) as rd:
        (b,) = list(rd.batches(10, 0))
        with pytest.raises(RuntimeError, match="malformed auxiliary"):
            EB.encode(b, mappings_from_oracle([{"best_score": None, "n_tied": 0,
                                                "suboptimal": None, "hits": []}]), names)


def test_corrupt_bgzf_is_an_error(tmp_path):
    """A BGZF block whose size field is too small, or whose stated inflated
    size is over 64 KiB, is an error status."""
    import struct
    from tests.test_bam_pairs import bgzf
    data = bytearray(bgzf(b"BAM\1" + bytes(8)))
    small = bytearray(data)
    small[16:18] = struct.pack("<H", 10)
    p = tmp_path / "small.bam"
    p.write_bytes(bytes(small))
    with pytest.raises(RuntimeError, match="BGZF"):
        EB.BamReader(str(p))
    bsize = struct.unpack("<H", data[16:18])[0] + 1
    big = bytearray(data)
    big[bsize - 4:bsize] = struct.pack("<I", 1 << 20)
    p = tmp_path / "big.bam"
    p.write_bytes(bytes(big))
    with pytest.raises(RuntimeError, match="BGZF|not a BAM"):
        EB.BamReader(str(p))


def test_output_header_carries_the_inputs_programs(oracle, tmp_path):
    """build_header (align.rs:1780-1808): @HD 1.6 with the sort order, the
    panel's @SQ lines, the input's @RG / @PG / @CO lines, and a @PG of its
    own after the input's last program."""
    from oracle import bam as B
    names, refs = trna_panel()
    with EB.BamReader(FIXTURE) as rd:
        text_in = rd.header_text
    h = EB.header_text(names, [len(r) for r in refs], True,
                       text_in + b"@RG\tID:grp1\tSM:s\n@CO\ta comment\n").decode().splitlines()
    assert h[0] == "@HD\tVN:1.6\tSO:coordinate"
    assert [x.split("\t")[1][3:] for x in h[1:1 + len(names)]] == names
    rest = h[1 + len(names):]
    assert rest[0] == "@RG\tID:grp1\tSM:s"
    assert [x for x in rest if x.startswith("@PG")][:3] == \
        [x for x in text_in.decode().splitlines() if x.startswith("@PG")]
    assert rest[-2] == "@PG\tID:eschalign-b200\tPN:eschalign-b200\tPP:samtools.1"
    assert rest[-1] == "@CO\ta comment"
    sc = OracleScorer(oracle, refs, (2, -1, -10, -1), True)
    out = str(tmp_path / "o.bam")
    EB.align_bam(sc, FIXTURE, out, names, refs)
    text_out, _, _ = B.read_bam(open(out, "rb").read())
    assert b"PP:samtools.1" in text_out and b"ID:bwa" in text_out


def test_encoder_refuses_a_hit_past_its_read(oracle):
    """A hit whose CIGAR is consistent but whose read coordinates run past
    the read (no traceback gives one) is refused by the encoder instead of
    becoming a record whose CIGAR and sequence disagree."""
    from eschalign_b200 import bam as EB
    o = flag_set("default")
    names, refs = trna_panel()
    ms = oracle_mappings(oracle, input_records(), o)
    with EB.BamReader(FIXTURE) as rd:
        b = next(iter(rd.batches(max_reads=7, max_read_len=o["max_read_len"])))
    m = mappings_from_oracle(ms[:len(b)])
    EB.encode(b, m, names)  # as traced: taken
    k = int(np.nonzero(m.reads["n_hits"])[0][0])
    h = int(m.reads["first_hit"][k])
    shift = int(b.reads()[2][k])  # the read's length
    m.hits["query_start"][h] += shift
    m.hits["query_end"][h] += shift
    with pytest.raises(RuntimeError, match="past the end of its read"):
        EB.encode(b, m, names)
