"""FASTA / FASTQ input of the BAM stage (esg_bam_open sniffing the format,
esg_bam_read_batch taking each record as an unmapped read), on the CPU.

Pinned on the reference's own unit answers for its FASTX reader
(crates/eschalign-cli/src/align.rs:2958-2982) and on its end-to-end claim
that FASTQ input (plain or gzip) gives the records uBAM input gives
(crates/eschalign-cli/tests/align_e2e.rs:293-350); the library's records
must equal the oracle's restatement (oracle/bam.py read_fastx +
build_records) byte for byte."""
import gzip
import re
import struct

import pytest

from eschalign_b200 import bam as EB
from tests.test_bam_golden import flag_set, input_records, trna_panel
from tests.test_bam_native import FIXTURE, mappings_from_oracle

EMPTY = {"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []}


def split_records(stream: bytes):
    out, at = [], 0
    while at < len(stream):
        n = 4 + struct.unpack("<I", stream[at:at + 4])[0]
        out.append(stream[at:at + n])
        at += n
    return out


def library_records(path, maps, names, secondary=False, max_read_len=1000, batch=7):
    """Every record the library writes for `path` with the given mappings
    (one per read, in order), as separate byte strings."""
    out = []
    with EB.BamReader(path) as rd:
        k = 0
        for b in rd.batches(batch, max_read_len):
            rec = EB.encode(b, mappings_from_oracle(maps[k:k + len(b)]), names, secondary)
            out += split_records(rec.bytes())
            k += len(b)
    assert k == len(maps)
    return out


def oracle_records(recs, maps, names, secondary=False):
    from oracle import bam as B
    out = []
    for r, m in zip(recs, maps):
        out += B.build_records(r, m, names, secondary)
    return out


def fastq_of(recs, crlf=False, comment=True):
    nl = "\r\n" if crlf else "\n"
    text = ""
    for r in recs:
        qual = "".join(chr(q + 33) for q in r["qual"]) if r["qual"][:1] != b"\xff" else \
            "I" * len(r["seq"])
        text += f"@{r['name'].decode()}{' comment' if comment else ''}{nl}" \
                f"{r['seq'].decode()}{nl}+{nl}{qual}{nl}"
    return text.encode()


def test_oracle_reader_known_answers():
    """align.rs:2958-2982: normalise_seq, FASTA line joining, FASTQ Phred."""
    from oracle import bam as B
    assert B.normalise_seq(b"acguNx*") == b"ACGTNNN"
    recs = B.read_fastx(b">a desc\nACG\nTT\n\n>b\nGG\n")
    assert [(r["name"], r["seq"], r["qual"]) for r in recs] == [(b"a", b"ACGTT", b""),
                                                                (b"b", b"GG", b"")]
    (r,) = B.read_fastx(b"@r1 x=1\nACGT\n+\nII#!\n")
    assert (r["name"], r["seq"], list(r["qual"])) == (b"r1", b"ACGT", [40, 40, 2, 0])


def test_library_reader_known_answers(tmp_path):
    """The same answers through esg_bam_open / esg_bam_encode (unmapped)."""
    from oracle import bam as B
    cases = [(b">a desc\nACG\nTT\n\n>b\nGG\n", [(b"a", b"ACGTT", None), (b"b", b"GG", None)]),
             (b"@r1 x=1\nACGT\n+\nII#!\n", [(b"r1", b"ACGT", [40, 40, 2, 0])]),
             (b">n\nacguNx*\n", [(b"n", b"ACGTNNN", None)])]
    for k, (text, want) in enumerate(cases):
        p = str(tmp_path / f"in{k}")
        open(p, "wb").write(text)
        got = library_records(p, [EMPTY] * len(want), ["r0"])
        _, _, parsed = B.read_bam(gzip.compress(b"BAM\1" + bytes(8) + b"".join(got)))
        assert [(r["name"], r["seq"]) for r in parsed] == [(n, s) for n, s, _ in want]
        for r, (_, s, q) in zip(parsed, want):
            assert r["flag"] == 4 and r["aux"] == []
            assert list(r["qual"]) == (q if q is not None else [255] * len(s))


@pytest.mark.parametrize("kind", ["fastq", "fastq.gz", "fastq_crlf", "fasta", "fasta.gz"])
def test_fastx_records_equal_the_oracle(oracle, tmp_path, kind):
    """The fixture reads as FASTQ / FASTA (gzip or not, CRLF lines, blank
    lines, multi-line FASTA, lower case, U and non-BAM letters), mapped by
    the oracle, encoded by the library: the oracle's bytes."""
    from oracle import bam as B
    names, refs = trna_panel()
    recs = input_records()
    if kind.startswith("fastq"):
        text = fastq_of(recs, crlf=kind.endswith("crlf"))
    else:
        text = b""
        for k, r in enumerate(recs):
            s = r["seq"].decode()
            if k % 3 == 0:
                s = s.lower()
            if k % 5 == 1:
                s = s.replace("T", "U")
            if k % 7 == 2:
                s = s[:5] + "x*" + s[5:]
            text += f">{r['name'].decode()}\tdesc\n".encode()
            text += "\n".join(s[i:i + 60] for i in range(0, len(s), 60)).encode() + b"\n\n"
    if kind.endswith(".gz"):
        text = gzip.compress(text)
    path = str(tmp_path / "in")
    open(path, "wb").write(text)
    want_recs = B.read_fastx(text)
    assert len(want_recs) == len(recs)
    for label in ("semiglobal_both_secondary", "default"):
        o = flag_set(label)
        ms = oracle.map_reads([r["seq"] for r in want_recs], refs, o["scoring"], o["local"],
                              min_score=o["min_score"], max_ties=o["max_ties"],
                              both_strands=o["both"])
        got = library_records(path, ms, names, o["secondary"])
        assert got == oracle_records(want_recs, ms, names, o["secondary"])


def test_fastq_input_matches_ubam_input(oracle, tmp_path):
    """align_e2e.rs:293-350: FASTQ of the fixture's reads (plain and gzip)
    gives the uBAM input's records -- name, flags, position, MAPQ, CIGAR,
    sequence, qualities and the owned tags -- and gzip changes nothing."""
    from oracle import bam as B
    names, refs = trna_panel()
    recs = input_records()
    text = fastq_of(recs)
    fq, fqgz = str(tmp_path / "reads.fq"), str(tmp_path / "reads.fastq.gz")
    open(fq, "wb").write(text)
    open(fqgz, "wb").write(gzip.compress(text, 1))
    o = flag_set("default")
    ms = oracle.map_reads([r["seq"] for r in recs], refs, o["scoring"], o["local"])
    from_bam = library_records(FIXTURE, ms, names)
    from_fq = library_records(fq, ms, names)
    assert library_records(fqgz, ms, names) == from_fq
    hdr = b"BAM\1" + bytes(8)
    _, _, xb = B.read_bam(gzip.compress(hdr + b"".join(from_bam)))
    _, _, xf = B.read_bam(gzip.compress(hdr + b"".join(from_fq)))
    assert len(xb) == len(xf) == len(recs)
    for a, b, ra, rb in zip(xb, xf, from_bam, from_fq):
        assert (a["name"], a["flag"], a["seq"], a["qual"]) == (b["name"], b["flag"], b["seq"],
                                                              b["qual"])
        assert ra[4:20] == rb[4:20]  # reference, position, name length, MAPQ, bin, CIGAR count, flag
        cig = 36 + ra[12]
        n_cig = struct.unpack("<H", ra[16:18])[0]
        assert ra[cig:cig + 4 * n_cig] == rb[cig:cig + 4 * n_cig]
        owned = (b"NM", b"MD", b"AS", b"XS", b"XA")
        assert [f for t, f in a["aux"] if t in owned] == [f for t, f in b["aux"] if t in owned]


@pytest.mark.parametrize("text,why", [
    (b"@r1\nACGT\nII\nIIII\n", "expected '+'"),
    (b"@r1\nACGT\n+\nIII\n", "quality values"),
    (b"@r1\nACGT\n", "expected '+'"),
    (b"@r1\nACGT\n+\n", "before quality"),
    (b"ACGT\n", "not a BAM, FASTA or FASTQ"),
    (b"\n\n   \n", "not a BAM, FASTA or FASTQ"),
    (b">a\nAC\n@b\n", None),
    (b"BAM\1" + bytes(8), "uncompressed BAM"),
])
def test_fastx_errors(tmp_path, text, why):
    """Malformed input is an error status, as the CLI's reader bails
    (align.rs:496-520); a FASTA record may hold any line not starting '>'."""
    p = str(tmp_path / "bad")
    open(p, "wb").write(text)
    if why is None:
        got = library_records(p, [EMPTY], ["r0"])
        assert len(got) == 1
        return
    with pytest.raises(RuntimeError, match=re.escape(why)):
        with EB.BamReader(p) as rd:
            list(rd.batches(10, 0))
