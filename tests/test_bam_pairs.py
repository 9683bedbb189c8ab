"""The CLI's paired run as records: the oracle's restatement (oracle/bam.py
read_pairs, pair_placements, build_pair_records over the oracle's
map_pairs) pinned on what crates/eschalign-cli/tests/align_paired.rs asserts
for its paired fixture, on the CPU.  The library's paired BAM stage is
checked against the same restatement byte for byte (test_bam_pairs_native
and the GPU tests)."""
import json
import os
import struct

import pytest

from tests.helpers import GOLDEN

STD = dict(scoring=(2, -1, -10, -1), local=False, both=False, secondary=False, min_score=40,
           max_ties=None, max_insert=500, trim=True, max_read_len=1000,
           adapters=(b"AGATCGGAAGAGCACACGTCTGAACTCCAGTCA", b"AGATCGGAAGAGCGTCGTGTAGGGAAAGAGTGT"),
           min_overlap=5)
CIGAR_OPS = "MIDNSHP=X"


def fixture():
    d = json.load(open(os.path.join(GOLDEN, "pairs_fixture.json")))
    return d["references"], d["pairs"]


def fastq_texts(suffix=False, comment=""):
    """The fixture's two mate files (pairs_R1.fq, pairs_R2.fq)."""
    _, pairs = fixture()
    t1 = "".join(f"@{p['name']}{'/1' if suffix else ''}{comment}\n{p['r1']}\n+\n{p['q1']}\n"
                 for p in pairs)
    t2 = "".join(f"@{p['name']}{'/2' if suffix else ''}{comment}\n{p['r2']}\n+\n{p['q2']}\n"
                 for p in pairs)
    return t1.encode(), t2.encode()


def interleaved_text():
    _, pairs = fixture()
    return "".join(f"@{p['name']}\n{p['r1']}\n+\n{p['q1']}\n@{p['name']}\n{p['r2']}\n+\n"
                   f"{p['q2']}\n" for p in pairs).encode()


def bgzf(raw: bytes) -> bytes:
    """`raw` as BGZF blocks of at most 0xff00 bytes, with the end-of-file
    block (a BAM file's compression)."""
    import zlib
    out = b""
    for i in range(0, len(raw), 0xff00):
        src = raw[i:i + 0xff00]
        c = zlib.compressobj(6, zlib.DEFLATED, -15)
        body = c.compress(src) + c.flush()
        out += (b"\x1f\x8b\x08\x04\0\0\0\0\0\xff\x06\0BC\x02\0" +
                struct.pack("<H", len(body) + 25) + body +
                struct.pack("<II", zlib.crc32(src), len(src)))
    return out + bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")


def paired_ubam(tags=False):
    """The fixture as an unaligned paired BAM (align_paired.rs:406-440):
    0x1 | 0x4 | 0x8 and 0x40 / 0x80, mates adjacent; with `tags`, a ZZ tag
    per record and a stale NM (align_paired.rs:603-631)."""
    from oracle import bam as B
    _, pairs = fixture()
    recs = b""
    k = 0
    for p in pairs:
        for m in range(2):
            seq, q = p["r1" if m == 0 else "r2"].encode(), p["q1" if m == 0 else "q2"]
            aux = []
            if tags:
                aux = [B.str_field(b"ZZ", f"tag{k}"), B.int_field(b"NM", 99)]
            recs += B.encode_record(-1, -1, 0, [], 0x1 | 0x4 | 0x8 | (0x40 if m == 0 else 0x80),
                                    p["name"].encode(), seq, bytes(ord(c) - 33 for c in q), aux)
            k += 1
    hdr = b"BAM\1" + struct.pack("<I", 0) + struct.pack("<I", 0)
    return bgzf(hdr + recs)


def run_oracle(oracle, o, data1, data2=None):
    """The paired run in the oracle: read, trim, map_pairs, build records."""
    from oracle import bam as B
    refs, _ = fixture()
    names = [r["name"] for r in refs]
    letters = [r["seq"].encode() for r in refs]
    pairs = B.read_pairs(data1, data2)
    mates, ads = [], []
    for a, b in pairs:
        if o["trim"]:
            ad = oracle.pair_adapters(a["seq"], b["seq"], *o["adapters"], o["min_overlap"],
                                      o["max_read_len"])
        else:
            ad = [0, 0]
        ads.append(ad)
        for r, x in ((a, ad[0]), (b, ad[1])):
            over = o["max_read_len"] and len(r["seq"]) > o["max_read_len"]
            mates.append(b"" if over else r["seq"][:len(r["seq"]) - x])
    pms = oracle.map_pairs([(mates[2 * i], mates[2 * i + 1]) for i in range(len(pairs))],
                           letters, o["scoring"], o["local"], min_score=o["min_score"],
                           max_ties=o["max_ties"], max_insert=o["max_insert"],
                           both_strands=o["both"])
    out = []
    for (a, b), pm, ad in zip(pairs, pms, ads):
        out += B.build_pair_records([a, b], pm, ad if o["trim"] else None, names, o["secondary"])
    return out


def parse(rec: bytes) -> dict:
    """A BAM record's fields (block_size included in `rec`)."""
    from oracle import bam as B
    (ref, pos, lrn, mapq, bin_, ncig, flag, lseq, mref, mpos, tlen) = struct.unpack(
        "<iiBBHHHIiii", rec[4:36])
    p = 36
    name = rec[p:p + lrn - 1].decode()
    p += lrn
    cig = "".join(f"{w >> 4}{CIGAR_OPS[w & 15]}" for w in struct.unpack(f"<{ncig}I",
                                                                         rec[p:p + 4 * ncig]))
    p += 4 * ncig
    sb = rec[p:p + (lseq + 1) // 2]
    seq = bytes(B.SEQ_CODES[(sb[k // 2] >> (0 if k % 2 else 4)) & 15] for k in range(lseq))
    p += (lseq + 1) // 2
    qual = rec[p:p + lseq]
    p += lseq
    tags = {}
    for t, f in B.split_aux(rec[p:]):
        ty = f[2:3]
        if ty == b"Z":
            tags[t.decode()] = f[3:-1].decode()
        else:
            fmt = {b"C": "<B", b"c": "<b", b"S": "<H", b"s": "<h", b"I": "<I", b"i": "<i"}[ty]
            tags[t.decode()] = struct.unpack(fmt, f[3:])[0]
    return {"name": name, "flag": flag, "ref": ref, "pos": pos + 1 if pos >= 0 else None,
            "mapq": mapq, "bin": bin_, "cigar": cig, "mate_ref": mref,
            "mate_pos": mpos + 1 if mpos >= 0 else None, "tlen": tlen, "seq": seq,
            "qual": qual, "tags": tags}


def mates(recs, pair):
    """align_paired.rs:147-157: mate 1 then mate 2, adjacent."""
    rs = [parse(r) for r in recs]
    i = next(k for k, r in enumerate(rs) if r["name"] == pair and r["flag"] & 0x40)
    a, b = rs[i], rs[i + 1]
    assert b["name"] == pair and b["flag"] & 0x80
    return a, b


def refname(r):
    refs, _ = fixture()
    return refs[r["ref"]]["name"] if r["ref"] >= 0 else None


def opts(**kw):
    o = dict(STD)
    o.update(kw)
    return o


def test_pair_resolves_paralog_tie(oracle):
    """align_paired.rs:188-243."""
    r1, r2 = fastq_texts()
    recs = run_oracle(oracle, opts(), r1, r2)
    a, b = mates(recs, "paralog")
    for r in (a, b):
        assert refname(r) == "P1" and r["mapq"] == 60 and "XA" not in r["tags"]
    assert a["tags"]["XS"] == a["tags"]["AS"]
    assert a["flag"] == 0x1 | 0x2 | 0x20 | 0x40
    assert b["flag"] == 0x1 | 0x2 | 0x10 | 0x80
    assert (a["pos"], b["pos"]) == (21, 91)
    assert (a["mate_pos"], a["tlen"], b["tlen"]) == (91, 130, -130)
    assert a["tags"]["MC"] == "60M"
    _, pairs = fixture()
    q2 = next(p["q2"] for p in pairs if p["name"] == "paralog")
    assert bytes(q + 33 for q in b["qual"]).decode() == q2[::-1]


def test_pair_tie_is_reported_in_xa_and_secondaries(oracle):
    """align_paired.rs:245-272."""
    r1, r2 = fastq_texts()
    a, b = mates(run_oracle(oracle, opts(), r1, r2), "pair_tie")
    for r in (a, b):
        assert r["mapq"] == 0 and refname(r) == "P1" and r["tags"]["XA"].startswith("P2,")
    secs = [parse(r) for r in run_oracle(oracle, opts(secondary=True), r1, r2)]
    secs = [r for r in secs if r["name"] == "pair_tie" and r["flag"] & 0x100]
    assert len(secs) == 2
    assert secs[0]["flag"] & 0x40 and secs[1]["flag"] & 0x80
    assert refname(secs[0]) == "P2" and secs[0]["mate_ref"] == secs[1]["ref"]
    assert secs[0]["flag"] & 0x2


def test_pair_insert_shorter_than_read(oracle):
    """align_paired.rs:274-294."""
    r1, r2 = fastq_texts()
    a, b = mates(run_oracle(oracle, opts(), r1, r2), "short_insert")
    assert refname(a) == "U1"
    assert (a["tlen"], b["tlen"]) == (40, -40)
    assert (a["cigar"], b["cigar"]) == ("40M20S", "20S40M")
    assert (a["pos"], b["pos"]) == (31, 31) and a["flag"] & 0x2
    assert (a["tags"]["MC"], b["tags"]["MC"]) == ("20S40M", "40M20S")
    assert len(a["seq"]) == len(b["seq"]) == 60


def test_pair_adapter_tag_counts(oracle):
    """align_paired.rs:296-338."""
    r1, r2 = fastq_texts()
    recs = run_oracle(oracle, opts(), r1, r2)

    def ad(pair, rs=recs):
        a, b = mates(rs, pair)
        return a["tags"].get("ad"), b["tags"].get("ad")
    assert ad("short_insert") == (20, 20)
    assert ad("one_mate_reads_through") == (15, 0)
    assert ad("plain") == (0, 0)
    a, b = mates(recs, "one_mate_reads_through")
    assert (a["cigar"], b["cigar"], a["tlen"]) == ("40M15S", "35M", 40)
    off = [parse(r) for r in run_oracle(oracle, opts(trim=False), r1, r2)]
    assert all("ad" not in r["tags"] for r in off)
    custom = run_oracle(oracle, opts(adapters=(b"T" * 16, b"T" * 16)), r1, r2)
    assert mates(custom, "short_insert")[0]["tags"]["ad"] == 0
    hi = run_oracle(oracle, opts(min_overlap=16), r1, r2)
    assert mates(hi, "one_mate_reads_through")[0]["tags"]["ad"] == 0


def test_pair_terminal_mismatch_not_clipped(oracle):
    """align_paired.rs:340-362."""
    refs, _ = fixture()
    u1 = next(r["seq"] for r in refs if r["name"] == "U1")
    r1, r2 = fastq_texts()
    a, b = mates(run_oracle(oracle, opts(), r1, r2), "terminal_mismatch")
    assert a["cigar"] == "60M" and a["tags"]["NM"] == 1
    assert a["tags"]["MD"] == f"59{u1[69]}0"
    assert b["cigar"] == "60M" and b["tags"]["NM"] == 1 and b["tags"]["MD"].endswith("0")
    a, _ = mates(run_oracle(oracle, opts(local=True), r1, r2), "terminal_mismatch")
    assert a["cigar"] == "59M1S"


def test_pair_over_max_insert_not_proper(oracle):
    """align_paired.rs:364-381."""
    r1, r2 = fastq_texts()
    a, b = mates(run_oracle(oracle, opts(max_insert=120), r1, r2), "over_max_insert")
    assert not a["flag"] & 0x2 and not b["flag"] & 0x2
    assert refname(a) == refname(b) == "U1"
    assert a["flag"] == 0x1 | 0x20 | 0x40 and b["flag"] == 0x1 | 0x10 | 0x80
    assert a["tlen"] == 150
    a, b = mates(run_oracle(oracle, opts(), r1, r2), "over_max_insert")
    assert a["flag"] & 0x2 and b["flag"] & 0x2


def test_pair_wrong_orientation_and_unmapped_mate(oracle):
    """align_paired.rs:383-403."""
    r1, r2 = fastq_texts()
    recs = run_oracle(oracle, opts(), r1, r2)
    a, b = mates(recs, "wrong_orientation")
    assert not a["flag"] & 0x2 and not b["flag"] & 0x2
    assert refname(a) == refname(b) == "U2"
    assert a["flag"] == 0x1 | 0x40 and b["flag"] == 0x1 | 0x80
    a, b = mates(recs, "one_unmapped")
    assert a["flag"] == 0x1 | 0x8 | 0x40 and b["flag"] == 0x1 | 0x4 | 0x80
    assert (b["ref"], b["pos"], b["mapq"]) == (a["ref"], a["pos"], 0)


@pytest.mark.parametrize("extra", [{}, {"both": True, "secondary": True}])
def test_pair_inputs_agree(oracle, extra):
    """align_paired.rs:462-505: two files, interleaved and paired uBAM give
    the same records; /1 /2 suffixes and comments change nothing."""
    import gzip
    r1, r2 = fastq_texts()
    o = opts(**extra)
    files = run_oracle(oracle, o, r1, r2)
    assert len(files) >= 18
    assert run_oracle(oracle, o, interleaved_text()) == files
    assert run_oracle(oracle, o, paired_ubam()) == files
    s1, s2 = fastq_texts(suffix=True, comment=" extra words")
    assert run_oracle(oracle, opts(trim=False, **extra), gzip.compress(s1), gzip.compress(s2)) \
        == run_oracle(oracle, opts(trim=False, **extra), r1, r2)


def test_pair_orphans_are_errors():
    """align_paired.rs:507-601: the left-over read is named."""
    from oracle import bam as B
    r1, r2 = fastq_texts()
    short = b"\n".join(r2.split(b"\n")[:-5]) + b"\n"  # the last record dropped
    with pytest.raises(ValueError, match="plain.*no mate"):
        B.read_pairs(r1, short)
    lines = r2.split(b"\n")
    swapped = b"\n".join(lines[4:8] + lines[0:4] + lines[8:])
    with pytest.raises(ValueError, match="paralog.*pair_tie|pair_tie.*paralog"):
        B.read_pairs(r1, swapped)
    with pytest.raises(ValueError, match="lonely.*no mate"):
        B.read_pairs(interleaved_text() + b"@lonely\nACGTACGTACGTACGTACGT\n+\n" + b"I" * 20
                     + b"\n")


def test_pair_ubam_tags_are_copied_on_both_mates(oracle):
    """align_paired.rs:603-631."""
    recs = [parse(r) for r in run_oracle(oracle, opts(), paired_ubam(tags=True))]
    assert len(recs) == 18
    for k, r in enumerate(recs):
        assert r["tags"]["ZZ"] == f"tag{k}" and r["tags"].get("NM") != 99


@pytest.mark.parametrize("extra", [{}, {"secondary": True, "both": True}])
def test_pair_sort_coordinate_model(oracle, extra):
    """align_paired.rs:633-688: the coordinate order is a stable sort on
    (reference, position, reverse), no reference last, and each record's
    mate fields point at its partner's place."""
    from oracle import bam as B
    r1, r2 = fastq_texts()
    recs = run_oracle(oracle, opts(**extra), r1, r2)
    srt = B.coordinate_order(recs)
    model = sorted(recs, key=lambda r: ((parse(r)["ref"] if parse(r)["ref"] >= 0 else 1 << 40),
                                        parse(r)["pos"] or 0, bool(parse(r)["flag"] & 0x10)))
    assert srt == model
    rs = [parse(r) for r in srt]
    for r in rs:
        if r["flag"] & 0x100:
            continue
        partner = next(p for p in rs if p["name"] == r["name"] and not p["flag"] & 0x100
                       and bool(p["flag"] & 0x40) != bool(r["flag"] & 0x40))
        if not r["flag"] & 0x8:
            assert (r["mate_pos"], r["mate_ref"]) == (partner["pos"], partner["ref"])
