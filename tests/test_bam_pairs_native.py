"""The library's paired BAM stage (esg_bam_open_pairs, esg_bam_read_pair_batch,
esg_bam_encode_pairs, the writer) against the oracle's restatement of the
CLI's paired run, byte for byte, on the CPU: the mappings are the oracle's
(handed over with esg_mapping_from_arrays + esg_mapping_set_pairs), the
adapters the library's own esg_pair_adapters (equal to the oracle's by
test), so everything else -- pair reading, placements, records -- is the
library's."""
import gzip

import numpy as np
import pytest

from eschalign_b200 import adapter as A
from eschalign_b200 import bam as EB
from eschalign_b200.scorer import (HIT_DTYPE, MAPPING_DTYPE, MAPPING_HAS_BEST,
                                   MAPPING_HAS_SUBOPTIMAL, PAIR_HIT_DTYPE, PAIR_MAPPING_DTYPE,
                                   Mappings)
from tests.test_bam_fastx import split_records
from tests.test_bam_pairs import (bgzf, fastq_texts, fixture, interleaved_text, opts,
                                  paired_ubam, run_oracle)

_OPS = "MIDNSHP=X"


def _hit(h, ops, md):
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
    return e


def pair_mappings_from_oracle(pms) -> Mappings:
    """The oracle's map_pairs dicts as esg_map_pairs' arrays."""
    n = len(pms)
    reads = np.zeros(2 * n, MAPPING_DTYPE)
    pairs = np.zeros(n, PAIR_MAPPING_DTYPE)
    hits, phits, ops, md = [], [], [], bytearray()
    for p, pm in enumerate(pms):
        if pm["proper"]:
            pr = pairs[p]
            pr["flags"] = 1 | (2 if pm["suboptimal"][0] is not None else 0) | \
                (4 if pm["suboptimal"][1] is not None else 0)
            pr["score"], pr["n_tied"], pr["n_hits"] = pm["score"], pm["n_tied"], len(pm["hits"])
            pr["suboptimal"] = [x if x is not None else 0 for x in pm["suboptimal"]]
            pr["first_hit"] = len(phits)
            for h in pm["hits"]:
                e = np.zeros((), PAIR_HIT_DTYPE)
                e["reference"], e["reverse"], e["insert"] = h["reference"], h["reverse"], \
                    h["insert"]
                e["mates"][0] = _hit(h["mates"][0], ops, md)
                e["mates"][1] = _hit(h["mates"][1], ops, md)
                phits.append(e)
            continue
        for m, mm in enumerate(pm["mates"]):
            r = reads[2 * p + m]
            r["first_hit"], r["n_hits"], r["n_tied"] = len(hits), len(mm["hits"]), mm["n_tied"]
            if mm["best_score"] is not None:
                r["best_score"], r["flags"] = mm["best_score"], r["flags"] | MAPPING_HAS_BEST
            if mm["suboptimal"] is not None:
                r["suboptimal"] = mm["suboptimal"]
                r["flags"] |= MAPPING_HAS_SUBOPTIMAL
            hits += [_hit(h, ops, md) for h in mm["hits"]]
    return Mappings(reads, np.array(hits, HIT_DTYPE), np.array(ops, np.uint32), bytes(md),
                    pairs, np.array(phits, PAIR_HIT_DTYPE))


def oracle_pms(oracle, o, pairs_letters, ads):
    """The oracle's map_pairs over the mates as the library trims them."""
    refs, _ = fixture()
    letters = [r["seq"].encode() for r in refs]
    mates = []
    for (a, b), ad in zip(pairs_letters, ads):
        for s, x in ((a, ad[0]), (b, ad[1])):
            over = o["max_read_len"] and len(s) > o["max_read_len"]
            mates.append(b"" if over else s[:len(s) - x])
    return oracle.map_pairs([(mates[2 * i], mates[2 * i + 1]) for i in range(len(pairs_letters))],
                            letters, o["scoring"], o["local"], min_score=o["min_score"],
                            max_ties=o["max_ties"], max_insert=o["max_insert"],
                            both_strands=o["both"])


def library_records(oracle, o, path1, path2=None, max_pairs=4):
    """Every record the library writes for the pairs of path1 (/ path2), the
    mappings the oracle's."""
    refs, _ = fixture()
    names = [r["name"] for r in refs]
    cfg = None
    if o["trim"]:
        cfg = A.config(o["adapters"][0], o["adapters"][1], o["min_overlap"], o["max_read_len"])
    out = []
    with EB.PairReader(path1, path2) as rd:
        for b in rd.batches(max_pairs):
            codes, off, lens = b.reads()
            if cfg is not None:
                ads, _ = A.pair_adapters((codes, off, lens), cfg)
            else:
                ads = np.zeros(len(lens), np.uint32)
            letters = [bytes(b"ACGTN"[int(c)] for c in codes[int(off[k]):int(off[k] + lens[k])])
                       for k in range(len(lens))]
            pms = oracle_pms(oracle, o, [(letters[2 * i], letters[2 * i + 1])
                                         for i in range(len(lens) // 2)],
                             [(int(ads[2 * i]), int(ads[2 * i + 1]))
                              for i in range(len(lens) // 2)])
            rec = EB.encode_pairs(b, pair_mappings_from_oracle(pms), names,
                                  ads if cfg is not None else None, o["secondary"])
            out += split_records(rec.bytes())
    return out


def test_library_adapters_equal_the_oracle(oracle):
    """esg_pair_adapters on the fixture equals the oracle's pair_adapters."""
    _, pairs = fixture()
    mates = [s.encode() for p in pairs for s in (p["r1"], p["r2"])]
    from eschalign_b200 import encode
    ads, _ = A.pair_adapters([encode(m) for m in mates], A.config())
    want = [x for p in pairs for x in oracle.pair_adapters(p["r1"].encode(), p["r2"].encode())]
    assert ads.tolist() == want


CASES = [{}, {"secondary": True, "both": True}, {"max_insert": 120}, {"trim": False},
         {"local": True, "trim": False, "secondary": True}, {"max_read_len": 55},
         {"max_ties": 0, "secondary": True}]


@pytest.mark.parametrize("extra", CASES, ids=[str(c) for c in CASES])
def test_paired_records_equal_the_oracle(oracle, tmp_path, extra):
    o = opts(**extra)
    r1, r2 = fastq_texts()
    p1, p2 = str(tmp_path / "r1.fq"), str(tmp_path / "r2.fq")
    open(p1, "wb").write(r1)
    open(p2, "wb").write(r2)
    want = run_oracle(oracle, o, r1, r2)
    assert library_records(oracle, o, p1, p2) == want


def test_paired_outcomes(oracle, tmp_path):
    """The run summary per mate (Outcome, align.rs:1420-1423): the oracle's
    placements give each mate unique, tied or unmapped."""
    from oracle import bam as B
    o = opts(both=True)
    r1, r2 = fastq_texts()
    p1, p2 = str(tmp_path / "r1.fq"), str(tmp_path / "r2.fq")
    open(p1, "wb").write(r1)
    open(p2, "wb").write(r2)
    refs, _ = fixture()
    names = [r["name"] for r in refs]
    got = {"unique": 0, "tied": 0, "unmapped": 0}
    want = dict(got)
    with EB.PairReader(p1, p2) as rd:
        for b in rd.batches(100):
            codes, off, lens = b.reads()
            ads, _ = A.pair_adapters((codes, off, lens), A.config())
            letters = [bytes(b"ACGTN"[int(c)] for c in codes[int(off[k]):int(off[k] + lens[k])])
                       for k in range(len(lens))]
            pms = oracle_pms(oracle, o, [(letters[2 * i], letters[2 * i + 1])
                                         for i in range(len(lens) // 2)],
                             [(int(ads[2 * i]), int(ads[2 * i + 1]))
                              for i in range(len(lens) // 2)])
            rec = EB.encode_pairs(b, pair_mappings_from_oracle(pms), names, ads)
            for k, v in rec.outcomes().items():
                got[k] += v
            for pm in pms:
                for pl in B.pair_placements(pm)[0]:
                    want["unmapped" if pl["primary"] is None else
                         ("unique" if pl["unique"] else "tied")] += 1
    assert got == want and sum(got.values()) == 18


@pytest.mark.parametrize("form", ["interleaved", "ubam", "gz_suffixed"])
def test_paired_input_forms(oracle, tmp_path, form):
    """align_paired.rs:462-505 through the library's readers: interleaved
    FASTQ, paired uBAM and gzip mate files with /1 /2 give the two-file
    records."""
    o = opts(secondary=True, both=True)
    r1, r2 = fastq_texts()
    want = run_oracle(oracle, o, r1, r2)
    if form == "interleaved":
        p = str(tmp_path / "il.fq")
        open(p, "wb").write(interleaved_text())
        got = library_records(oracle, o, p)
    elif form == "ubam":
        p = str(tmp_path / "pairs.ubam")
        open(p, "wb").write(paired_ubam())
        got = library_records(oracle, o, p)
    else:
        s1, s2 = fastq_texts(suffix=True, comment=" extra words")
        p1, p2 = str(tmp_path / "a_1.fq.gz"), str(tmp_path / "a_2.fq.gz")
        open(p1, "wb").write(gzip.compress(s1))
        open(p2, "wb").write(gzip.compress(s2))
        got = library_records(oracle, o, p1, p2)
    assert got == want


def test_paired_ubam_tags(oracle, tmp_path):
    """align_paired.rs:603-631: input tags kept on both mates, a stale NM
    replaced -- the oracle's bytes."""
    p = str(tmp_path / "tagged.ubam")
    data = paired_ubam(tags=True)
    open(p, "wb").write(data)
    assert library_records(oracle, opts(), p) == run_oracle(oracle, opts(), data)


def test_paired_orphans_are_errors(tmp_path):
    """align_paired.rs:507-601: the library names the read left over."""
    r1, r2 = fastq_texts()
    f1 = str(tmp_path / "full.fq")
    open(f1, "wb").write(r1)
    cases = []
    short = str(tmp_path / "short.fq")
    open(short, "wb").write(b"\n".join(r2.split(b"\n")[:-5]) + b"\n")
    cases.append((f1, short, "plain"))
    lines = r2.split(b"\n")
    sw = str(tmp_path / "swapped.fq")
    open(sw, "wb").write(b"\n".join(lines[4:8] + lines[0:4] + lines[8:]))
    cases.append((f1, sw, "pair_tie"))
    il = str(tmp_path / "il.fq")
    open(il, "wb").write(interleaved_text() + b"@lonely\nACGTACGTACGTACGTACGT\n+\n" + b"I" * 20
                         + b"\n")
    cases.append((il, None, "lonely"))
    from oracle import bam as B
    lost = str(tmp_path / "lost.bam")
    _, _, recs = B.read_bam(paired_ubam())
    body = b"".join(B.encode_record(-1, -1, 0, [], r["flag"], r["name"], r["seq"], r["qual"],
                                    [f for _, f in r["aux"]]) for r in recs[:-1])
    open(lost, "wb").write(bgzf(b"BAM\1" + bytes(8) + body))
    cases.append((lost, None, "plain"))
    for a, b, who in cases:
        with pytest.raises(RuntimeError, match=who):
            with EB.PairReader(a, b) as rd:
                list(rd.batches(100))


def test_paired_writer_sorts_mates_consistently(oracle, tmp_path):
    """align_paired.rs:633-688 through the writer: the coordinate-sorted
    file holds the oracle's coordinate order."""
    from oracle import bam as B
    from tests.test_bam_native import record_stream
    o = opts(secondary=True, both=True)
    r1, r2 = fastq_texts()
    p1, p2 = str(tmp_path / "r1.fq"), str(tmp_path / "r2.fq")
    open(p1, "wb").write(r1)
    open(p2, "wb").write(r2)
    recs = library_records(oracle, o, p1, p2)
    refs, _ = fixture()
    names = [r["name"] for r in refs]
    out = str(tmp_path / "s.bam")
    # push the library's records through the writer in two chunks
    with EB.PairReader(p1, p2) as rd, EB.BamWriter(out, b"", names,
                                                   [len(r["seq"]) for r in refs], True) as wr:
        for seq, b in enumerate(rd.batches(5)):
            codes, off, lens = b.reads()
            ads, _ = A.pair_adapters((codes, off, lens), A.config())
            letters = [bytes(b"ACGTN"[int(c)] for c in codes[int(off[k]):int(off[k] + lens[k])])
                       for k in range(len(lens))]
            pms = oracle_pms(oracle, o, [(letters[2 * i], letters[2 * i + 1])
                                         for i in range(len(lens) // 2)],
                             [(int(ads[2 * i]), int(ads[2 * i + 1]))
                              for i in range(len(lens) // 2)])
            wr.push(seq, EB.encode_pairs(b, pair_mappings_from_oracle(pms), names, ads, True))
    assert record_stream(out) == b"".join(B.coordinate_order(recs))


def test_proper_pair_without_a_pair_hit_is_refused():
    """A caller's paired mapping whose Proper pair lists no pair hit has
    nothing to place the mates by: esg_mapping_set_pairs refuses it."""
    from eschalign_b200 import bam as EB
    pm = {"proper": True, "score": 10, "n_tied": 1, "suboptimal": [None, None], "hits": []}
    m = pair_mappings_from_oracle([pm])
    m.pair_hits = np.zeros(0, m.pair_hits.dtype)
    with pytest.raises(RuntimeError, match="proper but has no pair hit"):
        EB.mapping_handle(m)
