"""The reference CLI's unpaired BAM output, pinned on its own golden digests.

crates/eschalign-cli/tests/align_unpaired.rs runs the eschalign binary on its
60-record fixture BAM against the tRNA panel under six flag sets and checks
the record count and the FNV-1a 64 digest of the uncompressed record stream
(tests/golden/unpaired_golden.json).  Here the oracle's restatement of the
CLI's record building and encoding (oracle/bam.py), over the oracle's
mappings, must give the same bytes for every flag set."""
import json
import os

import pytest

from tests.helpers import GOLDEN

SCHEMES = {"scoring_bwa": (1, -1, -2, -1)}


def flag_set(label):
    """(scoring, local, both_strands, secondary, sort, min_score, max_ties,
    max_read_len) of a golden flag set (the CLI's defaults otherwise:
    align.rs:133-289, mode local for unpaired input, align.rs:1923-1927)."""
    f = json.load(open(os.path.join(GOLDEN, "unpaired_golden.json")))["flags"][label]
    opt = dict(scoring=(2, -1, -10, -1), local=True, both=False, secondary=False, sort=False,
               min_score=0, max_ties=None, max_read_len=1000)
    i = 0
    while i < len(f):
        k = f[i]
        if k == "--secondary":
            opt["secondary"] = True
            i += 1
            continue
        v = f[i + 1]
        if k == "--mode":
            opt["local"] = v == "local"
        elif k == "--strand":
            opt["both"] = v == "both"
        elif k == "--sort":
            opt["sort"] = v == "coordinate"
        elif k == "--scoring":
            opt["scoring"] = tuple(int(x) for x in v.split(","))
        elif k == "--min-score":
            opt["min_score"] = int(v)
        elif k == "--max-ties":
            opt["max_ties"] = int(v)
        elif k == "--max-read-len":
            opt["max_read_len"] = int(v)
        i += 2
    return opt


def golden_digests():
    return json.load(open(os.path.join(GOLDEN, "unpaired_golden.json")))["digests"]


def trna_panel():
    d = json.load(open(os.path.join(GOLDEN, "panel_trna.json")))
    return [r["name"] for r in d["references"]], [r["seq"].encode() for r in d["references"]]


def input_records():
    from oracle import bam as B
    with open(os.path.join(GOLDEN, "unpaired_input.bam"), "rb") as fh:
        _, _, recs = B.read_bam(fh.read())
    return B.input_reads(recs)


@pytest.mark.parametrize("label", sorted(golden_digests()))
def test_oracle_reproduces_the_reference_record_stream(oracle, label):
    from oracle import bam as B
    want = golden_digests()[label]
    o = flag_set(label)
    names, refs = trna_panel()
    recs = input_records()
    keep = [k for k, r in enumerate(recs)
            if not (o["max_read_len"] and len(r["seq"]) > o["max_read_len"])]
    ms = oracle.map_reads([recs[k]["seq"] for k in keep], refs, o["scoring"], o["local"],
                          min_score=o["min_score"], max_ties=o["max_ties"],
                          both_strands=o["both"])
    maps = [{"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []} for _ in recs]
    for k, m in zip(keep, ms):
        maps[k] = m
    out = []
    for r, m in zip(recs, maps):
        out += B.build_records(r, m, names, o["secondary"])
    if o["sort"]:
        out = B.coordinate_order(out)
    assert len(out) == want["records"]
    assert format(B.fnv1a64(b"".join(out)), "016x") == want["fnv1a64"]
