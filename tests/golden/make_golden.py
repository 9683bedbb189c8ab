"""Extract golden vectors for the panel-scoring path from the reference's own fixtures.

Run once, in a container where the reference tree is mounted:

    python tests/golden/make_golden.py <reference checkout>

It reads, as data:

* ``crates/eschalign/tests/fixtures/align_golden.json`` -- parasail 1.3.4
  (``sw_trace`` / ``sg_trace``) scores for 48 pairs x {local, semiglobal} x
  {``2,-1,-10,-1``, ``1,-1,-2,-1``}, generated by the reference's
  ``gen_align_golden.py`` (seed 395) and checked by its
  ``tests/parasail_golden.rs:48-77``;
* ``crates/eschalign-cli/tests/fixtures/trna_reference.fa`` and
  ``trna_reference_ambiguous.fa`` -- the 47-reference tRNA panels the
  reference's ``tests/gpu_parity.rs:249-260`` scores the fixture reads against;
* ``crates/eschalign-cli/tests/fixtures/pairs/pairs_panel.fa``,
  ``pairs_R1.fq`` and ``pairs_R2.fq`` -- the 4-reference paired-end fixture
  (``gen_pair_fixture.py``, seed 20261004) the reference's
  ``tests/align_paired.rs`` aligns.

* ``crates/eschalign/tests/fixtures/calmd_golden.json`` -- MD / NM that
  samtools calmd wrote for 21 CIGARs over reference ``N``, IUPAC, lower case
  and ``U`` (the reference's ``gen_calmd_golden.py``, checked by its
  ``tests/sam_fields.rs``);
* ``crates/eschalign-cli/tests/fixtures/trna_mappings_padded.bam`` and
  ``unpaired_golden.tsv`` -- the 60-record input BAM the reference's
  ``tests/align_unpaired.rs`` aligns against ``trna_reference.fa`` under six
  flag sets, and for each the record count and FNV-1a 64 digest of the
  uncompressed output record stream its binary wrote;

and writes the subset this project tests against into ``tests/golden/``
(the input BAM's bytes unchanged as ``unpaired_input.bam``, the digests as
``unpaired_golden.json``):
``align_golden_scores.json`` (query, reference, mode, scheme, score and the
parasail end coordinates), the two panels as ``panel_trna*.json`` (name +
letters, file order) and the paired fixture as ``pairs_fixture.json`` (panel
and each pair's name and mate letters), and the calmd records as
``calmd_golden.json``.  Nothing else from the reference is copied.
"""
import json
import os
import sys


def read_fasta(path):
    """Minimal FASTA reader: first word of the header, sequence lines joined."""
    recs, name, seq = [], None, []
    with open(path, "rb") as fh:
        for raw in fh:
            line = raw.rstrip(b"\r\n")
            if line.startswith(b">"):
                if name is not None:
                    recs.append((name, b"".join(seq).decode()))
                words = line[1:].split()
                name, seq = words[0].decode(), []
            elif name is not None:
                seq.append(b"".join(line.split()))
    if name is not None:
        recs.append((name, b"".join(seq).decode()))
    return recs


def main(ref_root):
    here = os.path.dirname(os.path.abspath(__file__))
    src = os.path.join(ref_root, "crates/eschalign/tests/fixtures/align_golden.json")
    with open(src) as fh:
        g = json.load(fh)
    cases = []
    for p in g["pairs"]:
        for r in p["results"]:
            cases.append({
                "name": p["name"],
                "source": p["source"],
                "query": p["query"],
                "reference": p["reference"],
                "mode": r["mode"],
                "scheme": g["schemes"][r["scheme"]],
                "score": r["score"],
                "query_start": r["query_start"],
                "query_end": r["query_end"],
                "ref_start": r["ref_start"],
                "ref_end": r["ref_end"],
            })
    out = {
        "about": "parasail 1.3.4 golden scores (reference fixture align_golden.json, seed 395)",
        "cases": cases,
        "fixture_reads": [p["query"] for p in g["pairs"] if p["source"] != "random"],
    }
    with open(os.path.join(here, "align_golden_scores.json"), "w") as fh:
        json.dump(out, fh, indent=0)
    for fa, tag in (("trna_reference.fa", "panel_trna.json"),
                    ("trna_reference_ambiguous.fa", "panel_trna_ambiguous.json")):
        recs = read_fasta(os.path.join(ref_root, "crates/eschalign-cli/tests/fixtures", fa))
        with open(os.path.join(here, tag), "w") as fh:
            json.dump({"source": fa, "references": [{"name": n, "seq": s} for n, s in recs]},
                      fh, indent=0)
    pdir = os.path.join(ref_root, "crates/eschalign-cli/tests/fixtures/pairs")
    mates = []
    for fq in ("pairs_R1.fq", "pairs_R2.fq"):
        with open(os.path.join(pdir, fq)) as fh:
            lines = fh.read().splitlines()
        mates.append([(lines[i][1:], lines[i + 1], lines[i + 3])
                      for i in range(0, len(lines), 4)])
    pairs = [{"name": a[0], "r1": a[1], "r2": b[1], "q1": a[2], "q2": b[2]}
             for a, b in zip(*mates)]
    panel = read_fasta(os.path.join(pdir, "pairs_panel.fa"))
    with open(os.path.join(here, "pairs_fixture.json"), "w") as fh:
        json.dump({"source": "pairs/pairs_panel.fa, pairs_R1.fq, pairs_R2.fq",
                   "references": [{"name": n, "seq": s} for n, s in panel],
                   "pairs": pairs}, fh, indent=0)
    with open(os.path.join(ref_root, "crates/eschalign/tests/fixtures/calmd_golden.json")) as fh:
        cm = json.load(fh)
    with open(os.path.join(here, "calmd_golden.json"), "w") as fh:
        json.dump({"about": "MD/NM as samtools calmd wrote them (reference fixture "
                            "calmd_golden.json, " + str(cm.get("samtools", "")) + ")",
                   "reference": cm["reference"]["seq"],
                   "records": [{k: r[k] for k in ("name", "pos", "cigar", "seq", "md", "nm")}
                               for r in cm["records"]]}, fh, indent=0)
    fix = os.path.join(ref_root, "crates/eschalign-cli/tests/fixtures")
    with open(os.path.join(fix, "trna_mappings_padded.bam"), "rb") as fh:
        bam = fh.read()
    with open(os.path.join(here, "unpaired_input.bam"), "wb") as fh:
        fh.write(bam)
    rows = {}
    with open(os.path.join(fix, "unpaired_golden.tsv")) as fh:
        for line in fh:
            if line.strip():
                label, n, digest = line.split()
                rows[label] = {"records": int(n), "fnv1a64": digest}
    with open(os.path.join(here, "unpaired_golden.json"), "w") as fh:
        json.dump({"about": "records and FNV-1a 64 digest of the uncompressed BAM record "
                            "stream (header skipped) the reference CLI wrote for "
                            "unpaired_input.bam against the trna panel, per flag set "
                            "(reference fixture unpaired_golden.tsv, test align_unpaired.rs)",
                   "flags": {"default": [], "semiglobal_both_secondary":
                             ["--mode", "semiglobal", "--strand", "both", "--secondary"],
                             "sort_coordinate": ["--sort", "coordinate"],
                             "min_score_max_ties": ["--min-score", "60", "--max-ties", "1"],
                             "scoring_bwa": ["--scoring", "1,-1,-2,-1", "--strand", "both"],
                             "max_read_len": ["--max-read-len", "60"]},
                   "digests": rows}, fh, indent=1)
    print(f"{len(cases)} golden scores, {len(out['fixture_reads'])} fixture reads, "
          f"{len(pairs)} fixture pairs, {len(cm['records'])} calmd records")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    main(sys.argv[1])
