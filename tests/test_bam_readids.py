"""--read-ids through the library's readers (esg_bam_set_read_ids), on the CPU.

Restates crates/eschalign-cli/tests/align_e2e.rs:393-438 (every 7th read of
the fixture selected by a dashed ID list, and the same reads by the dashless
list) and checks the selection against the oracle's load_read_ids /
canonical_read_name / select_reads (align.rs:572-621, uuid_util.rs:10-30),
for single reads and for pairs."""
import pytest

from eschalign_b200 import bam as EB
from tests.test_bam_fastx import split_records
from tests.test_bam_golden import input_records, trna_panel
from tests.test_bam_native import FIXTURE, mappings_from_oracle

EMPTY = {"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []}


def selected_names(path, ids_path):
    """The names of the records the library writes for the reads its reader
    keeps (unmapped), and the reader's counts."""
    refs, _ = trna_panel()
    names = []
    with EB.BamReader(path, read_ids=ids_path) as rd:
        for b in rd.batches(5, 0):
            rec = EB.encode(b, mappings_from_oracle([EMPTY] * len(b)), refs)
            names += [r[36:36 + r[12] - 1] for r in split_records(rec.bytes())]
        counts = rd.counts()
    return names, counts


@pytest.mark.parametrize("form", ["dashed", "dashless"])
def test_read_ids_select_reads(tmp_path, form):
    """align_e2e.rs:393-438."""
    recs = input_records()
    wanted = [r["name"] for r in recs[::7]]
    ids = [w.replace(b"-", b"") if form == "dashless" else w for w in wanted]
    p = tmp_path / "ids.txt"
    p.write_bytes(b"\n".join(ids) + b"\n")
    got, counts = selected_names(FIXTURE, str(p))
    assert got == wanted
    assert counts == {"not_primary": 0, "filtered": len(recs) - len(wanted)}


def test_read_ids_spellings_comments_and_the_oracle(tmp_path):
    """Upper case, braced and urn:uuid: spellings, comments, blank lines and
    trailing words: the oracle's selection."""
    from oracle import bam as B
    recs = input_records()
    picks = recs[1::5]
    lines = [b"# a comment", b""]
    for k, r in enumerate(picks):
        n = r["name"]
        form = k % 4
        if form == 0:
            lines.append(n.upper() + b"  trailing words")
        elif form == 1:
            lines.append(b"{" + n + b"}")
        elif form == 2:
            lines.append(b"urn:uuid:" + n)
        else:
            lines.append(b"   " + n.replace(b"-", b"") + b"\t")
    lines.append(b"not-a-read")
    p = tmp_path / "ids.txt"
    p.write_bytes(b"\r\n".join(lines))
    wanted = B.load_read_ids(p.read_bytes())
    want = [r["name"] for r in B.select_reads(recs, wanted)]
    assert want == [r["name"] for r in picks]
    got, _ = selected_names(FIXTURE, str(p))
    assert got == want


def test_read_ids_oracle_known_answers():
    """uuid_util.rs's forms and a plain name (align.rs:572-583)."""
    from oracle import bam as B
    u = b"a1b2c3d4-e5f6-7890-abcd-ef1234567890"
    for s in (u, u.upper(), u.replace(b"-", b""), b"{" + u + b"}", b"urn:uuid:" + u):
        assert B.canonical_read_name(s) == u
    for s in (b"read_1", b"a1b2c3d4e5f67890abcdef123456789", b"{" + u):
        assert B.canonical_read_name(s) == s


def test_read_ids_empty_list_is_an_error(tmp_path):
    p = tmp_path / "ids.txt"
    p.write_bytes(b"# only a comment\n\n")
    with pytest.raises(RuntimeError, match="no read names"):
        EB.BamReader(FIXTURE, read_ids=str(p))


def test_read_ids_select_pairs_by_name(tmp_path):
    """read_pair_batches (align.rs:875-905): pairs kept by the pair's name,
    whatever /1 /2 the mates carry; two reads counted per pair dropped."""
    from oracle import bam as B
    from tests.test_bam_pairs import fastq_texts
    s1, s2 = fastq_texts(suffix=True)
    p1, p2 = tmp_path / "a_1.fq", tmp_path / "a_2.fq"
    p1.write_bytes(s1)
    p2.write_bytes(s2)
    ids = tmp_path / "ids.txt"
    ids.write_bytes(b"paralog\nplain\n")
    want = B.read_pairs(s1, s2, B.load_read_ids(ids.read_bytes()))
    assert [a["name"] for a, _ in want] == [b"paralog", b"plain"]
    with EB.PairReader(str(p1), str(p2), read_ids=str(ids)) as rd:
        got = sum(len(b) for b in rd.batches(4))
        counts = rd.counts()
    assert got == 4 and counts["filtered"] == 2 * (9 - 2)
