"""The C ABI from a compiled consumer: tests/c_consumer/unpaired_bam.c is
built with the C compiler against include/eschalign_b200.h and linked to
the library, as a binding in another compiled language would be, and runs
the host half of the CLI's unpaired run on the reference's 60-record
fixture BAM: the mapping arrays (the oracle's, for the flag set) handed over
with esg_mapping_from_arrays, records encoded and pushed to the writer out
of order.  The output must hold the record stream whose count and FNV-1a 64
digest the reference CLI gave for that flag set
(crates/eschalign-cli/tests/align_unpaired.rs:37-62).  No GPU is needed."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import eschalign_b200
from eschalign_b200 import _native
from eschalign_b200 import bam as EB
from tests.test_bam_golden import flag_set, golden_digests, input_records, trna_panel
from tests.test_bam_native import FIXTURE, mappings_from_oracle, oracle_mappings, record_stream

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def write_mapping(path, ms):
    """The mapping arrays as the C program reads them: four u64 counts, then
    the read, hit, CIGAR-word and MD arrays."""
    with open(path, "wb") as fh:
        fh.write(np.array([ms.reads.size, ms.hits.size, ms.ops.size, len(ms.md_bytes)],
                          np.uint64).tobytes())
        fh.write(ms.reads.tobytes() + ms.hits.tobytes() + ms.ops.tobytes() + ms.md_bytes)
    return path


@pytest.fixture(scope="module")
def consumer(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    eschalign_b200.load()  # builds the library when it is missing
    lib_dir = os.path.dirname(_native.LIB_PATH)
    exe = str(tmp_path_factory.mktemp("cabi") / "unpaired_bam")
    subprocess.run([cc, "-std=c11", "-O1", "-Wall", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "c_consumer", "unpaired_bam.c"),
                    "-o", exe, _native.LIB_PATH, f"-Wl,-rpath,{lib_dir}"], check=True)
    return exe


@pytest.mark.parametrize("label", ["default", "sort_coordinate", "semiglobal_both_secondary"])
def test_c_program_writes_the_reference_record_stream(oracle, consumer, tmp_path, label):
    from oracle import bam as B
    want = golden_digests()[label]
    o = flag_set(label)
    names, refs = trna_panel()
    ms = mappings_from_oracle(oracle_mappings(oracle, input_records(), o))
    mapping = write_mapping(tmp_path / "mapping.bin", ms)
    header = tmp_path / "header.txt"
    header.write_bytes(EB.header_text(names, [len(r) for r in refs], o["sort"]))
    refs_txt = tmp_path / "refs.txt"
    refs_txt.write_text("".join(f"{n} {len(r)}\n" for n, r in zip(names, refs)))
    out = str(tmp_path / "out.bam")
    run = subprocess.run([consumer, FIXTURE, out, str(header), str(refs_txt), str(mapping),
                          str(int(o["secondary"])), str(int(o["sort"])),
                          str(o["max_read_len"])], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    assert run.stdout.split() == ["records", str(want["records"])]
    text, refs_out, recs = B.read_bam(open(out, "rb").read())
    assert [n.decode() for n, _ in refs_out] == names and len(recs) == want["records"]
    assert format(B.fnv1a64(record_stream(out)), "016x") == want["fnv1a64"]


def test_c_program_refuses_a_short_mapping(oracle, consumer, tmp_path):
    """A mapping of fewer reads than the BAM holds is an error, not a crash."""
    names, refs = trna_panel()
    o = flag_set("default")
    ms = mappings_from_oracle(oracle_mappings(oracle, input_records(), o)[:5])
    mapping = write_mapping(tmp_path / "mapping.bin", ms)
    header = tmp_path / "header.txt"
    header.write_bytes(EB.header_text(names, [len(r) for r in refs]))
    refs_txt = tmp_path / "refs.txt"
    refs_txt.write_text("".join(f"{n} {len(r)}\n" for n, r in zip(names, refs)))
    run = subprocess.run([consumer, FIXTURE, str(tmp_path / "o.bam"), str(header),
                          str(refs_txt), str(mapping), "0", "0", "1000"],
                         capture_output=True, text=True, timeout=60)
    assert run.returncode == 1 and "more reads than the mapping" in run.stderr
