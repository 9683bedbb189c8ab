"""The BAM writer's blocks compressed on the device (esg_bam_writer_use_device,
k_bgzf_deflate): the file must hold the host writer's records, and every
block must be exactly what the compressor's steps give on the host
(esg_bgzf_deflate_host) for that block's bytes -- the kernel runs the same
steps, lane by lane, so its output is byte-identical, including the choice
of a stored block."""
import ctypes as C
import gzip
import struct
import zlib

import numpy as np
import pytest

from eschalign_b200 import GpuScorer, Mode, Scoring, _native, synth
from eschalign_b200 import bam as EB

pytestmark = pytest.mark.gpu

STORED = 0xFFFFFFFF


def _members(path):
    """(deflate data, crc, isize) of each BGZF member, the end marker last."""
    data = open(path, "rb").read()
    out, at = [], 0
    while at < len(data):
        assert data[at:at + 4] == b"\x1f\x8b\x08\x04"
        bsize = struct.unpack("<H", data[at + 16:at + 18])[0] + 1
        crc, isize = struct.unpack("<II", data[at + bsize - 8:at + bsize])
        out.append((data[at + 18:at + bsize - 8], crc, isize))
        at += bsize
    return out


def _host_steps(raw: bytes):
    lib = _native.load()
    out = np.zeros(65536 // 4, np.uint32)
    src = (C.c_uint8 * len(raw)).from_buffer_copy(raw)
    n = lib.esg_bgzf_deflate_host(src, len(raw), out.ctypes.data)
    return STORED if n == STORED else out.view(np.uint8)[:n].tobytes()


def _check_blocks(path):
    """Every block equals the host steps' output for its bytes; returns
    (blocks, stored)."""
    mem = _members(path)
    assert mem[-1][2] == 0  # the end marker
    n_stored = 0
    for cdata, crc, isize in mem[:-1]:
        raw = zlib.decompress(cdata, -15)
        assert len(raw) == isize and zlib.crc32(raw) == crc
        want = _host_steps(raw)
        if want == STORED:
            n_stored += 1
            assert cdata[0] == 1 and cdata[5:] == raw  # BFINAL, BTYPE 00, LEN, NLEN
        else:
            assert cdata == want
    return len(mem) - 1, n_stored


@pytest.fixture(scope="module")
def ubam(tmp_path_factory):
    import bench
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=30_000, seed=0x5EED_0DEF)
    path = str(tmp_path_factory.mktemp("defl") / "u.bam")
    bench.unmapped_bam(path, reads)
    return refs, path


@pytest.mark.parametrize("sort", [False, True])
def test_device_blocks_hold_the_host_writers_records(ubam, tmp_path, sort):
    from tests.test_bam_native import record_stream
    refs, src = ubam
    names = [f"ref{k}" for k in range(len(refs))]
    letters = [bytes(b"ACGTN"[int(c)] for c in r) for r in refs]
    dev, host = str(tmp_path / "dev.bam"), str(tmp_path / "host.bam")
    with GpuScorer(refs, Scoring(2, -1, -10, -1), Mode.LOCAL) as g:
        for path, on in ((dev, True), (host, False)):
            EB.align_bam(g, src, path, names, letters, both_strands=True, secondary=True,
                         sort_coordinate=sort, batch_size=7000, deflate_on_device=on)
    assert gzip.decompress(open(dev, "rb").read()) == gzip.decompress(open(host, "rb").read())
    assert len(record_stream(dev)) > 0
    blocks, stored = _check_blocks(dev)
    assert blocks > 50 and stored == 0
    # the host writer's blocks are zlib's, not the device's
    assert open(dev, "rb").read() != open(host, "rb").read()


def test_incompressible_blocks_are_stored(tmp_path):
    """A header of random letters does not compress: its blocks are written
    stored, read back from the device's copy of the input."""
    rng = np.random.default_rng(7)
    text = rng.integers(1, 256, 300_000, dtype=np.uint8).tobytes()
    path = str(tmp_path / "h.bam")
    with EB.BamWriter(path, text, ["r"], [100], device=0) as w:
        pass
    raw = gzip.decompress(open(path, "rb").read())
    assert raw[:4] == b"BAM\x01" and raw[8:8 + len(text)] == text
    blocks, stored = _check_blocks(path)
    assert blocks == 5 and stored >= 4


def test_writer_switches_back_to_host(tmp_path):
    """Nothing is compressed before the first drain; a writer switched back
    to the host threads writes everything with zlib."""
    rng = np.random.default_rng(8)
    letters = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 200_000)].tobytes()
    path = str(tmp_path / "c.bam")
    w = EB.BamWriter(path, letters, ["r"], [100], device=0)
    try:
        assert w.blocks() == (0, 0)
        assert _native.load().esg_bam_writer_use_device(w._h, -1) == 0
    finally:
        w.close()
    raw = gzip.decompress(open(path, "rb").read())
    assert raw[8:8 + len(letters)] == letters
    cdata = _members(path)[0][0]
    assert cdata != _host_steps(zlib.decompress(cdata, -15))


def test_bad_device_is_refused(tmp_path):
    with pytest.raises(Exception, match="no such device"):
        EB.BamWriter(str(tmp_path / "x.bam"), b"", ["r"], [1], device=4096)
