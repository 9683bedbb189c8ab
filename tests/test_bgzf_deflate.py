"""The device BGZF compressor's steps, run lane by lane on the host
(esg_bgzf_deflate_host), checked with zlib's inflate: every block must
inflate to its input exactly.  The cases cover what the steps branch on:
record-like data (matches at short distances across the lanes' stripes),
runs (258-byte matches at distance 1, a single distance symbol), random
bytes (the stored fallback), frequencies skewed enough that the Huffman
tree is deeper than 15 (the length fold), tiny and ragged blocks (empty
lanes), and a full 0xff00-byte block."""
import ctypes as C
import zlib

import numpy as np
import pytest

from eschalign_b200 import _native

STORED = 0xFFFFFFFF


def _deflate(data: bytes):
    lib = _native.load()
    out = np.zeros(65536 // 4, np.uint32)
    src = (C.c_uint8 * len(data)).from_buffer_copy(data)
    n = lib.esg_bgzf_deflate_host(src, len(data), out.ctypes.data)
    return n, out.view(np.uint8)


def _check(data: bytes):
    n, out = _deflate(data)
    assert n != 0
    if n == STORED:
        return None
    assert n <= len(data) + 5
    got = zlib.decompressobj(-15)
    back = got.decompress(out[:n].tobytes())
    assert got.eof, "the stream must end with its final block"
    assert back == data
    return n / len(data)


def _records(n_reads: int, seed: int) -> bytes:
    """Unaligned BAM records as the bench builds them (names, 4-bit bases,
    Phred qualities, a read group)."""
    import tempfile
    import os
    import bench
    from eschalign_b200 import synth
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=n_reads, seed=seed)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "u.bam")
        bench.unmapped_bam(path, reads)
        data = open(path, "rb").read()
    raw, at = [], 0
    while at < len(data):
        bsize = int.from_bytes(data[at + 16:at + 18], "little") + 1
        raw.append(zlib.decompress(data[at + 18:at + bsize - 8], -15))
        at += bsize
    return b"".join(raw)


def test_record_blocks_round_trip_and_compress():
    raw = _records(2000, 5)
    ratios = []
    for s in range(0, len(raw), 0xFF00):
        r = _check(raw[s:s + 0xFF00])
        assert r is not None
        ratios.append(r)
    # zlib level 1 gives 0.62 on these records, level 6 0.595
    assert max(ratios) < 0.66


def test_runs_single_distance_symbol():
    assert _check(b"A" * 0xFF00) < 0.01
    assert _check(b"AC" * 0x7F80) < 0.01
    assert _check(bytes(0xFF00)) < 0.01


def test_random_bytes_are_stored():
    rng = np.random.default_rng(1)
    data = rng.integers(0, 256, 0xFF00, dtype=np.uint8).tobytes()
    n, _ = _deflate(data)
    assert n == STORED
    # random over four letters compresses toward 2 bits a byte (greedy
    # 4-byte matches cost a little on such data: ~0.32)
    four = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 0xFF00)].tobytes()
    assert _check(four) < 0.35


def _lengths(freq, limit):
    lib = _native.load()
    f = np.ascontiguousarray(freq, np.uint32)
    out = np.zeros(len(f), np.uint8)
    assert lib.esg_bgzf_code_lengths(f.ctypes.data_as(C.POINTER(C.c_uint32)), len(f), limit,
                                     out.ctypes.data) == 0
    return out


def _optimal_cost(freq):
    import heapq
    h = [int(w) for w in freq if w]
    heapq.heapify(h)
    cost = 0
    while len(h) > 1:
        a, b = heapq.heappop(h), heapq.heappop(h)
        cost += a + b
        heapq.heappush(h, a + b)
    return cost


@pytest.mark.parametrize("limit", [15, 7])
def test_code_lengths_fold_deep_trees(limit):
    # Fibonacci frequencies: the unlimited tree is as deep as there are
    # symbols; the lengths must be folded to the limit, stay complete
    # (Kraft's sum exactly one) and code the heavy symbols shortest
    fib = [1, 1]
    while len(fib) < (24 if limit == 15 else 12):
        fib.append(fib[-1] + fib[-2])
    freq = np.zeros(286 if limit == 15 else 19, np.uint32)
    freq[:len(fib)] = fib
    ln = _lengths(freq, limit)
    used = ln[freq > 0]
    assert used.min() >= 1 and used.max() == limit
    assert (ln[freq == 0] == 0).all()
    assert sum(2.0 ** -int(x) for x in used) == 1.0
    assert all(ln[i] >= ln[i + 1] for i in range(len(fib) - 1))
    # within a few percent of the unlimited optimum
    assert int((freq * ln).sum()) <= 1.05 * _optimal_cost(freq)


def test_code_lengths_random_are_optimal_when_shallow():
    rng = np.random.default_rng(3)
    for _ in range(50):
        n = int(rng.integers(2, 287))
        freq = rng.integers(0, 1000, n).astype(np.uint32)
        freq[rng.random(n) < 0.3] = 0
        ln = _lengths(freq, 15)
        used = ln[freq > 0]
        if (freq > 0).sum() >= 2:
            assert int((freq * ln).sum()) == _optimal_cost(freq)
        assert sum(2.0 ** -int(x) for x in ln[ln > 0]) == 1.0


def test_code_lengths_one_or_no_symbol_still_complete():
    for freq in ([0] * 30, [5] + [0] * 29, [0] * 29 + [5]):
        ln = _lengths(np.array(freq, np.uint32), 15)
        assert (ln > 0).sum() == 2 and sum(2.0 ** -int(x) for x in ln[ln > 0]) == 1.0
        assert all(ln[i] > 0 for i in range(30) if freq[i])


def test_deep_huffman_block_round_trips():
    # skewed literals throughout a block (the tree folded or not, the block
    # must inflate)
    fib = [1, 1]
    while len(fib) < 22:
        fib.append(fib[-1] + fib[-2])
    sym = np.repeat(np.arange(len(fib), dtype=np.uint8) * 7 + 3, fib)
    rng = np.random.default_rng(2)
    rng.shuffle(sym)
    data = sym[:0xFF00].tobytes()
    assert _check(data) is not None


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 100, 2039, 2040, 2041, 4097, 33333, 0xFEFF,
                               0xFF00])
def test_ragged_block_sizes(n):
    raw = _records(400, 9)
    data = (raw * (n // len(raw) + 1))[:n]
    r = _check(data)
    if n >= 2040:
        assert r is not None


def test_text_across_stripes():
    words = b"the quick brown fox jumps over the lazy dog; " * 2000
    r = _check(words[:0xFF00])
    assert r is not None and r < 0.1


def test_bad_arguments():
    lib = _native.load()
    out = np.zeros(65536 // 4, np.uint32)
    src = (C.c_uint8 * 4)()
    assert lib.esg_bgzf_deflate_host(src, 0, out.ctypes.data) == 0
    assert lib.esg_bgzf_deflate_host(src, 0xFF01, out.ctypes.data) == 0
    assert lib.esg_bgzf_deflate_host(None, 4, out.ctypes.data) == 0
    f = np.ones(300, np.uint32)
    ln = np.zeros(300, np.uint8)
    fp = f.ctypes.data_as(C.POINTER(C.c_uint32))
    assert lib.esg_bgzf_code_lengths(fp, 300, 15, ln.ctypes.data) == -1  # n > 288
    assert lib.esg_bgzf_code_lengths(fp, 19, 16, ln.ctypes.data) == -1   # limit > 15
    assert lib.esg_bgzf_code_lengths(fp, 200, 7, ln.ctypes.data) == -1   # 200 symbols > 2^7
