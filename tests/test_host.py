"""Host-side logic: scoring, alphabet, panel, synthetic workloads, tie
selection helper."""
import numpy as np
import pytest

from eschalign_b200 import (Mode, Panel, PanelError, Scoring, ScoringError, encode,
                            reverse_complement_codes, select_hits, synth)
from eschalign_b200.scorer import ReadScores


def test_scoring_parse_and_validate():
    """scoring.rs:192-213."""
    s = Scoring.parse("2,-1,-10,-1")
    assert s == Scoring() and str(s) == "2,-1,-10,-1"
    assert s.gap(1) == -10 and s.gap(3) == -12
    for bad in ("2,-1,-10", "2,-1,10,-1", "0,-1,-10,-1", "2,3,-10,-1", "2,-1,-10,-x"):
        with pytest.raises(ScoringError):
            Scoring.parse(bad)
    assert Mode.parse("overlap") is Mode.SEMIGLOBAL and Mode.parse("local") is Mode.LOCAL


def test_alphabet():
    assert list(encode("ACGTUacgtu")) == [0, 1, 2, 3, 3, 0, 1, 2, 3, 3]
    assert all(v == 4 for v in encode("NnRYKMSWBDHV-*.X"))
    assert list(reverse_complement_codes(encode("ACGTN"))) == list(encode("NACGT"))


def test_panel_refusals():
    with pytest.raises(PanelError):
        Panel([])
    with pytest.raises(PanelError):
        Panel([("a", b"")])
    p = Panel([("a", b"ACGT"), ("b", b"AC")])
    assert len(p) == 2 and p.max_len() == 4 and p.total_len() == 6


def test_synthetic_workloads_are_deterministic():
    a = synth.panel_tiles()
    b = synth.panel_tiles()
    assert len(a) == 164 and all((x == y).all() for x, y in zip(a, b))
    lens = np.array([r.size for r in a])
    assert lens.min() >= 70 and lens.max() <= 180
    r1 = synth.reads_c1(a, n=2000)
    r2 = synth.reads_c1(a, n=2000)
    assert (r1.codes == r2.codes).all() and (r1.lens == r2.lens).all()
    assert r1.lens.min() >= 60 and r1.lens.max() <= 200 and r1.codes.max() <= 3
    c2 = synth.reads_c2(a, n=20000)
    assert c2.lens.min() >= 20 and c2.lens.max() <= 1000
    assert 100 <= np.median(c2.lens) <= 120


def test_select_hits():
    """mapper.rs:466-472."""
    s = ReadScores(24, 20, 3, [(0, False), (0, True), (5, False)], False, False)
    assert select_hits(s) == s.ties
    assert select_hits(s, max_ties=0) == [(0, False)]
    assert select_hits(s, min_score=25) == []
    assert select_hits(ReadScores(None, None, 0, [], False, False)) == []


def test_server_refuses_bad_requests_on_the_host():
    """esg_server_*: a request for a slot that does not exist, an unknown
    flag, a wait on an unknown ticket -- refused before anything reaches a
    device (no scorer needed)."""
    import ctypes as C

    from eschalign_b200 import _native
    from eschalign_b200.scorer import GpuError, _check

    lib = _native.load()
    h = C.c_void_p()
    _check(lib, lib.esg_server_new(None, C.byref(h)))
    try:
        codes = np.array([0, 1, 2, 3], np.uint8)
        off = np.array([0], np.uint64)
        lens = np.array([4], np.uint32)
        t = C.c_uint64()
        args = (codes.ctypes.data_as(C.POINTER(C.c_uint8)), off.ctypes.data_as(C.POINTER(C.c_uint64)),
                lens.ctypes.data_as(C.POINTER(C.c_uint32)), 1)
        assert lib.esg_server_submit(h, 0, *args, 0, C.byref(t)) == 7  # no slot 0
        assert b"slot" in lib.esg_last_error()
        assert lib.esg_server_submit(h, 0, *args, 2, C.byref(t)) == 7  # FULL_ROWS not served
        assert lib.esg_server_wait(h, 12345, 0, None, None, None) == 7
        st = _native.EsgServerStats()
        _check(lib, lib.esg_server_stats_get(h, C.byref(st)))
        assert st.requests == 0
        with pytest.raises(GpuError):
            _check(lib, lib.esg_server_add_scorer(h, None, None))
    finally:
        lib.esg_server_free(h)


def test_fits_f16_matches_the_reference_bound():
    """The known answers of crates/eschalign/src/cuda/mod.rs:783-792."""
    from eschalign_b200.scorer import fits_f16
    s = Scoring(2, -1, -10, -1)
    assert fits_f16(130, 200, s)
    assert fits_f16(4096, 200, s)           # min(n, L) = 200: 421
    assert fits_f16(1013, 4096, s)          # 2047
    assert not fits_f16(1014, 4096, s)      # 2049
    assert not fits_f16(1, 10, Scoring(1000, -1000, -1000, -1000))  # gaps alone 3000
    s = Scoring(3, -2, -5, -2)
    assert fits_f16(678, 1000, s)
    assert not fits_f16(679, 1000, s)


def test_mapping_results_decode_without_a_device():
    """Mappings turns the C ABI's arrays (esg_read_mapping, esg_hit,
    esg_pair_mapping, esg_pair_hit, CIGAR words, MD characters) into the
    reference's ReadMapping / PairMapping fields."""
    import numpy as np
    from eschalign_b200.scorer import (HIT_DTYPE, MAPPING_DTYPE, PAIR_HIT_DTYPE,
                                       PAIR_MAPPING_DTYPE, Mappings)
    ops = np.array([(5 << 4) | 0, (1 << 4) | 1, (3 << 4) | 0, (2 << 4) | 2, (4 << 4) | 0],
                   dtype=np.uint32)
    md = b"8^AC2G1" + b"12"
    hits = np.zeros(3, dtype=HIT_DTYPE)
    hits[0] = (2, 1, 17, 1, 10, 4, 15, 5, 0, 4, 7, 0)     # 5M1I3M2D4M, MD 8^AC2G1
    hits[1] = (0, 0, 24, 0, 12, 0, 12, 1, 4, 0, 2, 7)     # 4M (words 4..5), MD 12
    reads = np.zeros(3, dtype=MAPPING_DTYPE)
    reads[0] = (17, 9, 1, 3, 1, 0, 0)
    reads[1] = (5, 0, 2, 1, 0, 0, 1)                      # no suboptimal, unmapped
    reads[2] = (0, 0, 0, 0, 0, 0, 1)                      # empty read
    m = Mappings(reads, hits[:2], ops, md)
    assert len(m) == 3
    a = m.mapping(0)
    assert a["best_score"] == 17 and a["suboptimal"] == 9 and a["n_tied"] == 1
    assert a["hits"] == [{"reference": 2, "reverse": True, "score": 17, "query_start": 1,
                          "query_end": 10, "ref_start": 4, "ref_end": 15,
                          "cigar": "5M1I3M2D4M", "md": "8^AC2G1", "nm": 4}]
    assert m.mapping(1) == {"best_score": 5, "n_tied": 2, "suboptimal": None, "hits": []}
    assert m.mapping(2) == {"best_score": None, "n_tied": 0, "suboptimal": None, "hits": []}
    # a paired result: pair 0 Proper with one hit, pair 1 Separate (mates 2, 3)
    pairs = np.zeros(2, dtype=PAIR_MAPPING_DTYPE)
    pairs[0] = (1 | 2, 41, 1, 1, (17, -5), 0)              # XS of mate 1 only
    ph = np.zeros(1, dtype=PAIR_HIT_DTYPE)
    ph[0]["reference"], ph[0]["reverse"], ph[0]["insert"] = 2, 0, 22
    ph[0]["mates"][0] = hits[0]
    ph[0]["mates"][1] = hits[1]
    preads = np.zeros(4, dtype=MAPPING_DTYPE)
    preads[2] = (24, 0, 1, 1, 1, 0, 0)
    preads[3] = (0, 0, 0, 0, 0, 0, 1)
    pm = Mappings(preads, hits[1:2], ops, md, pairs, ph)
    assert len(pm) == 2
    p0 = pm.pair_mapping(0)
    assert p0["proper"] and p0["score"] == 41 and p0["suboptimal"] == [17, None]
    assert p0["hits"][0]["insert"] == 22 and p0["hits"][0]["mates"][1]["md"] == "12"
    p1 = pm.pair_mapping(1)
    assert not p1["proper"] and p1["mates"][0]["hits"][0]["cigar"] == "4M"
    assert p1["mates"][1]["best_score"] is None


def test_reads_pack_at_two_bits_and_unpack_to_their_codes():
    """The upload format: reads packed at 2 bits a base (each read on a byte,
    base i of a byte in bits 2i..2i+1), bases that are not A/C/G/T listed by
    position.  Unpacked the way the device does it (k0_unpack, then the
    listed positions set to 4), every read is its codes again, wildcards and
    odd bytes as the wildcard code."""
    import ctypes as C

    import numpy as np

    from eschalign_b200 import _native, pack_reads
    lib = _native.load()
    fn = lib.esg_internal_pack_reads
    fn.restype = C.c_uint64
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                   C.c_uint64, C.POINTER(C.c_uint64)]
    rng = np.random.default_rng(5)
    reads = []
    for n in [0, 1, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 100, 257] + list(rng.integers(1, 400, 60)):
        r = rng.integers(0, 4, int(n)).astype(np.uint8)
        if n and rng.random() < 0.4:
            r[rng.integers(0, n, max(1, int(n) // 20))] = rng.choice([4, 4, 5, 200])
        reads.append(r)
    codes, off, lens = pack_reads(reads)
    padded = int(((lens.astype(np.int64) + 3) // 4 * 4).sum())
    out = np.zeros(padded // 4 + 16, np.uint8)
    exc = np.zeros(int((codes > 3).sum()) + 1, np.uint64)
    n_exc = C.c_uint64(0)
    nbytes = fn(codes.ctypes.data, off.ctypes.data, lens.ctypes.data, len(reads),
                out.ctypes.data, exc.ctypes.data, exc.size, C.byref(n_exc))
    assert nbytes == padded // 4 and n_exc.value == int((codes > 3).sum())
    # the device's unpack: byte b -> bases b & 3, b >> 2 & 3, ...
    unpacked = np.stack([(out >> (2 * i)) & 3 for i in range(4)], 1).reshape(-1)
    unpacked[exc[:n_exc.value].astype(np.int64)] = 4
    pos = 0
    for r in reads:
        got = unpacked[pos:pos + r.size]
        assert np.array_equal(got, np.minimum(r, 4)), r
        pos += (r.size + 3) // 4 * 4
