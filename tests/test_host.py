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
