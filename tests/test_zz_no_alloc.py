"""esg_score_rows_noalloc: scoring for callers that cannot allocate.

A process whose device memory belongs to a framework's caching allocator,
or a real-time loop that must not enter the driver's allocator after
start-up, cannot let the library call cudaMalloc; it passes its own device
buffers and gets every (query, reference) score, the int32 kernel's column
buffer being a static device array.  Checked here through the C ABI on two
calls in a row against the scorer's own entry point (esg_score_batch with
full rows) and against the scalar oracle, exactly: scores are integers.
The reads include ones longer than 512 bases, whose passes go through the
static column buffer.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from eschalign_b200 import GpuScorer, Mode, Scoring, _native, encode, pack_reads
from tests.helpers import Rng, random_panel, random_seq, reads_for

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _noalloc(lib, torch, reads, panel, scoring, mode, max_ref_len=None):
    codes, off, lens = pack_reads(reads)
    rc, ro, rl = pack_reads(panel)
    d_codes, d_off, d_len = (_dev(torch, codes), _dev(torch, off.view(np.int64)),
                             _dev(torch, lens.view(np.int32)))
    d_rc, d_ro, d_rl = (_dev(torch, rc), _dev(torch, ro.astype(np.uint32).view(np.int32)),
                        _dev(torch, rl.view(np.int32)))
    rows = torch.full((len(reads), len(panel)), -7, dtype=torch.int32, device="cuda")
    sc = _native.EsgScoring(*scoring)
    mx = int(rl.max()) if max_ref_len is None else max_ref_len
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.esg_score_rows_noalloc(d_codes.data_ptr(), d_off.data_ptr(), d_len.data_ptr(),
                                    len(reads), d_rc.data_ptr(), d_ro.data_ptr(), d_rl.data_ptr(),
                                    len(panel), mx, C.byref(sc), int(mode), rows.data_ptr(),
                                    stream)
    torch.cuda.synchronize()
    return st, rows.cpu().numpy()


def test_noalloc_rows_equal_score_batch_and_oracle_twice(oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _native.load()
    rng = Rng(0x5EED_0A11)
    letters = random_panel(rng, 37, 20, 280)
    panel = [encode(s) for s in letters]
    # reads past 512 bases take several passes through the column buffer
    long_reads = [encode(letters[k] * (600 // len(letters[k]) + 1 + k % 3) +
                         random_seq(rng, 40, 0.02)) for k in range(0, 37, 6)]
    first = reads_for(rng, letters, 60) + long_reads[:4]
    second = reads_for(rng, letters, 90) + long_reads[4:]
    assert max(len(r) for r in first) > 512 and max(len(r) for r in second) > 512
    for scoring in ((2, -1, -10, -1), (3, 1, -5, -2)):
        for mode in (Mode.LOCAL, Mode.SEMIGLOBAL):
            local = mode == Mode.LOCAL
            with GpuScorer(panel, Scoring(*scoring), mode) as g:
                for reads in (first, second):  # two calls in a row, sharing the array
                    want = g.score_batch(reads, full_rows=True).rows
                    st, got = _noalloc(lib, torch, reads, panel, scoring, mode)
                    assert st == 0, lib.esg_last_error()
                    assert got.shape == want.shape
                    assert (got == want).all(), (scoring, mode)
                    assert (got == oracle.score_matrix(reads, panel, scoring, local)).all()


def test_noalloc_refuses_references_past_its_scratch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _native.load()
    panel = [np.zeros(100, np.uint8)]
    reads = [np.zeros(10, np.uint8)]
    st, _ = _noalloc(lib, torch, reads, panel, (2, -1, -10, -1), Mode.LOCAL, max_ref_len=8193)
    assert st == 3  # ESG_ERR_REFERENCE_TOO_LONG
    # a reference longer than the stated maximum scores ESG_NO_SCORE, nothing else
    st, rows = _noalloc(lib, torch, reads, [np.zeros(100, np.uint8), np.zeros(50, np.uint8)],
                        (2, -1, -10, -1), Mode.LOCAL, max_ref_len=60)
    assert st == 0 and rows[0, 0] == -(2**31) and rows[0, 1] == 20
    # max_ref_len 0: every reference is longer than that
    st, rows = _noalloc(lib, torch, reads, [np.zeros(5, np.uint8)], (2, -1, -10, -1),
                        Mode.LOCAL, max_ref_len=0)
    assert st == 0 and rows[0, 0] == -(2**31)
