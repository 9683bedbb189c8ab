"""The serving queue (esg_server_*) on the CUDA path.

Requests of random sizes for four resident scorers (two panels x two
modes), forward or both strands, submitted from several threads at once and
batched together by the server, must come back exactly as each request
scored alone (esg_score_batch on its own scorer) and as the CPU oracle
scores them.  Admission refuses a request whose batch can never fit the
memory budget, without disturbing the others; a wait that runs out of time
is a host-side timeout and the request is still there afterwards."""
import threading

import numpy as np
import pytest

from eschalign_b200 import GpuError, GpuScorer, Mode, Scoring, encode
from eschalign_b200.server import Server
from tests.helpers import Rng, random_panel, reads_for

pytestmark = pytest.mark.gpu

SCORING = (2, -1, -10, -1)
CAP = 8


def _panels():
    rng = Rng(0x5EED_0C05)
    a = [encode(s) for s in random_panel(rng, 37, 20, 280)]
    b = [encode(s) for s in random_panel(rng, 120, 290, 20)]
    return rng, a, b


def _requests(rng, letters_a, letters_b, n_req):
    """(slot, reads, both_strands) with slots 0..3 = (A local, A semi-global,
    B local, B semi-global)."""
    out = []
    for k in range(n_req):
        slot = rng.below(4)
        letters = letters_a if slot < 2 else letters_b
        n = 1 + rng.below(40) if k % 5 else 1 + rng.below(400)
        reads = reads_for(rng, letters, n)
        if k % 7 == 3:
            reads[0] = np.zeros(0, np.uint8)  # an empty read rides along
        out.append((slot, reads, bool(rng.below(2))))
    return out


def test_server_mix_equals_alone_and_oracle(oracle):
    rng = Rng(0x5EED_0C05)
    la = random_panel(rng, 37, 20, 280)
    lb = random_panel(rng, 120, 290, 20)
    pa, pb = [encode(s) for s in la], [encode(s) for s in lb]
    modes = (Mode.LOCAL, Mode.SEMIGLOBAL)
    specs = [(pa, modes[0]), (pa, modes[1]), (pb, modes[0]), (pb, modes[1])]
    reqs = _requests(rng, la, lb, 48)
    served = [GpuScorer(p, Scoring(*SCORING), m, tie_capacity=CAP) for p, m in specs]
    alone = [GpuScorer(p, Scoring(*SCORING), m, tie_capacity=CAP) for p, m in specs]
    got = [None] * len(reqs)
    errors = []
    with Server(served, max_batch_reads=600) as sv:
        def client(ids):
            try:
                tickets = [(i, sv.submit(reqs[i][0], reqs[i][1], reqs[i][2])) for i in ids]
                for i, t in tickets:
                    got[i] = sv.wait(t, timeout_ms=120_000)
            except Exception as e:  # reported below
                errors.append(e)

        threads = [threading.Thread(target=client, args=(list(range(k, len(reqs), 4)),))
                   for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        st = sv.stats()
    assert not errors, errors
    assert st["completed"] == len(reqs) and st["refused"] == 0
    assert st["batches"] < len(reqs)  # requests were batched together
    assert any(tm.batch_requests > 1 for _, tm in got)
    for i, (slot, reads, both) in enumerate(reqs):
        res, tm = got[i]
        want = alone[slot].score_batch(reads, both_strands=both)
        for f in ("best", "suboptimal", "n_tied", "flags"):
            assert np.array_equal(res.results[f], want.results[f]), (i, f)
        for k in range(len(reads)):
            n = min(int(want.results["n_tied"][k]), CAP)
            assert np.array_equal(res.ties[k, :n], want.ties[k, :n]), (i, k)
        assert tm.total_ms >= tm.queued_ms >= 0
        if i % 3 == 0 and len(reads) <= 60:  # the CPU oracle on a share of them
            panel = specs[slot][0]
            local = specs[slot][1] == Mode.LOCAL
            o_res, o_ties, _ = oracle.scalar_map_batch(reads, panel, SCORING, local, both, cap=CAP)
            for f in ("best", "suboptimal", "n_tied"):
                assert np.array_equal(res.results[f], o_res[f]), (i, f)
    for g in served + alone:
        g.close()


def test_server_admission_refuses_what_never_fits():
    rng, pa, pb = _panels()
    g = GpuScorer(pb, Scoring(*SCORING), Mode.LOCAL, tie_capacity=CAP)
    small = [pb[0][:50]]
    big = [pb[k % len(pb)] for k in range(20000)]
    with Server([g], memory_budget=2 << 20) as sv:
        t_big = sv.submit(0, big, True)
        t_small = sv.submit(0, small, True)
        with pytest.raises(GpuError) as ei:
            sv.wait(t_big, 60_000)
        assert ei.value.kind == "OutOfMemory"
        res, _ = sv.wait(t_small, 60_000)
        assert res.results["best"][0] == 100  # 50 matches at +2
        assert sv.stats()["refused"] == 1
    g.close()


def test_server_wait_timeout_is_host_side():
    rng, pa, pb = _panels()
    g = GpuScorer(pb, Scoring(*SCORING), Mode.LOCAL, tie_capacity=CAP)
    reads = [pb[k % len(pb)] for k in range(3000)]
    with Server([g]) as sv:
        t = sv.submit(0, reads, True)
        with pytest.raises(GpuError) as ei:
            sv.wait(t, 0)
        assert ei.value.kind == "Timeout"
        res, tm = sv.wait(t, 120_000)  # still queued: the second wait gets it
        assert res.results["best"][0] == 2 * pb[0].size
        assert tm.batch_reads == 3000
    g.close()


def test_server_splits_large_requests_into_pieces():
    """A request above max_batch_cells runs as several batches of whole
    reads; its results are reassembled in order, equal to scoring it alone,
    and small requests queued behind it ride in between."""
    rng, pa, pb = _panels()
    g = GpuScorer(pb, Scoring(*SCORING), Mode.SEMIGLOBAL, tie_capacity=CAP)
    solo = GpuScorer(pb, Scoring(*SCORING), Mode.SEMIGLOBAL, tie_capacity=CAP)
    letters = None
    big = [pb[(7 * k) % len(pb)][k % 50:k % 50 + 60 + k % 90] for k in range(300)]
    small = [pb[3][10:70]]
    with Server([g], max_batch_cells=50_000_000) as sv:
        tb = sv.submit(0, big, True)
        ts = sv.submit(0, small, False)
        rb, tmb = sv.wait(tb, 120_000)
        rs, tms = sv.wait(ts, 120_000)
        st = sv.stats()
    assert st["batches"] >= 10  # 300 reads x ~1.1e7 cells each, 5e7 cells per batch
    want = solo.score_batch(big, both_strands=True)
    for f in ("best", "suboptimal", "n_tied", "flags"):
        assert np.array_equal(rb.results[f], want.results[f]), f
    for k in range(len(big)):
        n = min(int(want.results["n_tied"][k]), CAP)
        assert np.array_equal(rb.ties[k, :n], want.ties[k, :n]), k
    assert rs.results["best"][0] == 120
    assert tms.total_ms <= tmb.total_ms  # the small one did not wait for all of the big one
    g.close()
    solo.close()
