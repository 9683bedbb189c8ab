"""Panel shards (eschalign_b200.shards) on CPU: the reference ranges, the
merge of per-shard results (esg_merge_read_results, host only) against the
oracle's whole-panel results, and the exchange over two gloo ranks -- the
CPU oracle stands in for each rank's GPU."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from eschalign_b200 import shards, synth

D = (2, -1, -10, -1)


def test_shard_ranges_partition_and_balance():
    rng = np.random.default_rng(5)
    lens = rng.integers(300, 1000, 1000)
    for world in (1, 2, 3, 8):
        r = shards.shard_ranges(lens, world)
        assert r[0][0] == 0 and r[-1][1] == lens.size
        assert all(a[1] == b[0] for a, b in zip(r, r[1:])) and all(hi > lo for lo, hi in r)
        per = [lens[lo:hi].sum() for lo, hi in r]
        assert max(per) - min(per) <= 2 * lens.max()
    assert shards.shard_ranges([5, 5, 5], 3) == [(0, 1), (1, 2), (2, 3)]


def _panel_with_copies():
    refs = synth.panel_tiles()[:24]
    # copies in different shards: ties across the cut, and truncated lists
    return refs + [refs[2].copy(), refs[5].copy(), refs[2].copy()]


def _shard_results(oracle, reads, refs, lo, hi, cap, local=True):
    res, ties, _ = oracle.scalar_map_batch(reads, refs[lo:hi], D, local, True, cap=cap)
    # the oracle leaves unused tie slots at 0; the library writes ESG_NO_TIE
    n = np.minimum(res["n_tied"], cap)
    ties = ties.copy()
    for k in range(len(reads)):
        ties[k, n[k]:] = shards.NO_TIE
    return res, shards.globalize_ties(ties, lo)


def _same(got_r, got_t, want_r, want_t, cap):
    for f in ("best", "suboptimal", "n_tied"):
        assert np.array_equal(got_r[f], want_r[f]), f
    assert np.array_equal(got_r["flags"] & 3, want_r["flags"] & 3)
    for k in range(got_r.size):
        n = min(int(want_r["n_tied"][k]), cap)
        assert np.array_equal(got_t[k, :n], want_t[k, :n]), k


def test_merge_equals_the_whole_panel(oracle):
    refs = _panel_with_copies()
    reads = synth.reads_c1(refs, n=120).list()
    reads += [refs[2][10:90].copy(), np.zeros(0, np.uint8)]
    for cap in (1, 2, 8):
        for world in (2, 3):
            ranges = shards.shard_ranges([len(r) for r in refs], world)
            parts = [_shard_results(oracle, reads, refs, lo, hi, cap) for lo, hi in ranges]
            got_r, got_t = shards.merge(parts, cap)
            want_r, want_t, _ = oracle.scalar_map_batch(reads, refs, D, True, True, cap=cap)
            _same(got_r, got_t, want_r, want_t, cap)
            assert got_r["n_tied"][-2] >= 3  # the copies tie across the cuts


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        refs = _panel_with_copies()
        reads = synth.reads_c1(refs, n=150).list()
        lo, hi = shards.shard_ranges([len(r) for r in refs], world)[rank]
        res, ties = _shard_results(O, reads, refs, lo, hi, 4)
        parts = shards.exchange(res, ties, world)
        got_r, got_t = shards.merge(parts, 4)
        want_r, want_t, _ = O.scalar_map_batch(reads, refs, D, True, True, cap=4)
        try:
            _same(got_r, got_t, want_r, want_t, 4)
            out.put((rank, True))
        except AssertionError as e:
            out.put((rank, str(e)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_merge_to_the_whole_panel():
    from oracle import oracle as O
    O.build()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: True, 1: True}, got
