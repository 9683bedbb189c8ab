"""Multi-GPU sharding logic on CPU: two gloo ranks each take a cell-balanced
slice, score it (the CPU oracle stands in for a GPU here), and the gathered
results equal one process scoring everything."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from eschalign_b200 import replicas, synth


def test_shard_bounds_partition_and_balance():
    rng = np.random.default_rng(3)
    lens = rng.integers(20, 1000, 5000)
    for world in (1, 2, 3, 8):
        b = replicas.shard_bounds(lens, world)
        assert b[0] == 0 and b[-1] == lens.size and (np.diff(b) >= 0).all()
        per = [lens[b[k]:b[k + 1]].sum() for k in range(world)]
        assert max(per) - min(per) <= 2 * lens.max()


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
        refs = synth.panel_tiles()[:20]
        reads = synth.reads_c1(refs, n=300)
        mine, first = replicas.shard(reads, rank, world)
        res, ties, _ = O.scalar_map_batch(mine.list(), refs, (2, -1, -10, -1), True, True)
        allr, allt = replicas.gather(res, ties, rank, world)
        if rank == 0:
            want, want_t, _ = O.scalar_map_batch(reads.list(), refs, (2, -1, -10, -1), True, True)
            out.put(bool((allr == want).all() and (allt == want_t).all()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_process():
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
    assert q.get(timeout=5) is True


class _OracleScorer:
    """Stands in for a GpuScorer on one device: score_batch over a
    (codes, off, lens) tuple, the oracle's per-read results and ties."""

    def __init__(self, refs, scoring):
        self.refs, self.scoring, self.calls = refs, scoring, []

    def score_batch(self, reads, both_strands=False):
        from types import SimpleNamespace

        from oracle import oracle as O
        part = synth.Packed(*reads)
        self.calls.append(len(part))
        res, ties, _ = O.scalar_map_batch(part.list(), self.refs, self.scoring, True,
                                          both_strands)
        return SimpleNamespace(results=res, ties=ties)


def test_score_on_devices_equals_one_scorer():
    """One process, several scorers on threads: cell-balanced slices, results
    in read order equal to one scorer over the whole batch; more scorers
    than reads leaves the extra ones an empty slice."""
    from oracle import oracle as O
    refs = synth.panel_tiles()[:16]
    reads = synth.reads_c1(refs, n=240)
    want, want_t, _ = O.scalar_map_batch(reads.list(), refs, (2, -1, -10, -1), True, True)
    for n in (1, 2, 3, 5):
        scs = [_OracleScorer(refs, (2, -1, -10, -1)) for _ in range(n)]
        (res, ties), parts = replicas.score_on_devices(scs, reads, both_strands=True)
        assert (res == want).all() and (ties == want_t).all(), n
        assert sum(len(s.calls) for s in scs) == n and sum(sum(s.calls) for s in scs) == 240
        assert len(parts) == n
    few = reads.slice(0, 2)
    scs = [_OracleScorer(refs, (2, -1, -10, -1)) for _ in range(4)]
    (res, ties), _ = replicas.score_on_devices(scs, few.tuple(), both_strands=False)
    want, want_t, _ = O.scalar_map_batch(few.list(), refs, (2, -1, -10, -1), True, False)
    assert (res == want).all() and (ties == want_t).all()
    assert sorted(s.calls[0] for s in scs) == [0, 0, 1, 1]
