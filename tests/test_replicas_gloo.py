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
