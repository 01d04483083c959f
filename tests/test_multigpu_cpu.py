"""Scene sharding across ranks (CPU tests, gloo, world size 2): every scene is
owned by exactly one rank, loads balance, and the only collectives are the
max-over-ranks timing and the stats gather."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pbf_b200 import multigpu, scenes


def test_assignment_partitions_and_balances():
    sc = scenes.config2(seed=0)
    counts = [s.n for s in sc]
    for world in (1, 2, 3, 4, 8):
        parts = multigpu.assign_scenes(counts, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(counts)))
        ld = multigpu.loads(counts, parts)
        # LPT bound: the heaviest rank exceeds the mean by less than the largest scene
        assert max(ld) - sum(ld) / world <= max(counts)
    with pytest.raises(ValueError):
        multigpu.assign_scenes(counts, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    counts = [s.n for s in scenes.config2(seed=1, n_scenes=16)]
    mine = multigpu.assign_scenes(counts, world)[rank]
    t = float(10 + rank)  # this rank's "time"
    tmax = multigpu.max_over_ranks(t)
    stats = multigpu.gather_stats({"rank": rank, "scenes": mine, "particles": sum(counts[i] for i in mine)})
    if rank == 0:
        q.put((tmax, stats, sum(counts)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tmax, stats, total = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tmax == 11.0
    owned = sorted(i for s in stats for i in s["scenes"])
    assert owned == list(range(16))
    assert sum(s["particles"] for s in stats) == total
