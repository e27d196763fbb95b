"""Two ranks over gloo on the CPU: view sharding, the map exchange between
passes and max-over-ranks timing (the multi-GPU host logic, without GPUs)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from sensemap_b200 import sharding


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, num_views, out_q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = sharding.shard(num_views, world, rank)
        local = {v: np.full((3, 4), v, np.float32) for v in mine}
        allmaps = sharding.all_gather_maps(local)
        t = sharding.max_over_ranks(1.0 + rank)
        out_q.put((rank, mine, sorted(allmaps), float(sum(m.sum() for m in allmaps.values())), t))
    finally:
        dist.destroy_process_group()


def test_shard_is_a_partition():
    for n in (0, 1, 5, 11, 64):
        for world in (1, 2, 3, 8):
            parts = [sharding.shard(n, world, r) for r in range(world)]
            flat = [i for p in parts for i in p]
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        sharding.shard(4, 2, 2)


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 11, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    assert results[0][1] + results[1][1] == list(range(11))
    for r in results:
        assert r[2] == list(range(11))
        assert r[3] == pytest.approx(12.0 * sum(range(11)))
        assert r[4] == 2.0
