"""Multi-process host logic of object sharding (world size 2, gloo, CPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from parahpop_b200.sharding import shard_bounds


def test_shard_bounds_partition():
    for n in (1, 7, 10000, 12345):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard_bounds(n, r, world)
                seen.extend(range(lo, hi))
                assert abs((hi - lo) - n / world) <= 1
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, q):
    import torch.distributed as dist
    from datetime import timedelta
    from parahpop_b200.sharding import gather_states, max_over_ranks, shard_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    lo, hi = shard_bounds(n, rank, world)
    ids = np.arange(lo, hi, dtype=np.float64)
    # stand-in propagation: epoch = id, state = id * (1..6)
    states = ids[:, None] * np.arange(1, 7)[None, :]
    ep, st = gather_states(ids, states, n)
    t = max_over_ranks(10.0 + rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ep.tolist(), st.tolist(), t))


def test_gather_and_max_time_world2():
    n = 11
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ep, st, t in res:
        assert ep == list(range(n))
        np.testing.assert_array_equal(np.array(st), np.arange(n)[:, None] * np.arange(1, 7)[None, :])
        assert t == 11.0
