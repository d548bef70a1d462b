"""The N > 1 path of bench.py on CPU: ranks are independent replicas (or query
shards) with no data-path collective; only the job time (max over ranks) and
the unit count (sum) are reduced. Two gloo ranks on 127.0.0.1."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import excent_b200 as X
    t, units = bench.reduce_over_ranks(1.5 + rank, 100 * (rank + 1), dist, "cpu")
    lo, hi = X.shard(256, world, rank)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([hi - lo]))
    q.put((rank, t, units, lo, hi, [int(s.item()) for s in sizes]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_reduce_time_and_units():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, units, lo, hi, sizes in out:
        assert t == 2.5                      # max over ranks
        assert units == 300                  # sum over ranks
        assert sum(sizes) == 256
    assert out[0][3] == 0 and out[0][4] == out[1][3] and out[1][4] == 256   # contiguous query shards


@pytest.mark.parametrize("count,world", [(256, 1), (256, 3), (7, 4), (0, 2)])
def test_shards_partition(count, world):
    import excent_b200 as X
    seen = []
    for r in range(world):
        lo, hi = X.shard(count, world, r)
        seen.extend(range(lo, hi))
    assert seen == list(range(count))
