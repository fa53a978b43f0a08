"""The multi-GPU form of the bench without GPUs: two gloo ranks on 127.0.0.1 shard the far-block
list of the 7,680-RWG sphere with the bench's own sharding (unordered group pairs dealt
round-robin, both directions of a pair on one rank), and the job time is the maximum over ranks."""
import importlib.util
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = _bench()
    m, part = b.build_workload("sphere7k")
    mine = b.shard_blocks(part.gt, part.gs, rank, world)
    t = b.max_over_ranks(10.0 * (rank + 1), world, "cpu")
    out[rank] = (mine.tolist(), t)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_max_time():
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    b = _bench()
    m, part = b.build_workload("sphere7k")
    shards = [set(res[r][0]) for r in range(world)]
    assert shards[0].isdisjoint(shards[1])
    assert shards[0] | shards[1] == set(range(part.n_blocks))
    # both directions of a pair on one rank
    where = {(int(t), int(s)): i for i, (t, s) in enumerate(zip(part.gt, part.gs))}
    for r in range(world):
        for i in shards[r]:
            j = where[(int(part.gs[i]), int(part.gt[i]))]
            assert j in shards[r]
    assert abs(len(shards[0]) - len(shards[1])) <= 2
    assert res[0][1] == res[1][1] == 20.0  # every rank reports the slowest rank's time
    # world 1 takes every block
    assert len(b.shard_blocks(part.gt, part.gs, 0, 1)) == part.n_blocks
