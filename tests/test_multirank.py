"""World-size-2 checks of bench.py's multi-rank host logic on CPU (gloo): every rank solves its own seeded
instance (weak scaling, no data-path collective) and the timing reduction is the max over ranks."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

import bench


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
        t = bench.reduce_max(1.0 + rank, dist, device="cpu")
        inst = bench.rank_instances(rank, world, 5)
        out[rank] = (t, inst, bench.rank_seed(rank))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0                       # max over ranks
    assert sorted(res[0][1] + res[1][1]) == list(range(5))     # instances split, none twice
    assert set(res[0][1]).isdisjoint(res[1][1])
    assert res[0][2] != res[1][2]                              # each rank its own seeded instance
