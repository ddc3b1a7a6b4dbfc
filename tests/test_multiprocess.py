"""The N > 1 plumbing of bench.py on CPU: two gloo ranks, as torchrun launches them.  Each GPU
runs an independent replica (no data-path collective); the only collectives are the barrier
around the timed region and the maximum of the per-rank times."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        bench._barrier(world)
        t = bench._max_over_ranks(10.0 + rank, world, torch.device("cpu"))
        bench._barrier(world)
        out[rank] = t
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_is_the_maximum():
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 11.0, 1: 11.0}
