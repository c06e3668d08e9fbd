"""Multi-process plumbing of bench.py on CPU (gloo, world size 2): the run is
replicas only (independent simulations, no collective on the data path), so
the processes meet only for the barrier around the timed region and the
max-over-ranks of the timings."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r, w, local = bench.dist_setup(world)
    assert (r, w, local) == (rank, world, rank)
    bench.barrier(w)
    out[rank] = bench.dist_max(10.0 + rank, w)
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_replicas_meet_for_timing_only():
    world = 2
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert dict(out) == {0: 11.0, 1: 11.0}
