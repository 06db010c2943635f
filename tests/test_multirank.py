"""The N > 1 path of bench.py on the CPU: two gloo ranks exchange their step
times (the job's time is the maximum over ranks), and the reference arm runs
on rank 0 only.  Replicas only: no residual data crosses ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    r, w, loc = bench.dist_env()
    assert (r, w, loc) == (rank, world, rank)
    bench.barrier_sync(world)
    out[rank] = bench.max_over_ranks(1.0 + rank * 2.5, world)

    class A:
        ref_cells, warmup, steps = 2, 0, 0
    if rank != 0:
        # the reference arm returns nothing off rank 0
        assert bench.reference_arm(A()) is None
    bench.barrier_sync(world)
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1] == 3.5
