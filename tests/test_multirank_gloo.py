"""The multi-GPU path of bench.py on CPU: two gloo ranks. TERRAIN chunks are independent,
so N GPUs run N replicas of the workload with no data-path collective; the only exchange
is the step time, reduced as the maximum over ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    import bench
    try:
        v = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        dist.barrier()
        out[rank] = v
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_max_over_two_ranks():
    ctx = mp.get_context('spawn')
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 15.0, 1: 15.0}


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
