"""Multi-process host path of bench.py (replicas only), world size 2 over gloo on CPU.

With N GPUs every rank advances its own independent replica; the only cross-rank
traffic is the barrier around the timed region and the max over ranks of the timed
duration.  These tests run that plumbing with two CPU processes.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    r, w, local = bench.dist_init(world)
    assert (r, w, local) == (rank, world, rank)
    assert dist.get_backend() == 'gloo'
    bench.barrier(w)
    # each rank "timed" a different duration; the job time is the slowest rank's
    ms = bench.max_over_ranks(10.0 * (rank + 1), w)
    # the reference arm runs on rank 0 only: other ranks return without work
    if rank != 0:
        assert bench.run_reference(None, rank, w) is None
    bench.barrier(w)
    out.put((rank, ms))
    dist.destroy_process_group()


def test_two_ranks_barrier_and_max_over_ranks():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    if any(c is None for c in codes):
        for p in procs:
            p.kill()
        pytest.fail('a rank did not finish')
    assert codes == [0, 0]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 20.0), (1, 20.0)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ('RANK', 'WORLD_SIZE', 'LOCAL_RANK'):
        os.environ.pop(k, None)
    assert bench.dist_init(1) == (0, 1, 0)
    assert bench.max_over_ranks(3.5, 1) == 3.5
