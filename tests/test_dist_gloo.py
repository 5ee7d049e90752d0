"""The multi-rank plumbing of bench.py (one process per GPU under torchrun,
independent replicas): process group set-up, the barrier, the max over
ranks of the timed region and the whole-job throughput, run as two gloo
ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch
    import bench
    w, r, local, dist = bench.dist_setup(world, backend="gloo")
    dev = torch.device("cpu")
    bench.barrier(dist, dev)
    # rank r processed (r + 1) * 1000 units in (r + 1) * 0.5 s
    units, secs = (r + 1) * 1000.0, (r + 1) * 0.5
    rate = bench.whole_job_rate(units, secs, dist, dev)
    tmax = bench.max_over_ranks(secs, dist, dev)
    bench.barrier(dist, dev)
    dist.destroy_process_group()
    out.put((r, w, rate, tmax))


def test_two_gloo_ranks_whole_job_rate():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, rate, tmax in res:
        assert w == world
        assert tmax == 1.0                      # slowest rank
        assert rate == pytest.approx(3000.0)    # (1000 + 2000) units / 1.0 s


def test_single_process_needs_no_group():
    import bench
    w, r, local, dist = bench.dist_setup(1)
    assert dist is None and w == 1
    assert bench.whole_job_rate(500.0, 2.0, None, None) == 250.0
    assert bench.max_over_ranks(3.0, None, None) == 3.0
