"""Multi-rank logic of bench.py on CPU (two gloo ranks over 127.0.0.1).

Each rank filters its own seeds (no data-path collective); the only
cross-rank steps are the timing barrier and the max over ranks of the device
time, from which the whole-job rate is computed.
"""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        ms = 10.0 + 5.0 * rank                     # rank 1 is the slower one
        out[rank] = bench.max_over_ranks(ms, torch.device("cpu"))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_with_two_gloo_ranks():
    import bench

    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 15.0
    rate = bench.whole_job_rate(1000.0, 2, 3, out[0])
    assert rate == 1000.0 * 2 * 3 / 0.015


def test_rank_seeds_are_disjoint():
    import bench

    seen = set()
    for r in range(8):
        s = set(bench.rank_seeds(r).tolist())
        assert len(s) == bench.NSEED
        assert not (s & seen)
        seen |= s
    assert np.all(bench.rank_seeds(0) == np.arange(bench.NSEED))
