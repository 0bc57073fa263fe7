"""Multi-rank replica path on CPU (gloo, world size 2): each rank runs its own
seeded system, and the job's throughput uses the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import numpy as np
    import torch.distributed as dist

    from mars_md_b200 import workloads as W
    from mars_md_b200.replicas import job_throughput, max_over_ranks, rank_env, replica_seed

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        w_, r_, _ = rank_env()
        assert (w_, r_) == (world, rank)
        w = W.plain_bd(seed=replica_seed(W.DEFAULT_SEED, rank), n=256)
        ms = max_over_ranks(10.0 + 5.0 * rank)
        digests = [None] * world
        dist.all_gather_object(digests, float(np.float64(w.pos[:, :3]).sum()))
        out[rank] = (ms, job_throughput(w.n, 4, ms, world), digests)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_time_on_the_slowest_rank():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world,
                       start_method="spawn", join=True)
    (ms0, v0, d0), (ms1, v1, d1) = out[0], out[1]
    assert ms0 == ms1 == 15.0
    assert v0 == v1 == pytest.approx(2 * 256 * 4 / 0.015)
    assert d0 == d1 and d0[0] != d0[1]   # distinct systems per rank


def test_single_process_is_identity():
    from mars_md_b200.replicas import job_throughput, max_over_ranks, replica_seed
    assert max_over_ranks(3.5) == 3.5
    assert job_throughput(100, 10, 1000.0, 1) == 1000.0
    assert replica_seed(5, 0) == 5 and replica_seed(5, 3) == 8
