"""Multi-GPU runs of bench.py are independent replicas (one simulation batch
per rank, no exchange on the data path): the job time is the slowest rank's,
taken by an all-reduce MAX, and every rank builds its own members.  Checked
here with two gloo ranks on the CPU."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from tetfit_b200.cases import batch_cases


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = [10.0 * (rank + 1), 1.5 - rank, 3.0]
        out[rank] = (bench.max_over_ranks(mine, dist, "cpu"),
                     [c.n for c in batch_cases(6, 8, 48, steps=10, seed=bench.replica_seed(31337, rank))])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_build_their_own_members():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        assert res[r][0] == [20.0, 1.5, 3.0]
    assert res[0][1] != res[1][1]


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks([1.0, 2.0]) == [1.0, 2.0]


def test_reference_arm_runs_on_rank_zero_only():
    class A:
        workload, steps, warmup = "batch128", 1, 3
    assert bench.run_batch_reference(A(), rank=1) is None
    assert bench.run_reference(A(), rank=1) is None
