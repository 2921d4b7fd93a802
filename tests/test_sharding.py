"""One generation over several ranks (evolution_simulator_gpu_b200.shard),
run as two gloo processes on the CPU. Each rank evaluates its cost-balanced
range with the CPU oracle standing in for its GPU, and the gathered results
must equal one rank's evaluation of the whole generation."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import shard
from evolution_simulator_gpu_b200.configs import WORKLOADS


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def make_wave():
    world = ce.make_world(duration=1.0)
    pop = ce.generate(WORKLOADS["game"].spec, 300)
    return world, ce.pack(pop, world)


def oracle_evaluate(world):
    from oracle.ref import Oracle
    o = Oracle()

    def run(wave):
        res, _ = o.run(wave, ce.make_params(world), ce.world_flags(world), threads=1)
        return res
    return run


def worker(rank, world_size, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        world, wave = make_wave()
        res = shard.evaluate_sharded(oracle_evaluate(world), wave, rank, world_size)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), res)
    finally:
        dist.destroy_process_group()


def test_plan_balances_cost():
    cost = np.array([1.0] * 10 + [10.0] * 10)
    b = shard.plan(cost, 2)
    assert b[0] == 0 and b[-1] == 20
    left, right = cost[:b[1]].sum(), cost[b[1]:].sum()
    assert abs(left - right) <= 10.0
    assert (np.diff(shard.plan(np.ones(7), 3)) >= 2).all()


def test_two_ranks_gather_the_whole_generation(tmp_path):
    port = free_port()
    mp.start_processes(worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    world, wave = make_wave()
    whole = oracle_evaluate(world)(wave)
    for r in range(2):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert (got.view(np.uint32) == whole.view(np.uint32)).all()
