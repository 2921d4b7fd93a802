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


def test_global_top_k_on_one_rank():
    v = np.array([3.0, np.nan, 5.0, 5.0, -np.inf, 1.0])
    ids = np.array([10, 11, 12, 9, 13, 14])
    top, which = shard.global_top_k(v, ids, 3)
    assert which.tolist() == [9, 12, 10] and top.tolist() == [5.0, 5.0, 3.0]


def topk_worker(rank, world_size, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        rng = np.random.default_rng(rank)
        v = rng.normal(size=500)
        v[::17] = np.nan
        ids = np.arange(500) + 500 * rank
        top, which = shard.global_top_k(v, ids, 64, world_size)
        total = shard.all_sum([v[np.isfinite(v)].sum(), 1.0], world_size)
        np.save(os.path.join(out_dir, f"top{rank}.npy"), np.stack([top, which.astype(np.float64)]))
        np.save(os.path.join(out_dir, f"sum{rank}.npy"), total)
    finally:
        dist.destroy_process_group()


def test_two_ranks_choose_the_same_elites(tmp_path):
    port = free_port()
    mp.start_processes(topk_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    v = np.concatenate([np.random.default_rng(r).normal(size=500) for r in range(2)])
    v[np.arange(1000) % 500 % 17 == 0] = np.nan
    top, which = shard.global_top_k(v, np.arange(1000), 64)
    for r in range(2):
        got = np.load(tmp_path / f"top{r}.npy")
        assert (got[1] == which).all() and (got[0] == top).all()
        s = np.load(tmp_path / f"sum{r}.npy")
        assert np.isclose(s[0], np.nansum(v)) and s[1] == 2.0


class OracleEngine:
    """The engine's run / forward surface on the CPU oracle, with zero
    gradients, for checking how the search splits over ranks."""

    def __init__(self):
        from oracle.ref import Oracle
        self.o = Oracle()

    def run(self, wave, world):
        res, _ = self.o.run(wave, ce.make_params(world), ce.world_flags(world), threads=1)
        return res, 1e-6 * len(wave)

    def forward(self, wave, world):
        eng = self

        class Tape:
            def __enter__(self):
                self.results, _ = eng.run(wave, world)
                self.shape = (int((wave.heads[:, 0] & 255).max()), int(wave.heads[:, 1].max()))
                self.seconds = (1e-6 * len(wave), 2e-6 * len(wave))
                return self

            def __exit__(self, *exc):
                return False

            def backward(self):
                rows, mm = self.shape
                return np.zeros((len(wave), 9 * mm + 4 * rows), np.float32)
        return Tape()


def search_worker(rank, world_size, port, out_dir):
    import torch.distributed as dist
    from evolution_simulator_gpu_b200 import refine
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        w = WORKLOADS["refine"]
        rep = refine.search(OracleEngine(), w.spec, w.world(duration=0.5), parents=16, count=600, elites=40, steps=1, ascent="host",
                            resample=False, rank=rank, world_size=world_size)
        np.save(os.path.join(out_dir, f"rep{rank}.npy"),
                np.array([rep["elite_mean_fitness"], rep["refine"]["mean_best"], rep["sample_gpu_s"],
                          rep["refine"]["gpu_s"], float(rep["refine"]["first_equal"])]))
    finally:
        dist.destroy_process_group()


def test_refined_search_splits_over_two_ranks(tmp_path):
    """Two ranks draw and evaluate halves of the samples and choose the same
    elites one rank would: the elites' fitness and the GPU-second totals
    agree with a one-rank search."""
    from evolution_simulator_gpu_b200 import refine
    port = free_port()
    mp.start_processes(search_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    w = WORKLOADS["refine"]
    one = refine.search(OracleEngine(), w.spec, w.world(duration=0.5), parents=16, count=600, elites=40, steps=1, ascent="host",
                        resample=False)
    for r in range(2):
        got = np.load(tmp_path / f"rep{r}.npy")
        assert np.isclose(got[0], one["elite_mean_fitness"], rtol=1e-12)
        assert np.isclose(got[1], one["refine"]["mean_best"], rtol=1e-12)
        assert np.isclose(got[2], one["sample_gpu_s"]) and np.isclose(got[3], one["refine"]["gpu_s"])
        assert got[4] == 1.0
