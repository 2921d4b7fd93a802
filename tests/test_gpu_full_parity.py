"""Parity with the reference kernel on the full workloads, to the bit.

The smaller parity tests (test_gpu_parity.py) compare a few thousand
creatures; these compare whole generations at the sizes the engine is
measured on, against the reference's own kernel (shaders/creature.cu built
for sm_100a with the reference's compile options, launched with the
reference engine's wave and grid rule):

* the small workload as specified: 4,096 creatures (seed 0), 3-6 nodes, calm
  world, 20 s trials, every result, and the replay frames of creatures 0-15
  (population order) recorded in one batch against the reference's
  one-creature recordings;
* the game workload: 3,000,000 creatures (seed 1), 3-10 nodes, 2-24
  muscles, calm world, 20 s trials;
* the effects workload: 3,000,000 creatures (seed 2), 3-24 nodes, the
  effects world, 20 s trials.

Equal results give equal niche cells, which the host computes from the
result fields alone (src/scheduler.rs:890-923, src/qd.rs:795-808); the test
checks the cells too. On the game and effects generations it also runs the
device entry with the niche epilogue fused into the creature kernel
(ce_advance_device_cells) and checks its results against the reference
kernel's and its metrics rows and cells against the host's, computed from
the reference kernel's results. It also checks run-to-run repeatability on
the GPU (tests/gpu_repeatability.rs:18-68 in the reference) on the effects
generation, whose claim order varies between runs.
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS
from oracle.ref import RefKernel

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32).reshape(len(a), -1)


def assert_same_bits(mine, ref, what):
    mb, rb = bits(mine), bits(ref)
    bad = np.nonzero((mb != rb).any(axis=1))[0]
    assert len(bad) == 0, (f"{what}: {len(bad)} of {len(mine)} creatures differ; first {bad[:5]}: "
                           f"mine {mine[bad[0]]} ref {ref[bad[0]]}")


def niche_cells(pop, wave, res, world):
    """Niche cells of the packed creatures from their results."""
    order = wave.slots.astype(np.int64)
    nodes = (wave.heads[:, 0] & 255).astype(np.uint32)
    metrics = ce.to_metrics(res, nodes, world)
    return ce.niche_cells(pop, metrics, indices=order)


def fused_cells(engine, pop, wave, world):
    """Results, metrics rows and cells of the device entry with the fused
    niche epilogue (global layout), on device-resident records."""
    import torch
    dev = torch.device("cuda", 0)
    n = len(wave)
    flags, rate = ce.world_flags(world), world.rate or 60
    params = ce.make_params(world, 0, n, 0)
    d_lanes = torch.from_numpy(wave.lanes.view(np.int32)).to(dev)
    d_muscles = torch.from_numpy(wave.muscles).to(dev)
    d_heads = torch.from_numpy(wave.heads.view(np.int32).reshape(-1)).to(dev)
    d_shapes = torch.from_numpy(ce.shape_classes(pop, wave)).to(dev)
    d_res = torch.full((n * 19,), float("nan"), dtype=torch.float32, device=dev)
    d_metrics = torch.zeros(n * ce.METRICS_DTYPE.itemsize // 4, dtype=torch.int32, device=dev)
    d_cells = torch.full((n,), -7, dtype=torch.int64, device=dev)
    d_counter = torch.zeros(16, dtype=torch.int32, device=dev)
    d_scratch = torch.empty(engine.scratch_bytes(flags, rate, wave.max_nodes, wave.max_muscles, n),
                            dtype=torch.uint8, device=dev)
    engine.advance_device_cells(d_lanes.data_ptr(), d_muscles.data_ptr(), d_heads.data_ptr(), d_res.data_ptr(),
                                d_counter.data_ptr(), d_scratch.data_ptr(), params, world, wave.max_nodes,
                                wave.max_muscles, d_shapes.data_ptr(), d_cells.data_ptr(), d_metrics.data_ptr(),
                                torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    return (d_res.cpu().numpy().view(ce.RESULT_DTYPE), d_metrics.cpu().numpy().view(ce.METRICS_DTYPE),
            d_cells.cpu().numpy())


def check_fused_cells(engine, pop, wave, world, ref):
    res, metrics, cells = fused_cells(engine, pop, wave, world)
    assert_same_bits(res, ref, "fused-epilogue entry against the reference kernel")
    nodes = (wave.heads[:, 0] & 255).astype(np.uint32)
    host_m = ce.to_metrics(ref, nodes, world)
    assert (metrics.view(np.uint32) == host_m.view(np.uint32)).all(), "metrics rows differ from the host's"
    host_cells = ce.niche_cells(pop, host_m, indices=wave.slots)
    bad = np.nonzero(cells != host_cells)[0]
    assert len(bad) == 0, f"{len(bad)} cells differ; first {bad[:5]}: {cells[bad[:5]]} vs {host_cells[bad[:5]]}"


def full_generation(engine, name):
    w = WORKLOADS[name]
    world = w.world()
    pop = ce.generate(w.spec, w.count)
    wave = ce.pack(pop, world)
    mine, _ = engine.run(wave, world)
    ref, _ = RefKernel(ce.world_flags(world), world.rate or 60).run(wave, ce.make_params(world))
    return w, world, pop, wave, mine, ref


def test_small_workload_results_and_first_frames_match_bits(engine):
    w = WORKLOADS["small"]
    world = w.world()
    assert ce.trial_steps(world) == 1200
    pop = ce.generate(w.spec, w.count)
    wave = ce.pack(pop, world)
    mine, _ = engine.run(wave, world)
    ref, _ = RefKernel(ce.world_flags(world)).run(wave, ce.make_params(world))
    assert_same_bits(mine, ref, "small workload, 4,096 x 20 s")
    assert (niche_cells(pop, wave, mine, world) == niche_cells(pop, wave, ref, world)).all()

    # Creatures 0-15 of the population, recorded together.
    where = np.argsort(wave.slots)[:16]
    assert (wave.slots[where] == np.arange(16)).all()
    sixteen = wave.take(where)
    frames, res = engine.record(sixteen, world)
    assert_same_bits(res, mine[where], "recorded results against scored results")
    stride = ce.frame_stride(sixteen.max_muscles)
    per = ce.settle_frames(world) + ce.trial_steps(world) + 1
    assert frames.shape[1] == per == 1301
    rec = RefKernel(ce.world_flags(world), 60, record=True)
    for c in range(16):
        one = sixteen.take([c])
        s1 = ce.frame_stride(one.max_muscles)
        rf, rr = rec.record_one(one, ce.make_params(world, 0, 1, s1), per, s1)
        n, m = int(one.heads[0, 0] & 255), int(one.heads[0, 1])
        np.testing.assert_array_equal(frames[c][:, :32 + m + n].view(np.uint32), rf[:, :32 + m + n].view(np.uint32),
                                      err_msg=f"creature {c}: node, muscle and force slots")
        np.testing.assert_array_equal(frames[c][:, stride - 1].view(np.uint32), rf[:, s1 - 1].view(np.uint32),
                                      err_msg=f"creature {c}: broken-joint bits")
        assert_same_bits(res[c:c + 1], rr, f"creature {c}: recording's result")


def test_game_workload_full_generation_matches_bits(engine):
    w, world, pop, wave, mine, ref = full_generation(engine, "game")
    assert len(mine) == 3_000_000
    assert_same_bits(mine, ref, "game workload, 3M x 20 s")
    assert (niche_cells(pop, wave, mine, world) == niche_cells(pop, wave, ref, world)).all()
    check_fused_cells(engine, pop, wave, world, ref)
    # The trials run long enough to be worth measuring on.
    assert ce.creature_substeps(mine, world) > 0.5 * len(mine) * 1200 * 16


def test_effects_workload_full_generation_matches_bits_and_repeats(engine):
    w, world, pop, wave, mine, ref = full_generation(engine, "effects")
    assert len(mine) == 3_000_000
    assert_same_bits(mine, ref, "effects workload, 3M x 20 s")
    assert (niche_cells(pop, wave, mine, world) == niche_cells(pop, wave, ref, world)).all()
    check_fused_cells(engine, pop, wave, world, ref)
    again, _ = engine.run(wave, world)
    assert_same_bits(again, mine, "effects workload, second run")
