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
checks the cells too. It also checks run-to-run repeatability on the GPU
(tests/gpu_repeatability.rs:18-68 in the reference) on the effects
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
    # The trials run long enough to be worth measuring on.
    assert ce.creature_substeps(mine, world) > 0.5 * len(mine) * 1200 * 16


def test_effects_workload_full_generation_matches_bits_and_repeats(engine):
    w, world, pop, wave, mine, ref = full_generation(engine, "effects")
    assert len(mine) == 3_000_000
    assert_same_bits(mine, ref, "effects workload, 3M x 20 s")
    assert (niche_cells(pop, wave, mine, world) == niche_cells(pop, wave, ref, world)).all()
    again, _ = engine.run(wave, world)
    assert_same_bits(again, mine, "effects workload, second run")
