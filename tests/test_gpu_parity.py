"""Parity of the engine's kernel with the reference kernel, bit for bit.

The reference kernel is the reference's own shaders/creature.cu, built for
sm_100a with the reference's compile options (oracle/build_ref.py) and
launched with the reference engine's launch rule. Both eat the same packed
records, so every field of every result must match to the bit, in every
compiled world, and a recording's frames must match the reference's
recording of the same creature frame by frame.
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS, effects_world_kw
from oracle.ref import RefKernel

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32).reshape(len(a), -1)


def compare(engine, spec, world, n, duration=None):
    if duration is not None:
        world.duration = duration
    pop = ce.generate(spec, n)
    wave = ce.pack(pop, world)
    mine, _ = engine.run(wave, world)
    ref, _ = RefKernel(ce.world_flags(world), world.rate or 60).run(wave, ce.make_params(world))
    mb, rb = bits(mine), bits(ref)
    bad = np.nonzero((mb != rb).any(axis=1))[0]
    assert len(bad) == 0, (
        f"{len(bad)} of {n} creatures differ; first {bad[:5]}: mine {mine[bad[0]]} ref {ref[bad[0]]}")
    return mine


def test_calm_world_small_bodies_match_bits(engine):
    res = compare(engine, WORKLOADS["small"].spec, ce.make_world(), 2048)
    assert np.isfinite(res["fitness"]).all()


def test_calm_world_uneven_bodies_match_bits(engine):
    compare(engine, WORKLOADS["game"].spec, ce.make_world(), 2048, duration=10.0)


def test_effects_world_matches_bits(engine):
    compare(engine, WORKLOADS["effects"].spec, ce.make_world(**effects_world_kw()), 2048, duration=10.0)


def test_quake_world_matches_bits(engine):
    w = ce.make_world(**dict(effects_world_kw(), terrain=1, quake=0.05))
    compare(engine, WORKLOADS["refine"].spec, w, 1024, duration=10.0)


def test_every_effect_matches_bits(engine):
    w = ce.make_world(terrain=2, gravity=14.7, air_retention=0.985, ground_friction=1.0, slope=0.03, wind=-1.0,
                      mud=0.05, brambles=3.0, water=0.12, patches=0.5, gaps=0.35, hurdles=0.08, quake=0.05)
    assert ce.world_flags(w) == 0xFFF
    compare(engine, WORKLOADS["effects"].spec, w, 1024, duration=5.0)


def test_screen_and_rungs_match_bits(engine):
    rungs = [((0.5, 0.2, -0.1, -0.01, 0.3, 0.1), 0.05, 0b10000000),
             ((0.4, 0.3, 0.0, -0.02, 0.2, 0.0), 0.2, 0)]
    w = ce.make_world(screen=(5.0, 0.02, 0.01, 0.0), rungs=rungs)
    spec = WORKLOADS["small"].spec
    pop = ce.generate(spec, 1024)
    pop.genomes["flags"] = np.array([0, 1, 2, 4, 8, 16, 32, 0], np.uint32)[np.arange(1024) % 8]
    wave = ce.pack(pop, w)
    mine, _ = engine.run(wave, w)
    ref, _ = RefKernel(ce.world_flags(w)).run(wave, ce.make_params(w))
    assert (bits(mine) == bits(ref)).all()
    assert (mine["screened"] > 0).any(), "the screen and the rungs stopped nobody"


def test_fine_rate_matches_bits(engine):
    compare(engine, WORKLOADS["small"].spec, ce.make_world(rate=120), 512, duration=5.0)


def test_recording_matches_reference_frames(engine):
    world = ce.make_world(duration=3.0)
    pop = ce.generate(WORKLOADS["small"].spec, 6)
    wave = ce.pack(pop, world)
    frames, res = engine.record(wave, world)
    stride = ce.frame_stride(wave.max_muscles)
    per = ce.settle_frames(world) + ce.trial_steps(world) + 1
    ref = RefKernel(ce.world_flags(world), 60, record=True)
    for c in range(len(wave)):
        one = wave.take([c])
        p = ce.make_params(world, 0, 1, ce.frame_stride(one.max_muscles))
        # The reference's frames have the slots of a batch of this creature
        # alone; the engine's frames are as wide as the widest creature.
        rf, rr = ref.record_one(one, p, per, ce.frame_stride(one.max_muscles))
        s1 = ce.frame_stride(one.max_muscles)
        m = int(one.heads[0, 1])
        n = int(one.heads[0, 0] & 255)
        mine = frames[c]
        np.testing.assert_array_equal(mine[:, :32 + m + n].view(np.uint32), rf[:, :32 + m + n].view(np.uint32))
        np.testing.assert_array_equal(mine[:, stride - 1].view(np.uint32), rf[:, s1 - 1].view(np.uint32))
        assert bits(res[c:c + 1]).tolist() == bits(rr).tolist()
