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


@pytest.mark.parametrize("effects", [False, True])
def test_largest_bodies_match_bits(engine, effects):
    """Bodies at the engine's limits: 28-32 nodes and 64-96 muscles, all of
    them one size class, the widest tables and lane slots."""
    spec = ce.GenSpecPy(seed=9, min_nodes=28, max_nodes=32, muscle_rule=1, min_muscles=64, max_muscles=96,
                        joint_lo_deg=30.0, joint_hi_deg=150.0)
    world = ce.make_world(**effects_world_kw()) if effects else ce.make_world()
    res = compare(engine, spec, world, 384, duration=3.0)
    assert (res["fitness"] > -1e19).any()


def _two_node_population(n):
    rng = np.random.default_rng(4)
    nodes = np.zeros(2 * n, ce.api.NODE_DTYPE)
    nodes["x"] = rng.uniform(0, 1, 2 * n)
    nodes["y"] = rng.uniform(0, 1, 2 * n)
    nodes["diameter"] = rng.uniform(0.06, 0.12, 2 * n)
    nodes["friction"] = rng.uniform(0, 1, 2 * n)
    bones = np.zeros(n, ce.api.BONE_DTYPE)
    bones["a"], bones["b"] = 0, 1
    d = np.hypot(nodes["x"][1::2] - nodes["x"][0::2], nodes["y"][1::2] - nodes["y"][0::2])
    bones["rest_length"] = np.clip(d, 0.03, 2.0)
    bones["min_angle"], bones["max_angle"] = -1.0, 1.0
    genomes = np.zeros(n, ce.api.GENOME_DTYPE)
    genomes["node_start"] = 2 * np.arange(n)
    genomes["node_count"] = 2
    genomes["bone_start"] = np.arange(n)
    genomes["bone_count"] = 1
    genomes["id"] = 1 + np.arange(n)
    return ce.Population(nodes, bones, np.zeros(0, ce.api.MUSCLE_DTYPE), genomes, np.zeros(0, np.float32))


def test_two_node_bodies_and_one_creature_batches_match_bits(engine):
    """The smallest body (two nodes, one bone, no joint, no muscle) in the
    calm and the effects world, in a batch and as a batch of one."""
    pop = _two_node_population(200)
    for world in (ce.make_world(duration=3.0), ce.make_world(duration=3.0, **effects_world_kw())):
        wave = ce.pack(pop, world)
        mine, _ = engine.run(wave, world)
        ref, _ = RefKernel(ce.world_flags(world)).run(wave, ce.make_params(world))
        assert (bits(mine) == bits(ref)).all()
        for c in (0, 57, 199):
            one = wave.take([c])
            m1, _ = engine.run(one, world)
            assert (bits(m1) == bits(mine[c:c + 1])).all()
