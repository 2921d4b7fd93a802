"""Recorded trials decoded to the creatures' own node numbering: the frame of
the scoring step gives the fitness (centre of mass's x) within 1e-3, as the
reference's replay check asks (tests/gpu_repeatability.rs:74-140)."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def test_recorded_frames_decode_to_the_fitness(engine):
    w = WORKLOADS["small"]
    world = w.world(duration=4.0)
    pop = ce.generate(w.spec, 16)
    wave = ce.pack(pop, world)
    frames, results = engine.record(wave, world)
    settle = ce.settle_frames(world)
    steps = ce.trial_steps(world)
    rate = world.rate or 60
    for c in range(len(wave)):
        i = int(wave.slots[c])
        nodes, bones, muscles, _ = pop.creature(i)
        out = ce.replay_decode(bones, len(muscles), frames[c])
        n = len(nodes)
        ro = int(wave.heads[c, 3])
        lf = wave.lanes.view(np.float32)
        order = [0] + [int(b) for b in bones["b"]]
        mass = np.zeros(n)
        for k in range(n):
            mass[order[k]] = lf[ro + 6 * k]
        r = results[c]
        ran = int(round(r["fall_time"] * rate)) if r["fall_time"] > 0 else steps
        com = float((mass * out["positions"][settle + ran, :, 0]).sum() / mass.sum())
        assert abs(com - float(r["fitness"])) <= 1e-3, (c, com, float(r["fitness"]))


def test_many_creature_recording_equals_single_recordings(engine):
    """A recording of 400 creatures runs as one launch over several blocks;
    each creature's frames and result equal those of recording it alone."""
    w = WORKLOADS["small"]
    world = w.world(duration=2.0)
    wave = ce.pack(ce.generate(w.spec, 400), world)
    frames, results = engine.record(wave, world)
    stride = frames.shape[2]
    for c in (0, 1, 127, 128, 255, 399):
        one = wave.take([c])
        f1, r1 = engine.record(one, world)
        m, n = int(one.heads[0, 1]), int(one.heads[0, 0] & 255)
        np.testing.assert_array_equal(frames[c][:, :32 + m + n].view(np.uint32), f1[0][:, :32 + m + n].view(np.uint32))
        np.testing.assert_array_equal(frames[c][:, stride - 1].view(np.uint32), f1[0][:, -1].view(np.uint32))
        assert results[c:c + 1].view(np.uint32).tolist() == r1.view(np.uint32).tolist()
