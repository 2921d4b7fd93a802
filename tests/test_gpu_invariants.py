"""Invariants the reference's own GPU tests hold its kernel to, re-expressed
against this engine (tests/cuda_physics.rs:132-266,
tests/gpu_repeatability.rs:18-68 in the reference):

* a creature's result does not depend on the batch it runs in, its place in
  the batch, or the run (bit for bit);
* nodes do not sink into flat ground by more than 2 cm.
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS, effects_world_kw

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("effects", [False, True])
def test_results_do_not_depend_on_the_batch(engine, effects):
    w = WORKLOADS["effects"]
    world = ce.make_world(duration=4.0, **(effects_world_kw() if effects else {}))
    pop = ce.generate(w.spec, 6000)
    whole = ce.evaluate(engine, pop, world)
    again = ce.evaluate(engine, pop, world)
    assert (whole.view(np.uint32) == again.view(np.uint32)).all()
    # The same creatures in three shuffled batches, each with strangers.
    rng = np.random.default_rng(1)
    order = rng.permutation(6000)
    strangers = ce.generate(w.spec, 3000, first=50_000)
    for part in np.array_split(order, 3):
        idx = np.concatenate([part, 6000 + rng.permutation(3000)[:1000]]).astype(np.uint32)
        both = _joined(pop, strangers)
        got = ce.evaluate(engine, both, world, indices=idx)
        assert (got[:len(part)].view(np.uint32) == whole[part].view(np.uint32)).all()


def _joined(a, b):
    g = b.genomes.copy()
    g["node_start"] += len(a.nodes)
    g["bone_start"] += len(a.bones)
    g["muscle_start"] += len(a.muscles)
    return ce.Population(np.concatenate([a.nodes, b.nodes]), np.concatenate([a.bones, b.bones]),
                         np.concatenate([a.muscles, b.muscles]), np.concatenate([a.genomes, g]),
                         np.concatenate([a.strength, b.strength]))


def test_nodes_stay_above_flat_ground(engine):
    w = WORKLOADS["small"]
    world = w.world(duration=4.0)
    pop = ce.generate(w.spec, 48)
    wave = ce.pack(pop, world)
    frames, _ = engine.record(wave, world)
    lf = wave.lanes.view(np.float32)
    for c in range(len(wave)):
        n = int(wave.heads[c, 0] & 255)
        ro = int(wave.heads[c, 3])
        radius = np.array([lf[ro + 6 * i + 1] for i in range(n)])
        low = (frames[c, :, :n, 1] - radius[None, :]).min()
        assert low >= -0.02, (c, low)
