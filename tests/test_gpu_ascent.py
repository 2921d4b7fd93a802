"""The refinement's ascent on the device (ce_ascent: one CUDA graph of
checkpointed forward runs, backward runs, gene gradients, clipped ascent
steps and device repacking) against the same ascent run step by step through
the host: ce_forward + ce_backward, the host's gene-gradient chain rule
(ce_gene_gradients), refine.ascend in numpy and the host packer. Every
step's fitness and the final genes must be equal to the bit, in the calm
world of the gradients workload and the refined-search world (rough ground,
hurdles, tremors, water, ice, wind, thick air)."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import refine
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def host_ascent(engine, pop, world, steps, step):
    fits, x = [], pop
    for _ in range(steps):
        wave = ce.pack(x, world)
        with engine.forward(wave, world) as tape:
            f = np.empty(len(wave), np.float32)
            f[wave.slots] = tape.results["fitness"]
            g = tape.backward()
            shape = tape.shape
        mg, ng = ce.gene_gradients(x, wave, world, g, shape)
        x = refine.ascend(x, mg, ng, step)
        fits.append(f)
    wave = ce.pack(x, world)
    res, _ = engine.run(wave, world)
    f = np.empty(len(wave), np.float32)
    f[wave.slots] = res["fitness"]
    fits.append(f)
    return fits, x


@pytest.mark.parametrize("name,count,seconds", [("gradients", 256, 1.0), ("refine", 384, 0.5)])
def test_device_ascent_equals_the_host_ascent(engine, name, count, seconds):
    w = WORKLOADS[name]
    world = w.world(duration=seconds)
    pop = ce.generate(w.spec, count)
    steps, step = 3, 1e-2
    want, x = host_ascent(engine, pop, world, steps, step)
    with ce.Ascent(engine, pop, world, steps, step) as asc:
        secs = asc.launch()
        got = [asc.fitness(k) for k in range(steps + 1)]
        y = asc.population()
        again = asc.launch()
    assert secs > 0 and again > 0
    for k in range(steps + 1):
        assert (got[k].view(np.uint32) == want[k].view(np.uint32)).all(), f"step {k}"
    for field in ("short", "long", "phase", "duty"):
        assert (y.muscles[field].view(np.uint32) == x.muscles[field].view(np.uint32)).all(), field
    assert (y.strength.view(np.uint32) == x.strength.view(np.uint32)).all()
    assert (y.nodes["friction"].view(np.uint32) == x.nodes["friction"].view(np.uint32)).all()
    # The genes moved.
    assert (y.muscles["long"] != pop.muscles["long"]).any()
