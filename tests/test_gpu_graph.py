"""Generations captured as one CUDA graph (ce_graph_open/launch): each
generation's results equal a plain submission's to the bit, over worlds
whose batches split into both size classes."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def test_graph_generations_equal_plain_submissions(engine):
    w = WORKLOADS["effects"]
    world = w.world(duration=3.0)
    waves = [ce.pack(ce.generate(w.spec, 20_000, first=20_000 * k), world) for k in range(3)]
    assert any((wv.heads[:, 0] & 255).max() > 16 for wv in waves)
    with ce.GenerationGraph(engine, waves, world) as g:
        secs = g.launch()
        assert secs > 0
        for k, wv in enumerate(waves):
            plain, _ = engine.run(wv, world)
            assert (g.results(k).view(np.uint32) == plain.view(np.uint32)).all()
        g.launch()
        for k, wv in enumerate(waves):
            plain, _ = engine.run(wv, world)
            assert (g.results(k).view(np.uint32) == plain.view(np.uint32)).all()
