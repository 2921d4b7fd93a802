"""The launch-shape autotuner (ce_autotune): it keeps one of the grid's
settings, and a batch's results under the kept setting equal those under the
default launch shape to the bit (a creature's trial does not depend on which
warp or block runs it)."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def test_autotune_keeps_a_grid_setting_and_results(engine):
    w = WORKLOADS["effects"]
    world = w.world(duration=1.0)
    sample = ce.pack(ce.generate(w.spec, 8192), world)
    wave = ce.pack(ce.generate(w.spec, 30_000, first=8192), world)
    plain, _ = engine.run(wave, world)
    with ce.Engine(0) as tuned:
        best, secs = tuned.autotune(sample, world)
        assert best["ctas_per_sm"] in (0, 3)
        assert best["chunk_k"] in (16, 32, 64)
        assert best["small_body"] in (10, 12, 16, 24)
        assert secs > 0
        got, _ = tuned.run(wave, world)
    assert (got.view(np.uint32) == plain.view(np.uint32)).all()


@pytest.mark.parametrize("opts", [dict(ctas_per_sm=3, chunk_k=8, small_body=12), dict(chunk_k=2, small_body=24)])
def test_launch_shape_does_not_change_results(engine, opts):
    w = WORKLOADS["effects"]
    world = w.world(duration=1.0)
    wave = ce.pack(ce.generate(w.spec, 20_000, first=50_000), world)
    plain, _ = engine.run(wave, world)
    with ce.Engine(0, **opts) as other:
        got, _ = other.run(wave, world)
    assert (got.view(np.uint32) == plain.view(np.uint32)).all()
