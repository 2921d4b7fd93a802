"""A small gradient-refined search generation on the GPU (refine.search):
the checkpointed forward run scores the elites exactly as the batched
evaluation did, every arm (resampling, guided, CMA-ES) keeps each elite's
best fitness, and the report carries GPU times and gains."""
import numpy as np
import pytest

from evolution_simulator_gpu_b200 import refine
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def test_small_refined_search(engine):
    w = WORKLOADS["refine"]
    rep = refine.search(engine, w.spec, w.world(duration=1.0), parents=32, count=4096, elites=256, steps=2,
                        guided=True, cma_samples=8)
    r, s, g, c = rep["refine"], rep["resample"], rep["guided"], rep["cma"]
    assert r["first_equal"] is True
    assert np.isfinite(rep["elite_mean_fitness"])
    assert c["generations"] >= 1 and np.float32(0.01) <= c["sigma_median"] <= 30
    for arm in (r, s, g, c):
        assert arm["gpu_s"] > 0 and arm["gain"] >= 0 and np.isfinite(arm["gain_per_gpu_s"])
    assert s["children_per_elite"] >= 1
