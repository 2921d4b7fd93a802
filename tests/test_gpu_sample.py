"""Samples of parent genomes drawn on the GPU (ce_sample_device): the same
samples whichever ranges the calls draw, every gene within its clamps, the
stated spread, and parents themselves at zero spread."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import refine
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu

W = WORKLOADS["refine"]
FIELDS = ("nodes", "bones", "muscles", "genomes", "strength")


def _same(a, b):
    return all((getattr(a, f).view(np.uint8) == getattr(b, f).view(np.uint8)).all() for f in FIELDS)


def test_device_samples_do_not_depend_on_the_range(engine):
    parents = ce.generate(W.spec, 100)
    whole, parent = refine.samples_gpu(parents, 5000, 0.05, seed=7)
    a, _ = refine.samples_gpu(parents, 1234, 0.05, seed=7)
    b, _ = refine.samples_gpu(parents, 5000 - 1234, 0.05, seed=7, first=1234)
    assert _same(whole, refine.concat([a, b]))
    again, _ = refine.samples_gpu(parents, 5000, 0.05, seed=7)
    assert _same(whole, again)
    other, _ = refine.samples_gpu(parents, 5000, 0.05, seed=8)
    assert not (other.nodes["x"] == whole.nodes["x"]).all()
    assert (parent == np.arange(5000) % 100).all() and (whole.genomes["id"] == 1 + np.arange(5000)).all()


def test_device_samples_keep_limits_and_spread(engine):
    parents = ce.generate(W.spec, 64)
    pop, parent = refine.samples_gpu(parents, 20_000, 0.05, seed=3)
    src = refine.take(parents, parent)
    for f in ("node_count", "bone_count", "muscle_count"):
        assert (pop.genomes[f] == src.genomes[f]).all()
    n, b, m = pop.nodes, pop.bones, pop.muscles
    assert (n["y"] >= 0).all() and (n["diameter"] >= 0.06).all() and (n["diameter"] <= 0.12).all()
    assert (n["friction"] >= 0).all() and (n["friction"] <= 1).all()
    assert (b["rest_length"] >= 0.03).all() and (b["min_angle"] <= 0).all() and (b["max_angle"] >= 0).all()
    assert (m["long"] >= m["short"]).all() and (m["phase"] >= 0).all() and (m["phase"] < 1).all()
    assert (m["duty"] >= 0.05).all() and (m["duty"] <= 0.95).all()
    assert (m["stiffness"] >= 1).all() and (m["stiffness"] <= 120).all()
    assert (pop.strength == src.strength).all()
    dx = n["x"].astype(np.float64) - src.nodes["x"]
    assert abs(dx.mean()) < 0.002 and abs(dx.std() - 0.05) < 0.002
    owner = np.repeat(np.arange(len(pop)), pop.genomes["muscle_count"].astype(np.int64))
    ratio = m["period"] / src.muscles["period"]
    for c in range(40):
        r = ratio[owner == c]
        assert np.allclose(r, r[0], rtol=1e-5)
    ce.pack(pop, W.world())
    zero, _ = refine.samples_gpu(parents, 500, 0.0, seed=3)
    same = refine.take(parents, np.arange(500) % 64)
    assert (zero.nodes == same.nodes).all()
    for f in ("a", "b", "rest_length", "organ_mass", "organ_at"):
        assert (zero.bones[f] == same.bones[f]).all()
    lim = np.float32(120.0 * np.pi / 180.0)
    assert (zero.bones["min_angle"] == np.clip(same.bones["min_angle"], -lim, 0)).all()
    assert (zero.bones["max_angle"] == np.clip(same.bones["max_angle"], 0, lim)).all()
    for f in ("short", "long", "phase", "duty", "anchor_a", "anchor_b"):
        assert (zero.muscles[f] == same.muscles[f]).all()
    assert np.allclose(zero.muscles["period"], same.muscles["period"], rtol=1e-6)
