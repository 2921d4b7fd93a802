"""Host side of the device metrics epilogue: the height-bin edges reproduce
the host's log-height bin exactly, and the shape classes are those of
ce_niche."""
import numpy as np

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS


def _height_digit(pop, mean_height):
    m = np.zeros(1, ce.METRICS_DTYPE)
    m["mean_height"] = mean_height
    m["feet"] = 1
    _, niche = ce.niche(pop, 0, m[0])
    return int(niche[3])


def test_height_edges_are_where_the_host_bin_steps():
    pop = ce.generate(WORKLOADS["small"].spec, 1)
    edges = ce.height_bin_edges()
    assert (np.diff(edges) > 0).all()
    for b, t in enumerate(edges, start=1):
        below = np.nextafter(np.float32(t), np.float32(0))
        assert _height_digit(pop, t) == b
        assert _height_digit(pop, below) == b - 1
    rng = np.random.default_rng(0)
    for h in rng.uniform(0, 3, 2000).astype(np.float32):
        assert _height_digit(pop, h) == int((h >= edges).sum())


def test_shape_classes_match_the_host_niche():
    w = WORKLOADS["game"]
    world = w.world()
    pop = ce.generate(w.spec, 500)
    wave = ce.pack(pop, world)
    shapes = ce.shape_classes(pop, wave)
    m = np.zeros(1, ce.METRICS_DTYPE)
    m["feet"] = 1
    for c in range(len(wave)):
        _, niche = ce.niche(pop, int(wave.slots[c]), m[0])
        assert shapes[c] == niche[2]
