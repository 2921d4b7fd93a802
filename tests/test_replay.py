"""Replay decode (engine::recorded, src/engine.rs:1062-1127) on synthetic
frames: node rows go back to the creature's own numbering, the force slots
follow the muscles, the broken-joint bits sit in the frame's last slot."""
import numpy as np

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS


def test_replay_decode_renumbers_nodes_and_forces():
    pop = ce.generate(WORKLOADS["small"].spec, 4)
    for i in range(len(pop)):
        nodes, bones, muscles, _ = pop.creature(i)
        n, m = len(nodes), len(muscles)
        stride = ce.frame_stride(m)
        count = 5
        frames = np.zeros((count, stride, 2), np.float32)
        order = [0] + [int(b) for b in bones["b"]]
        for t in range(count):
            for k in range(n):
                frames[t, k] = (1000 * t + k, -(1000 * t + k))
            for q in range(m):
                frames[t, 32 + q] = (t + 0.25 * q, 2 * t + q)
            for k in range(n):
                frames[t, 32 + m + k] = (3 * t + k, 4 * t + k)
            frames[t, stride - 1] = np.array([t, 7 * t], np.uint32).view(np.float32)
        out = ce.replay_decode(bones, m, frames)
        for t in range(count):
            for k in range(n):
                assert tuple(out["positions"][t, order[k]]) == (1000 * t + k, -(1000 * t + k))
                assert out["ground"][t, order[k]] == 3 * t + k
                assert out["friction"][t, order[k]] == 4 * t + k
            assert (out["energy"][t] == t + 0.25 * np.arange(m)).all()
            assert (out["pull"][t] == 2 * t + np.arange(m)).all()
            assert out["broken"][t] == t | (7 * t) << 32
