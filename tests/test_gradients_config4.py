"""The FP64 dual-number tangent of the CPU oracle against central finite
differences of the same FP64 physics, on the gradients workload as
specified: 256 creatures (seed 3, 4-12 nodes, 4-20 muscles, flat grippy
ground) over 20 s trials. No GPU is used.

Every record field the gradient covers (per muscle the stroke amplitude,
hill factor, force cap, 1/capacity, phase, duty, 1/duty, 1/(1-duty),
stiffness; per node the friction) moves by a relative step h of its value,
each with a random sign. Over a 20 s trial most such moves flip a contact,
stick/slip or joint-limit mode somewhere, and then no derivative exists for
a difference to estimate; so a creature counts only where the move keeps
the modes, which shows as the two one-sided differences agreeing within
0.1%. At h = 1e-4 that keeps about one creature in seven, and for those
the central difference equals the tangent within 1e-2 and, for nine in ten,
within 1e-3 (the rest: the difference's own O(h^2) error on a chaotic
trajectory). At config 4's h = 1e-3 about one in a hundred keeps its modes
over 20 s; the numbers are in the design notes.
"""
import numpy as np

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS
from oracle.ref import Oracle

# Record float index of each gradient field of a muscle (kernel record layout).
FIELDS = [8, 3, 4, 5, 10, 11, 12, 13, 14]


def _moved(wave, dm, dn, h):
    lanes, mus = wave.lanes.copy(), wave.muscles.copy()
    lf = lanes.view(np.float32)
    for c in range(len(wave)):
        M, N = int(wave.heads[c, 1]), int(wave.heads[c, 0] & 255)
        mo, ro = int(wave.heads[c, 4]), int(wave.heads[c, 3])
        for k in range(M):
            idx = mo + 20 * k + np.array(FIELDS)
            mus[idx] = (mus[idx].astype(np.float64) + h * dm[c, k]).astype(np.float32)
        rows = ro + 6 * np.arange(N) + 2
        lf[rows] = (lf[rows].astype(np.float64) + h * dn[c, :N]).astype(np.float32)
    return ce.WavePack(lanes, mus, wave.heads, wave.slots, wave.info)


def test_fp64_tangent_matches_central_differences_over_20_s():
    w = WORKLOADS["gradients"]
    world = w.world()
    assert ce.trial_steps(world) == 1200
    wave = ce.pack(ce.generate(w.spec, 256), world)
    p, flags = ce.make_params(world), ce.world_flags(world)
    rows, mm = int((wave.heads[:, 0] & 255).max()), int(wave.heads[:, 1].max())
    rng = np.random.default_rng(3)
    dm, dn = np.zeros((len(wave), mm, 9)), np.zeros((len(wave), rows))
    lf = wave.lanes.view(np.float32)
    for c in range(len(wave)):
        M, N = int(wave.heads[c, 1]), int(wave.heads[c, 0] & 255)
        mo, ro = int(wave.heads[c, 4]), int(wave.heads[c, 3])
        for k in range(M):
            dm[c, k] = wave.muscles[mo + 20 * k + np.array(FIELDS)] * rng.choice([-1.0, 1.0], 9)
        dn[c, :N] = lf[ro + 6 * np.arange(N) + 2] * rng.choice([-1.0, 1.0], N)
    o = Oracle()
    tangent, _, _ = o.tangent(wave, p, flags, dm, dn)
    f0 = o.fitness64.copy()
    h = 1e-4
    zm, zn = np.zeros_like(dm), np.zeros_like(dn)
    o.tangent(_moved(wave, dm, dn, h), p, flags, zm, zn)
    fp = o.fitness64.copy()
    o.tangent(_moved(wave, dm, dn, -h), p, flags, zm, zn)
    fm = o.fitness64.copy()
    up, down = (fp - f0) / h, (f0 - fm) / h
    kept = np.abs(up - down) <= 1e-3 * np.maximum(np.abs(up), np.abs(down))
    central = (fp - fm) / (2 * h)
    rel = np.abs(central - tangent)[kept] / np.maximum(np.abs(tangent[kept]), 1e-12)
    assert kept.mean() >= 0.08, kept.mean()
    assert (rel < 1e-2).mean() >= 0.97, (rel < 1e-2).mean()
    assert (rel < 1e-3).mean() >= 0.8, (rel < 1e-3).mean()
