"""Metrics and niche cells against a second restatement of the reference's
rules, written here in Python from the Rust source, on many results.

The engine's host model (csrc/host_model.cpp) restates these rules in C++;
this file restates them again, independently, in float32 numpy with the C
library's logf and roundf (what Rust's f32::ln and f32::round call), and
compares every metrics field and every cell on results that land on and
around every bin edge:

* trial_steps and to_metrics: src/scheduler.rs:858-923
  (GpuResult::feet: src/creature_kernel.rs:97-99);
* descriptor: src/qd.rs:762-790 (start-pose aspect from the node genes);
* niche_in, height_axis, bin: src/qd.rs:795-846, classes_of: src/qd.rs:125-130,
  the layouts: src/qd.rs:16, 61-86 (max_bone 2 m: src/physics.rs:150);
* cell_index: src/qd.rs:988-999.

Only the rules are restated; no output of the reference itself is involved,
since its Rust crate cannot be built here.
"""
import ctypes as C

import numpy as np

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

F = np.float32
LIBM = C.CDLL("libm.so.6")
LIBM.logf.restype = C.c_float
LIBM.logf.argtypes = [C.c_float]
LIBM.roundf.restype = C.c_float
LIBM.roundf.argtypes = [C.c_float]

MOVEMENT_BINS = (6, 8, 6, 5)
LAYOUTS = {True: ((F(0.9), F(1.4), F(2.5)), (9, 11, 14)),   # GLOBAL_CLASSES
           False: ((F(1.2), F(2.0)), (9, 12))}              # ISLAND_CLASSES
MAX_BONE = F(2.0)


def f32_to_u32_sat(x):
    """Rust's `as u32` of an f32: NaN -> 0, saturating."""
    if np.isnan(x):
        return 0
    return int(min(max(np.floor(x) if x >= 0 else np.ceil(x), 0), 2 ** 32 - 1))


def trial_steps(r, rate, steps):
    ended = r["fall_time"] if r["fall_time"] > 0 else r["screened"]
    if ended > 0:
        return min(max(f32_to_u32_sat(LIBM.roundf(F(ended * F(rate)))), 1), max(steps, 1))
    return max(steps, 1)


def to_metrics(r, node_count, rate, steps):
    n = trial_steps(r, rate, steps)
    denom = F(n * node_count)
    vo, gf = r["vertical_oscillation"], r["gait_frequency"]
    feet = bin(int(np.array(r["lift_lo"], np.float32).view(np.uint32))).count("1")
    return {
        "ground_contact": F(np.clip(F(r["ground_contact"] / denom), F(0), F(1))),
        "vertical_oscillation": F(max(vo, F(0))) if np.isfinite(vo) else F(0),
        "gait_frequency": F(max(gf, F(0))) if np.isfinite(gf) else F(0),
        "mean_height": F(max(F(r["height_sum"] / F(n)), F(0))),
        "feet": F(feet),
        "steps": n,
    }


def height_axis(h):
    low = F(0.15)
    high = max(F(F(0.6) * MAX_BONE), F(F(2.0) * low))
    v = F(LIBM.logf(F(max(h, low) / low)) / LIBM.logf(F(high / low)))
    return F(min(max(v, F(0)), F(1)))


def bin_of(value, low, high, count):
    v = F(min(max(F(value), F(low)), F(high)))
    x = np.floor(F(F(F(v - F(low)) / F(F(high) - F(low))) * F(count)))
    return min(int(x), count - 1)


def niche(nodes, muscle_count, m, global_layout):
    xs, ys = nodes["x"].astype(F), nodes["y"].astype(F)
    width = max(F(xs.max() - xs.min()), F(0.01))
    height = max(F(ys.max() - ys.min()), F(0.01))
    aspect = F(min(max(F(width / height), F(0.0625)), F(16.0)))
    contact = F(min(max(m["ground_contact"], F(0)), F(1)))
    cadence = F(min(max(m["gait_frequency"], F(0)), F(20)))
    mean_height = F(max(m["mean_height"], F(0)))
    feet = F(max(m["feet"], F(0)))
    edges, sizes = LAYOUTS[global_layout]
    shape = sum(1 for e in edges if aspect >= e)
    size = sum(1 for e in sizes if len(nodes) >= e)
    feet_b = min(max(int(LIBM.roundf(feet)), 1), MOVEMENT_BINS[3]) - 1
    cell = [bin_of(contact, 0.0, 1.0, MOVEMENT_BINS[0]), bin_of(cadence, 0.0, 6.0, MOVEMENT_BINS[1]), shape,
            bin_of(height_axis(mean_height), 0.0, 1.0, MOVEMENT_BINS[2]), feet_b, size]
    bins = (MOVEMENT_BINS[0], MOVEMENT_BINS[1], len(edges) + 1, MOVEMENT_BINS[2], MOVEMENT_BINS[3], len(sizes) + 1)
    index = 0
    for a, b in zip(cell, bins):
        assert a < b
        index = index * b + a
    return index, cell


def random_results(n, rng, steps):
    """Results whose metrics fall on and around every bin edge."""
    r = np.zeros(n, ce.RESULT_DTYPE)
    nodes = rng.integers(3, 11, n)
    ran = rng.integers(1, steps + 1, n)
    ended = rng.random(n) < 0.6
    r["fall_time"] = np.where(ended & (rng.random(n) < 0.7), ran / 60.0, 0.0).astype(F)
    r["screened"] = np.where(ended & (r["fall_time"] == 0), ran / 60.0, 0.0).astype(F)
    walked = np.where(ended, ran, steps)
    # Contact shares at k/6 of the steps x nodes, just under and just over.
    share = rng.integers(0, 7, n) / 6.0 + rng.choice([-1e-6, 0.0, 1e-6], n)
    r["ground_contact"] = np.clip(share, 0, 1) * walked * nodes
    # Cadences at k x 0.75 Hz, over 6 Hz, NaN or infinite.
    cad = rng.integers(0, 10, n) * 0.75 + rng.choice([-1e-6, 0.0, 1e-6], n)
    cad[rng.random(n) < 0.02] = np.nan
    cad[rng.random(n) < 0.02] = np.inf
    r["gait_frequency"] = cad
    osc = rng.random(n).astype(F)
    osc[rng.random(n) < 0.03] = np.inf
    r["vertical_oscillation"] = osc
    # Mean heights at the log-axis edges 0.15 * 8^(k/6) m.
    h = 0.15 * 8.0 ** (rng.integers(0, 8, n) / 6.0) * (1 + rng.choice([-1e-6, 0.0, 1e-6], n))
    odd = rng.random(n) < 0.05
    h[odd] = rng.uniform(0.0, 3.0, odd.sum())
    r["height_sum"] = h * walked
    lift = rng.integers(0, 2 ** 10, n, dtype=np.uint64).astype(np.uint32)
    r["lift_lo"] = lift.view(np.float32)
    return r, nodes


def test_metrics_and_cells_match_a_second_restatement():
    w = WORKLOADS["game"]
    world = w.world()
    steps = ce.trial_steps(world)
    rng = np.random.default_rng(11)
    pop = ce.generate(w.spec, 4000)
    res, _ = random_results(len(pop), rng, steps)
    node_counts = pop.genomes["node_count"].astype(np.uint32)
    got = ce.to_metrics(res, node_counts, world)
    for layout in (True, False):
        cells = ce.niche_cells(pop, got, global_layout=layout)
        for i in range(len(pop)):
            want = to_metrics(res[i], int(node_counts[i]), 60, steps)
            for k, v in want.items():
                g = got[i][k]
                assert (g == v) or (np.isnan(g) and np.isnan(v)), (i, k, g, v, res[i])
            n, _, m, _ = pop.creature(i)
            cell, parts = niche(n, len(m), got[i], layout)
            assert cells[i] == cell, (i, layout, cells[i], cell, parts, got[i])


def test_bin_edges_by_hand():
    # bin(): a value on an edge goes to the bin above it, the top edge to
    # the last bin, values outside to the first or last (src/qd.rs:844-846).
    assert bin_of(0.5, 0.0, 1.0, 6) == 3
    assert bin_of(1.0, 0.0, 1.0, 6) == 5
    assert bin_of(-3.0, 0.0, 1.0, 6) == 0
    assert bin_of(0.75, 0.0, 6.0, 8) == 1
    assert bin_of(6.0, 0.0, 6.0, 8) == 7
    # height_axis: 0.15 m -> 0, 1.2 m (0.6 x the 2 m bone limit) -> 1.
    assert height_axis(F(0.15)) == 0 and height_axis(F(1.2)) == 1 and height_axis(F(0.05)) == 0
