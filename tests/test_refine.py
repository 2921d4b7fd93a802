"""Host side of the gradient-refined search (evolution_simulator_gpu_b200/
refine.py): gathering creatures, Gaussian samples on the optimizer's
parameter vector with the reference's clamps (src/qd.rs:2700-2811), and the
clipped ascent step. No GPU is used."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import refine
from evolution_simulator_gpu_b200.configs import WORKLOADS

W = WORKLOADS["refine"]


def _same(a, b):
    return (np.asarray(a).view(np.uint8) == np.asarray(b).view(np.uint8)).all()


def test_take_equals_subset():
    pop = ce.generate(W.spec, 40)
    idx = [7, 3, 7, 39, 0]
    a, b = refine.take(pop, idx), pop.subset(idx)
    for f in ("nodes", "bones", "muscles", "genomes", "strength"):
        assert _same(getattr(a, f), getattr(b, f)), f


def test_samples_keep_the_parameter_limits():
    parents = ce.generate(W.spec, 64)
    pop, parent = refine.samples(parents, 5000, 0.05, seed=9)
    assert len(pop) == 5000 and (parent == np.arange(5000) % 64).all()
    assert (pop.genomes["id"] == 1 + np.arange(5000)).all()
    for f in ("node_count", "bone_count", "muscle_count"):
        assert (pop.genomes[f] == parents.genomes[f][parent]).all()
    n, b, m = pop.nodes, pop.bones, pop.muscles
    assert (n["y"] >= 0).all() and (n["diameter"] >= 0.06).all() and (n["diameter"] <= 0.12).all()
    assert (n["friction"] >= 0).all() and (n["friction"] <= 1).all()
    assert (b["rest_length"] >= 0.03).all() and (b["rest_length"] <= 2.0).all()
    assert (b["min_angle"] <= 0).all() and (b["max_angle"] >= 0).all()
    assert (b["organ_mass"] >= 0).all() and (b["organ_at"] >= 0).all() and (b["organ_at"] <= 1).all()
    assert (m["short"] >= 0.01).all() and (m["long"] >= m["short"]).all() and (m["long"] <= 2.0).all()
    assert (m["phase"] >= 0).all() and (m["phase"] < 1).all()
    assert (m["duty"] >= 0.05).all() and (m["duty"] <= 0.95).all()
    assert (m["stiffness"] >= 1).all() and (m["stiffness"] <= 120).all()
    assert (m["period"] >= 0.2).all() and (m["period"] <= 10).all()
    # One body clock a creature: every muscle's period moves by one factor.
    owner = np.repeat(np.arange(len(pop)), pop.genomes["muscle_count"].astype(np.int64))
    src = refine.take(parents, parent).muscles["period"].astype(np.float64)
    ratio = m["period"] / src
    for c in range(50):
        r = ratio[owner == c]
        assert np.allclose(r, r[0], rtol=1e-5)
    # The moves have the stated spread where no clamp acts.
    dx = n["x"].astype(np.float64) - refine.take(parents, parent).nodes["x"]
    assert abs(dx.std() - 0.05) < 0.002
    ce.pack(pop, W.world())


def test_zero_spread_samples_are_their_parents():
    parents = ce.generate(W.spec, 16)
    pop, parent = refine.samples(parents, 48, 0.0, seed=1)
    same = refine.take(parents, parent)
    for f in ("x", "y", "diameter", "friction"):
        assert (pop.nodes[f] == same.nodes[f]).all()
    for f in ("short", "long", "phase", "duty", "anchor_a", "anchor_b"):
        assert (pop.muscles[f] == same.muscles[f]).all()
    assert np.allclose(pop.muscles["period"], same.muscles["period"], rtol=1e-6)
    assert np.allclose(pop.muscles["stiffness"], same.muscles["stiffness"], rtol=1e-5)


def test_ascent_step_follows_the_gradient_within_its_clip():
    pop = ce.generate(W.spec, 32)
    rng = np.random.default_rng(2)
    gm = rng.normal(size=(len(pop.muscles), 5))
    gn = rng.normal(size=len(pop.nodes))
    assert _same(refine.ascend(pop, np.zeros_like(gm), np.zeros_like(gn), 1e-2).muscles, pop.muscles)
    step = 1e-3
    out = refine.ascend(pop, gm, gn, step)
    m0, m1 = pop.muscles, out.muscles
    T = m0["period"].astype(np.float64)
    d_short = m1["short"].astype(np.float64) - m0["short"]
    free = (m0["short"] > 0.011) & (m0["short"] < 1.59) & (m0["long"] > m0["short"] + 0.01)
    assert np.allclose(d_short[free], step * gm[free, 0], atol=1e-6)
    # The first-order gain <gene gradient, move> is positive: phase and duty
    # moves map back to on and off times.
    dphase = (m1["phase"].astype(np.float64) - m0["phase"] + 0.5) % 1.0 - 0.5
    dduty = m1["duty"].astype(np.float64) - m0["duty"]
    d_on = -T * dphase
    d_off = d_on + T * dduty
    gain = (gm[:, 3] * d_on + gm[:, 4] * d_off).sum()
    assert gain > 0
    # Large gradients move by the coordinate's unit step at most.
    big = refine.ascend(pop, gm * 1e9, gn * 1e9, 1e-2)
    assert np.abs(big.nodes["friction"].astype(np.float64) - pop.nodes["friction"]).max() <= 0.03 + 1e-6
    assert np.abs(big.muscles["duty"].astype(np.float64) - pop.muscles["duty"]).max() <= 0.05 + 1e-6
    # Non-finite gradients do not move a coordinate.
    bad = refine.ascend(pop, np.full_like(gm, np.nan), np.full_like(gn, np.inf), 1e-2)
    assert _same(bad.nodes, pop.nodes)


def test_pick_takes_each_creatures_genes_from_its_chosen_candidate():
    pop = ce.generate(W.spec, 24)
    pop.strength = np.ones(len(pop.muscles), np.float32)
    rng = np.random.default_rng(4)
    cands = [refine.ascend(pop, rng.normal(size=(len(pop.muscles), 5)), rng.normal(size=len(pop.nodes)), 1e-2)
             for _ in range(3)]
    choice = rng.integers(-1, 3, size=len(pop))
    out = refine.pick(cands, choice, pop)
    for c in range(len(pop)):
        src = pop if choice[c] < 0 else cands[choice[c]]
        want, got = src.creature(c), out.creature(c)
        for a, b in zip(want[:3], got[:3]):
            assert _same(a, b), c
        g = pop.genomes[c]
        sl = slice(int(g["muscle_start"]), int(g["muscle_start"] + g["muscle_count"]))
        assert _same(out.strength[sl], src.strength[sl]), c


def test_host_samples_do_not_depend_on_the_range():
    """A sample's moves come from its block's own stream: drawing samples
    [0, 10000) at once or as [0, 3000) and [3000, 10000) gives the same
    genes, as the ranks of a split search rely on."""
    parents = ce.generate(W.spec, 100)
    whole, parent = refine.samples(parents, 10_000, 0.05, seed=4)
    a, pa = refine.samples(parents, 3000, 0.05, seed=4)
    b, pb = refine.samples(parents, 7000, 0.05, seed=4, first=3000)
    joined = refine.concat([a, b])
    for f in ("nodes", "bones", "muscles", "genomes", "strength"):
        assert _same(getattr(whole, f), getattr(joined, f)), f
    assert (np.concatenate([pa, pb]) == parent).all()
    other, _ = refine.samples(parents, 10_000, 0.05, seed=5)
    assert not (other.nodes["x"] == whole.nodes["x"]).all()


def test_sample_rows_count_the_tiled_parents():
    """ce_sample_rows (the device sampler's output sizes): samples
    [first, first + count) of P parents hold the rows of parents
    first mod P, ..., (first + count - 1) mod P."""
    import ctypes as C
    parents = ce.generate(W.spec, 37)
    g = parents.genomes
    for first, count in ((0, 100), (5, 1), (36, 74), (1000, 333), (0, 0)):
        idx = (first + np.arange(count)) % len(parents)
        rows = [C.c_size_t() for _ in range(3)]
        assert ce.lib().ce_sample_rows(ce.api._ptr(g), len(parents), first, count, *[C.byref(r) for r in rows]) == 0
        want = [int(g[f][idx].sum()) for f in ("node_count", "bone_count", "muscle_count")]
        assert [r.value for r in rows] == want


def test_sample_rows_refuse_more_rows_than_32_bit_starts_hold():
    import ctypes as C
    parents = ce.generate(ce.GenSpecPy(seed=2, min_nodes=32, max_nodes=32, min_muscles=96, max_muscles=96,
                                       muscle_rule=1), 1)
    rows = [C.c_size_t() for _ in range(3)]
    g = parents.genomes
    assert ce.lib().ce_sample_rows(ce.api._ptr(g), 1, 0, 40_000_000, *[C.byref(r) for r in rows]) == 0
    assert ce.lib().ce_sample_rows(ce.api._ptr(g), 1, 0, 50_000_000, *[C.byref(r) for r in rows]) \
        == ce.CE_ERR_INVALID
    assert b"2^32" in ce.lib().ce_last_error()
