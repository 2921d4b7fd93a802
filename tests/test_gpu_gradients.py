"""The gradient path on the GPU (ce_forward / ce_backward) against the FP64
dual-number tangent of the host physics and FP64 finite differences.

The backward kernel differentiates the FP32 trajectory the forward kernel
took, through its contact, stick/slip, joint-limit and clamp modes. The FP64
tangent (oracle/creature_oracle.cpp) differentiates the FP64 trajectory of
the same trial; the two agree while the trajectories take the same modes,
which holds for nearly every creature over a few steps and for fewer as the
trial grows (a mode taken differently near a threshold changes the
derivative), so the checks below are on short trials. Central differences
of the FP32 kernel are not a usable check: its trajectories respond to
record changes below about 1e-2 relative with rounding noise.
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS, effects_world_kw
from oracle.ref import Oracle

pytestmark = pytest.mark.gpu

W = WORKLOADS["gradients"]
R = WORKLOADS["refine"]


def _record_direction(wave, rows, mm, rng, part="records"):
    """A random direction in the record fields (muscle fields, friction,
    mass) or in the start positions alone."""
    n = len(wave)
    dm = rng.normal(size=(n, mm, 9))
    dn = rng.normal(size=(n, rows))
    dmass = rng.normal(size=(n, rows)) * 0.01
    ds = rng.normal(size=(n, rows, 2))
    if part == "records":
        ds[:] = 0.0
    else:
        dm[:], dn[:], dmass[:] = 0.0, 0.0, 0.0
    for c in range(n):
        nodes = int(wave.heads[c, 0] & 255)
        dm[c, int(wave.heads[c, 1]):] = 0.0
        dn[c, nodes:] = 0.0
        dmass[c, nodes:] = 0.0
        ds[c, nodes:] = 0.0
    return dm, dn, dmass, ds


def _project(g, rows, mm, dm, dn, dmass, ds):
    g = g.astype(np.float64)
    n = len(g)
    return ((g[:, :9 * mm].reshape(n, mm, 9) * dm).sum(axis=(1, 2)) + (g[:, 9 * mm:9 * mm + rows] * dn).sum(axis=1)
            + (g[:, 9 * mm + rows:9 * mm + 2 * rows] * dmass).sum(axis=1)
            + (g[:, 9 * mm + 2 * rows:9 * mm + 4 * rows] * ds.reshape(n, 2 * rows)).sum(axis=1))


@pytest.mark.parametrize("name,quake", [("gradients", True), ("refine", True), ("refine", False)])
def test_forward_results_equal_the_plain_kernel(engine, name, quake):
    w = WORKLOADS[name]
    world = w.world(duration=2.0) if quake else w.world(duration=2.0, quake=0.0)
    wave = ce.pack(ce.generate(w.spec, 4096), world)
    plain, _ = engine.run(wave, world)
    with engine.forward(wave, world) as tape:
        res = tape.results
    assert (res.view(np.uint32) == plain.view(np.uint32)).all()


@pytest.mark.parametrize("name,part,seconds,median,share", [
    ("gradients", "records", 0.05, 1e-4, 0.95), ("gradients", "records", 0.25, 1e-3, 0.55),
    ("refine", "records", 0.05, 1e-4, 0.9), ("refine", "records", 0.25, 1e-3, 0.5),
    ("gradients", "start", 0.1, 1e-4, 0.9), ("refine", "start", 0.1, 1e-4, 0.9)])
def test_adjoint_matches_fp64_tangent(engine, name, part, seconds, median, share):
    """<gradient, u> against the FP64 tangent along u for 256 creatures, u a
    random direction in the record fields (muscles, friction, mass) or in the
    start positions, in the calm world and in the refined-search world
    (rough ground with hurdles and tremors, water, ice, wind, thick air)."""
    w = WORKLOADS[name]
    world = w.world(duration=seconds)
    wave = ce.pack(ce.generate(w.spec, 256), world)
    with engine.forward(wave, world) as tape:
        g = tape.backward()
        rows, mm = tape.shape
        res = tape.results
    dm, dn, dmass, ds = _record_direction(wave, rows, mm, np.random.default_rng(7), part)
    tangent, _, _ = Oracle().tangent(wave, ce.make_params(world), ce.world_flags(world), dm, dn, dmass=dmass,
                                     dstart=ds)
    adj = _project(g, rows, mm, dm, dn, dmass, ds)
    ok = res["fitness"] > -1e19
    rel = np.abs(adj - tangent)[ok] / np.maximum(np.abs(tangent[ok]), 1e-12)
    assert np.median(rel) < median, np.median(rel)
    assert (rel < 1e-3).mean() >= share, (rel < 1e-3).mean()


# Record float index of each gradient field of a muscle (kernel record layout).
FIELDS = [8, 3, 4, 5, 10, 11, 12, 13, 14]


def _record_change(wa, wb, h):
    """d records / d h of a one-creature pack by central differences: the
    gradient's record fields (muscle fields, friction, mass, start x and y)
    as (muscle, node, mass, start) direction arrays for the FP64 tangent."""
    M, N = int(wa.heads[0, 1]), int(wa.heads[0, 0] & 255)
    mo, ro = int(wa.heads[0, 4]), int(wa.heads[0, 3])
    la, lb = wa.lanes.view(np.float32).astype(np.float64), wb.lanes.view(np.float32).astype(np.float64)
    ma, mb = wa.muscles.astype(np.float64), wb.muscles.astype(np.float64)
    dm = np.zeros((1, M, 9))
    for k in range(M):
        dm[0, k] = (ma[mo + 20 * k + np.array(FIELDS)] - mb[mo + 20 * k + np.array(FIELDS)]) / (2 * h)
    rows = ro + 6 * np.arange(N)
    dn = ((la[rows + 2] - lb[rows + 2]) / (2 * h))[None]
    dmass = ((la[rows] - lb[rows]) / (2 * h))[None]
    ds = np.stack([(la[rows + 3] - lb[rows + 3]) / (2 * h), (la[rows + 4] - lb[rows + 4]) / (2 * h)], 1)[None]
    return dm, dn, dmass, ds


def test_adjoint_at_the_fine_rate_matches_fp64_tangent(engine):
    """The 120 steps/s kernels (the reference's fine fidelity): the adjoint
    against the FP64 tangent along random record directions, over 96
    substeps (the 60 steps/s comparisons at that length agree as often)."""
    world = W.world(duration=0.05, rate=120)
    wave = ce.pack(ce.generate(W.spec, 256), world)
    with engine.forward(wave, world) as tape:
        g = tape.backward()
        rows, mm = tape.shape
        res = tape.results
    dm, dn, dmass, ds = _record_direction(wave, rows, mm, np.random.default_rng(9))
    tangent, _, _ = Oracle().tangent(wave, ce.make_params(world), ce.world_flags(world), dm, dn, rate=120,
                                     dmass=dmass)
    adj = _project(g, rows, mm, dm, dn, dmass, ds)
    ok = res["fitness"] > -1e19
    rel = np.abs(adj - tangent)[ok] / np.maximum(np.abs(tangent[ok]), 1e-12)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert (rel < 1e-3).mean() >= 0.8, (rel < 1e-3).mean()


@pytest.mark.parametrize("name,count,seconds", [("gradients", 64, 0.1), ("refine", 384, 0.05)])
def test_gene_gradients_match_fp64_differences(engine, name, count, seconds):
    """End to end: GPU record gradient, gene chain rule, against central
    differences of the FP64 host physics over repacked genes (h = 2e-4),
    where the FP64 fitness is differentiable at the genes: its one-sided
    differences agree, and its FP64 tangent along the packer's record
    change equals the central difference. The second test matters on uneven
    ground, where the start pose rests its lowest node exactly on the
    ground: whether a repacked pose touches there turns on rounding, and the
    contact branch has other derivatives than the free one."""
    w = WORKLOADS[name]
    world = w.world(duration=seconds)
    pop = ce.generate(w.spec, count)
    wave = ce.pack(pop, world)
    with engine.forward(wave, world) as tape:
        g = tape.backward()
        shape = tape.shape
    mg, ng = ce.gene_gradients(pop, wave, world, g, shape)
    rng = np.random.default_rng(11)
    o = Oracle()
    p, flags = ce.make_params(world), ce.world_flags(world)
    checked = agree = 0
    for c in range(len(wave)):
        i = int(wave.slots[c])
        one = pop.subset([i])
        m = one.muscles
        vm = rng.normal(size=(len(m), 5))
        vn = rng.normal(size=len(one.nodes))
        # No on/off move where duty sits at its clamp or phase near its wrap.
        kink = (m["duty"] <= 0.0501) | (m["duty"] >= 0.9499) | (m["phase"] < 0.01) | (m["phase"] > 0.99)
        vm[kink, 3:] = 0.0

        def moved(h):
            mm_ = m.copy()
            nn = one.nodes.copy()
            T = mm_["period"].astype(np.float64)
            mm_["short"] = (mm_["short"] + h * vm[:, 0]).astype(np.float32)
            mm_["long"] = (mm_["long"] + h * vm[:, 1]).astype(np.float32)
            mm_["phase"] = (mm_["phase"] - h * vm[:, 3] / T).astype(np.float32)
            mm_["duty"] = (mm_["duty"] + h * (vm[:, 4] - vm[:, 3]) / T).astype(np.float32)
            nn["friction"] = (nn["friction"] + h * vn).astype(np.float32)
            st = (one.strength + h * vm[:, 2]).astype(np.float32)
            return ce.pack(ce.Population(nn, one.bones, mm_, one.genomes, st), world)

        def fitness(w1):
            o.tangent(w1, p, flags, np.zeros((1, int(w1.heads[0, 1]), 9)), np.zeros((1, int(w1.heads[0, 0] & 255))))
            return float(o.fitness64[0])

        h = 2e-4
        w0 = moved(0.0)
        f0, fp, fm = fitness(w0), fitness(moved(h)), fitness(moved(-h))
        up, down = (fp - f0) / h, (f0 - fm) / h
        if abs(up - down) > 0.05 * max(abs(up), abs(down)) + 1e-9:
            continue
        fd = (fp - fm) / (2 * h)
        dm, dn, dmass, ds = _record_change(moved(1e-3), moved(-1e-3), 1e-3)
        along, _, _ = o.tangent(w0, p, flags, dm, dn, dmass=dmass, dstart=ds)
        if abs(float(along[0]) - fd) > 2e-2 * max(abs(fd), 1e-6):
            continue
        gs = pop.genomes[i]
        got = float((mg[gs["muscle_start"]:gs["muscle_start"] + gs["muscle_count"]] * vm).sum()
                    + (ng[gs["node_start"]:gs["node_start"] + gs["node_count"]] * vn).sum())
        checked += 1
        agree += abs(got - fd) <= 2e-2 * max(abs(fd), 1e-6)
    assert checked >= 20, checked
    assert agree >= 0.8 * checked, (agree, checked)


def test_backward_is_linear_in_the_fitness_weights(engine):
    """Weights scale each creature's gradient (up to FP32 rounding, compared
    where the gradient is moderate: trials whose gradients explode through
    near-degenerate joint configurations amplify rounding)."""
    world = W.world(duration=0.25)
    wave = ce.pack(ce.generate(W.spec, 512), world)
    with engine.forward(wave, world) as tape:
        g1 = tape.backward()
        w = np.random.default_rng(3).normal(size=len(wave)).astype(np.float32)
        gw = tape.backward(w)
        g0 = tape.backward(np.zeros(len(wave), np.float32))
    assert (g0 == 0).all()
    moderate = np.isfinite(g1).all(axis=1) & (np.abs(g1).max(axis=1) < 1e3)
    assert moderate.mean() > 0.8
    a, b = gw[moderate], (g1 * w[:, None])[moderate]
    close = np.abs(a - b) <= 1e-3 * np.abs(b) + 1e-6 * np.abs(b).max()
    assert close.mean() > 0.999, close.mean()


def test_gradients_refuse_unsupported_batches(engine):
    muddy = ce.make_world(duration=1.0, **dict(effects_world_kw(), mud=0.5))
    wave = ce.pack(ce.generate(W.spec, 16), muddy)
    with pytest.raises(ce.EngineError) as err:
        engine.forward(wave, muddy)
    assert err.value.status == ce.CE_ERR_UNSUPPORTED
    world = W.world(duration=1.0)
    wave = ce.pack(ce.generate(W.spec, 16), world)
    sensed = ce.WavePack(wave.lanes, wave.muscles.copy(), wave.heads, wave.slots, wave.info)
    sensed.muscles.view(np.uint32)[int(wave.heads[0, 4]) + 16] = 0
    with pytest.raises(ce.EngineError) as err:
        engine.forward(sensed, world)
    assert err.value.status == ce.CE_ERR_UNSUPPORTED
    with pytest.raises(ce.EngineError):
        engine.forward(wave, world, checkpoint_every=128)
    # Bodies whose backward tables do not fit a block's shared memory.
    big = ce.GenSpecPy(seed=9, min_nodes=32, max_nodes=32, muscle_rule=1, min_muscles=96, max_muscles=96)
    wave = ce.pack(ce.generate(big, 8), world)
    with pytest.raises(ce.EngineError) as err:
        engine.forward(wave, world)
    assert err.value.status == ce.CE_ERR_UNSUPPORTED


def test_checkpoints_hold_the_state_every_16_steps(engine):
    """The forward run's checkpoints (stored creature-minor on the device,
    returned per creature): checkpoint 0 is the packed start pose at rest
    with full energy stores, and the positions of checkpoint 2 (after 32
    steps) put the centre of mass where a 32-step trial of the plain kernel
    ends (its fitness)."""
    world = W.world(duration=1.0)
    wave = ce.pack(ce.generate(W.spec, 1024), world)
    with engine.forward(wave, world) as tape:
        ck = tape.checkpoints(ce.trial_steps(world))
        rows, mm = tape.shape
    short = W.world(duration=32.0 / 60.0)
    assert ce.trial_steps(short) == 32
    res, _ = engine.run(wave, short)
    lf = wave.lanes.view(np.float32)
    com = np.zeros(len(wave))
    for c in range(len(wave)):
        n, m, ro = int(wave.heads[c, 0] & 255), int(wave.heads[c, 1]), int(wave.heads[c, 3])
        start = np.stack([lf[ro + 6 * np.arange(n) + 3], lf[ro + 6 * np.arange(n) + 4]], axis=1).reshape(-1)
        assert (ck[c, 0, :2 * n] == start).all(), c
        assert (ck[c, 0, 2 * rows:2 * rows + 2 * n] == 0).all(), c
        assert (ck[c, 0, 4 * rows:4 * rows + m] == 1).all(), c
        mass = lf[ro + 6 * np.arange(n)].astype(np.float64)
        com[c] = (mass * ck[c, 2, 0:2 * n:2]).sum() / mass.sum()
    # Bodies that fall within the 32 steps (about a third, toppling as they
    # settle) end their trial before checkpoint 2.
    ok = (res["fall_time"] == 0) & (res["fitness"] > -1e19)
    assert ok.sum() >= 256, ok.sum()
    assert np.allclose(com[ok], res["fitness"][ok], rtol=1e-5, atol=1e-5)


@pytest.fixture(scope="module")
def tangent_cases(engine):
    """Per world and trial length: the backward's gradient terms and the
    tangent-linear run's d fitness along random directions of the start
    positions, the muscle record fields, the frictions and the masses (each
    part alone),
    and which trials count; computed once, on first use."""
    cache = {}

    def get(name, seconds):
        if (name, seconds) in cache:
            return cache[name, seconds]
        w = WORKLOADS[name]
        world = w.world(duration=seconds)
        wave = ce.pack(ce.generate(w.spec, 256), world)
        n = len(wave)
        with engine.forward(wave, world) as tape:
            rows, mm = tape.shape
            g = tape.backward().astype(np.float64)
            res = tape.results
            rng = np.random.default_rng(11)
            nodes, muscles = (wave.heads[:, 0] & 255).astype(int), wave.heads[:, 1].astype(int)
            ds = rng.normal(size=(n, rows, 2)).astype(np.float32)
            dm = rng.normal(size=(n, mm, 9)).astype(np.float32)
            df = rng.normal(size=(n, rows)).astype(np.float32)
            dn = rng.normal(size=(n, rows)).astype(np.float32)
            for c in range(n):
                ds[c, nodes[c]:], df[c, nodes[c]:], dm[c, muscles[c]:], dn[c, nodes[c]:] = 0, 0, 0, 0
            parts = {
                "start": (tape.tangent(dstart=ds), g[:, 9 * mm + 2 * rows:9 * mm + 4 * rows] * ds.reshape(n, -1)),
                "muscle": (tape.tangent(dmuscle=dm), g[:, :9 * mm] * dm.reshape(n, -1)),
                "friction": (tape.tangent(dfriction=df), g[:, 9 * mm:9 * mm + rows] * df),
                "mass": (tape.tangent(dmass=dn), g[:, 9 * mm + rows:9 * mm + 2 * rows] * dn),
            }
        cache[name, seconds] = (parts, res["fitness"] > -1e19)
        return cache[name, seconds]

    return get


@pytest.mark.parametrize("part", ["start", "muscle", "friction", "mass"])
@pytest.mark.parametrize("seconds,share", [(16.0 / 60.0, 0.98), (20.0, 0.95)])
@pytest.mark.parametrize("name", ["gradients", "refine", "effects"])
def test_adjoint_equals_the_tangent_linear_run(tangent_cases, name, part, seconds, share):
    """The dot-product test of the adjoint: for a random direction u of the
    start positions, of the muscles' record fields, of the frictions or of the
    node masses,
    <backward's gradient, u> against the tangent-linear run (ce_tangent)
    along u. Both differentiate the forward run's own FP32 trajectory with
    its contact, slip and joint-limit modes, so they differ only by the
    rounding of the two FP32 derivative computations (the FP64 tangent of the
    oracle takes its own modes). 256 creatures in the calm world of config 4,
    the refined-search world of config 5 (rough ground with hurdles and
    tremors, water, ice, wind, thick air) and the effects world, over one
    16-step segment and over 20 s, where derivatives reach 1e30 on
    near-degenerate joints. The difference is measured against the sum of
    the dot product's term magnitudes (a dot product of terms that cancel
    loses their rounding relative to itself); the plain relative
    difference's median is bounded too."""
    parts, ok = tangent_cases(name, seconds)
    tan, terms = parts[part]
    adj = terms.sum(axis=1)
    ok = ok & np.isfinite(adj) & np.isfinite(tan)
    assert ok.mean() > 0.95
    diff = np.abs(adj - tan.astype(np.float64))[ok]
    scaled = diff / np.maximum(np.abs(terms).sum(axis=1)[ok], 1e-30)
    assert (scaled < 1e-3).mean() >= share, (scaled < 1e-3).mean()
    assert (scaled < 1e-2).mean() >= 0.99, (scaled < 1e-2).mean()
    assert np.median(diff / np.maximum(np.abs(tan[ok]), 1e-30)) < 2e-4


@pytest.mark.parametrize("name,count,seconds", [("gradients", 1024, 2.0), ("refine", 1024, 2.0),
                                                 ("effects", 1024, 2.0), ("gradients", 256, 20.0)])
def test_backward_reruns_reproduce_the_forward_run(engine, name, count, seconds):
    """The backward reruns every segment from its checkpoint and every
    substep from the segment tape; its gradients are those of the forward
    run only if those reruns land on the forward run's own states. The
    checked backward compares, to the bit, each segment's rerun with the
    next checkpoint and each substep's kept rerun with the next tape state,
    in the calm world, the refined-search world (tremors) and the effects
    world, and over config 4's 20 s trials, and its gradients equal the
    unchecked backward's."""
    w = WORKLOADS[name]
    world = w.world(duration=seconds)
    wave = ce.pack(ce.generate(w.spec, count), world)
    with engine.forward(wave, world) as tape:
        plain = tape.backward()
        checked, bad = tape.backward(check=True)
    assert (bad == 0).all(), f"{int((bad != 0).sum())} creatures' reruns left the forward run (bits {np.unique(bad)})"
    assert (plain.view(np.uint32) == checked.view(np.uint32)).all()
