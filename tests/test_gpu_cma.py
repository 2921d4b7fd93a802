"""CMA-ES emitters on the device (ce_cma_init / ask / tell) against the
float32 restatement of the reference's emitters (oracle/cma_ref.py,
src/qd.rs:2130-2474) and of its breeding streams (src/evolution.rs:455-600).

Ask is bit-exact: given the emitter state the device holds, every drawn
coordinate equals the restatement's, and so does every gene except an
optimizer's period and stiffness, which go through exp (CUDA's against
numpy's: a few units in the last place). The means of optimizers go through
ln for the same two coordinates. Tell's outputs are compared with tolerances
sized from those ulps: a log coordinate off by one ulp (5e-7 at ln 120)
moves a normalised step y by 5e-7 / (sigma x 0.1).
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import cma, refine
from oracle import cma_ref as R

pytestmark = pytest.mark.gpu

SPEC = ce.GenSpecPy(seed=5, min_nodes=3, max_nodes=10, max_muscles=20)
NODE_FIELDS = ("x", "y", "diameter", "friction")
BONE_FIELDS = ("a", "b", "rest_length", "min_angle", "max_angle", "organ_mass", "organ_at")
EXACT_MUSCLE = ("bone_a", "bone_b", "anchor_a", "anchor_b", "short", "long", "phase", "duty", "sensor", "reset",
                "tendon")
MODES = {"optimizer": False, "cma-me": True, "mixed": [0, 1, 1, 0, 1, 0], "cma-me-fresh": True}


def body(pop, i):
    g = pop.genomes[i]
    return (pop.nodes[g["node_start"]:g["node_start"] + g["node_count"]].copy(),
            pop.bones[g["bone_start"]:g["bone_start"] + g["bone_count"]].copy(),
            pop.muscles[g["muscle_start"]:g["muscle_start"] + g["muscle_count"]].copy())


def modes(mode, E):
    m = MODES[mode]
    return np.resize(np.asarray(m, bool), E) if isinstance(m, list) else np.full(E, m)


def log_mask(n, b, m):
    mask = np.zeros(4 * n + 5 * b + 1 + 8 * m, bool)
    mask[4 * n + 5 * b] = True
    mask[4 * n + 5 * b + 1 + 6::8] = True
    return mask


def random_state(opt, rng):
    for e in range(len(opt)):
        mean, cov, pc, ps, sig = opt.state(e)
        D = len(mean)
        explores = opt.exploring is not None and opt.exploring[e]
        sig = rng.uniform(0.05, 0.3) if explores else rng.uniform(0.2, 0.8)
        opt.set_state(e, mean, rng.uniform(0.3, 3.0, D), rng.normal(0, 0.5, D), rng.normal(0, 0.5, D), sig)


@pytest.mark.parametrize("mode", ["optimizer", "cma-me"])
def test_init_puts_the_means_at_the_templates(engine, mode):
    pop = ce.generate(SPEC, 40)
    ex = modes(mode, 40)
    opt = cma.CmaEmitters(pop, exploring=ex)
    for e in range(len(pop)):
        t = body(pop, e)
        mean, cov, pc, ps, sig = opt.state(e)
        assert (cov == 1).all() and (pc == 0).all() and (ps == 0).all()
        if ex[e]:
            assert (mean == R.explore_parameters(*t)).all() and sig == np.float32(0.12)
            continue
        p = R.parameters(*t)
        logs = log_mask(*map(len, t))
        assert (mean[~logs] == p[~logs]).all() and sig == np.float32(0.5)
        np.testing.assert_allclose(mean[logs], p[logs], rtol=4e-7, atol=4e-7)


@pytest.mark.parametrize("mode", ["optimizer", "cma-me", "mixed", "cma-me-fresh"])
def test_ask_is_the_references_sample(engine, mode):
    # "fresh": the state CmaEmitter::new leaves, a zero evolution path, so
    # no rank-one term and the genes' sub-stream at the cursor's first draw.
    E, count = 30, 600
    pop = ce.generate(SPEC, E)
    ex = modes(mode, E)
    opt = cma.CmaEmitters(pop, exploring=ex)
    if not mode.endswith("fresh"):
        random_state(opt, np.random.default_rng(1))
    states = [opt.state(e) for e in range(E)]
    draw = dict(seed=9, generation=4, round=2, first_id=100, strength=1.5, friction=(0.0, 1.0))
    genes, vals = opt.ask_device(count, values=True, first=77, **draw)
    vals = vals.cpu().numpy()
    got = opt.download(genes)
    # The layout is ce_sample_device's for the same parents.
    lay, _ = refine.samples_gpu(pop, count, 0.0, seed=0, first_id=100, first=77)
    assert (got.genomes == lay.genomes).all()
    assert (got.strength == lay.strength).all()
    for c in range(count):
        g = 77 + c
        e = g % E
        t = body(pop, e)
        D = len(states[e][0])
        want_v = R.sample(states[e], t, ex[e], g, seed=9, generation=4, round_=2, strength=1.5)
        assert (vals[c, :D] == want_v).all(), (c, np.flatnonzero(vals[c, :D] != want_v)[:5])
        if ex[e]:
            want = R.apply_explore(*t, want_v, friction=(0.0, 1.0))
        else:
            want = R.apply(*t, want_v, friction=(0.0, 1.0))
        have = body(got, c)
        for f in NODE_FIELDS:
            assert (have[0][f] == want[0][f]).all(), (c, f)
        for f in BONE_FIELDS:
            assert (have[1][f] == want[1][f]).all(), (c, f)
        for f in EXACT_MUSCLE:
            assert (have[2][f] == want[2][f]).all(), (c, f)
        for f in ("period", "stiffness"):
            if ex[e]:
                assert (have[2][f] == want[2][f]).all(), (c, f)
            else:
                np.testing.assert_allclose(have[2][f], want[2][f], rtol=6e-7)


def test_ask_does_not_depend_on_the_range(engine):
    pop = ce.generate(SPEC, 16)
    opt = cma.CmaEmitters(pop, exploring=modes("mixed", 16))
    random_state(opt, np.random.default_rng(2))
    _, whole = opt.ask_device(4000, seed=3, generation=1, values=True, first=0)
    _, a = opt.ask_device(1234, seed=3, generation=1, first=0, values=True)
    _, b = opt.ask_device(4000 - 1234, seed=3, generation=1, first=1234, values=True)
    whole = whole.cpu().numpy()
    assert (np.concatenate([a.cpu().numpy(), b.cpu().numpy()]) == whole).all()
    _, other = opt.ask_device(4000, seed=3, generation=2, values=True, first=0)
    assert (other.cpu().numpy() != whole).any()


@pytest.mark.parametrize("mode,per_emitter", [("optimizer", 7), ("optimizer", 1500), ("cma-me", 7),
                                              ("cma-me", 1500), ("mixed", 40)])
def test_tell_matches_the_restatement(engine, mode, per_emitter):
    E = 6
    pop = ce.generate(SPEC, E)
    ex = modes(mode, E)
    opt = cma.CmaEmitters(pop, exploring=ex)
    rng = np.random.default_rng(per_emitter)
    random_state(opt, rng)
    before = [opt.state(e) for e in range(E)]
    count = E * per_emitter
    first = 3 * E + 2  # the range need not start at emitter 0
    samples = opt.ask(count, seed=4, first=first, friction=(0.0, 1.0))
    keys = rng.normal(1.0, 1.0, count).astype(np.float32)
    keys[rng.random(count) < 0.1] = R.FAILED
    keys[rng.random(count) < 0.02] = np.nan
    keys[rng.random(count) < 0.02] = -np.inf
    keys[[c for c in range(count) if (first + c) % E == 4]] = R.FAILED  # emitter 4 keeps nothing
    opt.tell(samples, keys, first=first)
    for e in range(E):
        mine = [c for c in range(count) if (first + c) % E == e]
        want = R.tell(before[e], body(pop, e), [body(samples, c) for c in mine], keys[mine], ex[e])
        have = opt.state(e)
        if e == 4:
            for x, y in zip(have, before[e]):
                assert (np.asarray(x) == np.asarray(y)).all()
            continue
        np.testing.assert_allclose(have[0], want[0], rtol=1e-5, atol=2e-6)   # mean
        np.testing.assert_allclose(have[1], want[1], rtol=1e-4, atol=1e-5)   # covariance
        np.testing.assert_allclose(have[2], want[2], rtol=1e-4, atol=1e-4)   # path_c
        np.testing.assert_allclose(have[3], want[3], rtol=1e-4, atol=1e-4)   # path_sigma
        np.testing.assert_allclose(have[4], want[4], rtol=1e-5)               # sigma


@pytest.mark.parametrize("mode", ["optimizer", "cma-me"])
def test_tell_drops_samples_of_another_plan(engine, mode):
    # cma_feedback_ignores_candidates_with_changed_topology (src/qd.rs:3033-3050),
    # on the device: every sample of emitter 1 has its first muscle moved to
    # another bone, so emitter 1 keeps its state and the others update.
    E = 3
    pop = ce.generate(SPEC, E)
    opt = cma.CmaEmitters(pop, exploring=modes(mode, E))
    samples = opt.ask(E * 8, seed=1, first=0)
    g = samples.genomes
    for c in range(1, E * 8, E):
        first_muscle = g["muscle_start"][c]
        bones = g["bone_count"][c]
        samples.muscles["bone_b"][first_muscle] = (samples.muscles["bone_b"][first_muscle] + 1) % bones
    before = [opt.state(e) for e in range(E)]
    opt.tell(samples, np.arange(E * 8, dtype=np.float32))
    after = [opt.state(e) for e in range(E)]
    for x, y in zip(after[1], before[1]):
        assert (np.asarray(x) == np.asarray(y)).all()
    for e in (0, 2):
        assert after[e][4] != before[e][4] and not (after[e][0] == before[e][0]).all()


@pytest.mark.parametrize("mode", ["optimizer", "cma-me"])
def test_emitter_moves_toward_its_better_samples(engine, mode):
    # optimizer_moves_toward_its_faster_samples (src/qd.rs:3071-3094), on the device.
    pop = ce.generate(SPEC, 1)
    opt = cma.CmaEmitters(pop, exploring=modes(mode, 1))
    shifted = refine.take(pop, np.zeros(4, np.int64))
    own = refine._owner(shifted, "node_start", "node_count")
    for k, shift in enumerate((0.05, -0.05, 0.04, -0.04)):
        shifted.nodes["x"][own == k] += np.float32(shift)
    before = opt.state(0)[0][0]
    opt.tell(shifted, np.array([4.0, 1.0, 3.0, 2.0], np.float32), first=0)
    assert opt.state(0)[0][0] > before


@pytest.mark.parametrize("mode", ["optimizer", "cma-me"])
def test_tell_breaks_ties_by_sample_index(engine, mode):
    # Keys rounded to 0.5 tie in runs that straddle the cut at the mu best;
    # the device sorts ties by sample index, as the restatement does (the
    # reference's unstable sort leaves their order open).
    E = 3
    pop = ce.generate(SPEC, E)
    ex = modes(mode, E)
    opt = cma.CmaEmitters(pop, exploring=ex)
    rng = np.random.default_rng(11)
    random_state(opt, rng)
    before = [opt.state(e) for e in range(E)]
    count = E * 60
    samples = opt.ask(count, seed=8, first=0, friction=(0.0, 1.0))
    keys = (np.round(rng.normal(1.0, 1.0, count) * 2.0) / 2.0).astype(np.float32)
    assert len(np.unique(keys)) < count // 4
    opt.tell(samples, keys, first=0)
    for e in range(E):
        mine = [c for c in range(count) if c % E == e]
        want = R.tell(before[e], body(pop, e), [body(samples, c) for c in mine], keys[mine], ex[e])
        have = opt.state(e)
        np.testing.assert_allclose(have[0], want[0], rtol=1e-5, atol=2e-6)
        np.testing.assert_allclose(have[1], want[1], rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(have[4], want[4], rtol=1e-5)


@pytest.mark.parametrize("mode", ["optimizer", "cma-me"])
def test_bodies_at_the_engines_limits(engine, mode):
    # 32 nodes and 96 muscles: 1,052 optimizer coordinates (927 CMA-ME), the
    # size of the tell kernel's shared coordinate arrays.
    spec = ce.GenSpecPy(seed=9, min_nodes=32, max_nodes=32, min_muscles=96, max_muscles=96, muscle_rule=1)
    E = 2
    pop = ce.generate(spec, E)
    ex = modes(mode, E)
    opt = cma.CmaEmitters(pop, exploring=ex)
    rng = np.random.default_rng(21)
    random_state(opt, rng)
    before = [opt.state(e) for e in range(E)]
    assert len(before[0][0]) == (927 if ex[0] else 1052)
    count = E * 24
    genes, vals = opt.ask_device(count, seed=2, first=0, values=True, friction=(0.0, 1.0))
    vals = vals.cpu().numpy()
    samples = opt.download(genes)
    for c in range(count):
        e = c % E
        want_v = R.sample(before[e], body(pop, e), ex[e], c, seed=2)
        assert (vals[c, :len(want_v)] == want_v).all()
    keys = rng.normal(1.0, 1.0, count).astype(np.float32)
    opt.tell(samples, keys, first=0)
    for e in range(E):
        mine = list(range(e, count, E))
        want = R.tell(before[e], body(pop, e), [body(samples, c) for c in mine], keys[mine], ex[e])
        have = opt.state(e)
        np.testing.assert_allclose(have[0], want[0], rtol=1e-5, atol=2e-6)
        np.testing.assert_allclose(have[1], want[1], rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(have[2], want[2], rtol=1e-4, atol=1e-4)
        np.testing.assert_allclose(have[3], want[3], rtol=1e-4, atol=1e-4)
        np.testing.assert_allclose(have[4], want[4], rtol=1e-5)


@pytest.mark.parametrize("mode", ["optimizer", "cma-me"])
def test_recentered_keeps_the_learned_steps_for_the_same_plan(engine, mode):
    # CmaEmitter::recentered (src/qd.rs:2166-2177): emitter 0 restarts from a
    # body of its own plan (keeps covariance, paths and step size), emitter 1
    # from a body whose first muscle joins other bones (restarts), emitter 2
    # from a body of other counts (rejected: left as it was).
    E = 3
    pop = ce.generate(SPEC, E)
    ex = modes(mode, E)
    opt = cma.CmaEmitters(pop, exploring=ex)
    random_state(opt, np.random.default_rng(31))
    before = [opt.state(e) for e in range(E)]
    samples = opt.ask(E, seed=5, first=0, friction=(0.0, 1.0))
    other = ce.generate(ce.GenSpecPy(seed=77, min_nodes=3, max_nodes=10, max_muscles=20), 50)
    k = int(np.flatnonzero(other.genomes["node_count"] != pop.genomes["node_count"][2])[0])
    bodies = refine.concat([refine.take(samples, np.array([0, 1])), refine.take(other, np.array([k]))])
    m1 = int(bodies.genomes["muscle_start"][1])
    bodies.muscles["bone_b"][m1] = (bodies.muscles["bone_b"][m1] + 1) % bodies.genomes["bone_count"][1]
    rejected = opt.recenter([0, 1, 2], bodies)
    assert list(rejected) == [False, False, True]
    for e in range(2):
        want = R.recentered(before[e], body(pop, e), body(bodies, e), ex[e])
        have = opt.state(e)
        if ex[e]:
            assert (have[0] == want[0]).all()
        else:
            np.testing.assert_allclose(have[0], want[0], rtol=4e-7, atol=4e-7)
        for x, y in zip(have[1:], want[1:]):
            assert (np.asarray(x) == np.asarray(y)).all()
    assert (opt.state(0)[1] == before[0][1]).all() and opt.state(0)[4] == before[0][4]
    assert (opt.state(1)[1] == 1).all() and opt.state(1)[4] == np.float32(0.12 if ex[1] else 0.5)
    for x, y in zip(opt.state(2), before[2]):
        assert (np.asarray(x) == np.asarray(y)).all()
    # The device templates follow: the next ask samples around the new bodies.
    t = opt.templates
    assert (opt._t[0].cpu().numpy().view(t.nodes.dtype) == t.nodes).all()
    assert (opt._t[2].cpu().numpy().view(t.muscles.dtype) == t.muscles).all()
    assert (t.nodes[:int(t.genomes["node_count"][0])] == body(bodies, 0)[0]).all()
    # converged (src/qd.rs:2184-2187): an optimizer below a step size of 0.05.
    s0 = opt.state(0)
    opt.set_state(0, *s0[:4], 0.04)
    assert opt.converged()[0] == (not ex[0]) and not opt.converged()[1]


def test_saved_emitters_resume_where_they_stopped(engine, tmp_path):
    # A save and a load between two generations: the resumed emitters hold
    # the same state and draw the same next samples, to the bit.
    E = 5
    pop = ce.generate(SPEC, E)
    opt = cma.CmaEmitters(pop, exploring=modes("mixed", E))
    rng = np.random.default_rng(41)
    for gen in range(2):
        kids = opt.ask(E * 12, seed=3, generation=gen, friction=(0.0, 1.0))
        opt.tell(kids, rng.normal(1.0, 1.0, len(kids)).astype(np.float32))
    opt.save(tmp_path / "emitters.npz")
    back = cma.CmaEmitters.load(tmp_path / "emitters.npz")
    assert back.asked == opt.asked
    for e in range(E):
        for x, y in zip(back.state(e), opt.state(e)):
            assert (np.asarray(x) == np.asarray(y)).all()
    a = opt.ask(E * 12, seed=3, generation=2, friction=(0.0, 1.0))
    b = back.ask(E * 12, seed=3, generation=2, friction=(0.0, 1.0))
    for f in ("nodes", "bones", "muscles", "genomes", "strength"):
        assert (getattr(a, f).view(np.uint8) == getattr(b, f).view(np.uint8)).all()


def test_recenter_rejects_an_emitter_past_the_last(engine):
    import ctypes as C

    import torch
    from evolution_simulator_gpu_b200 import api
    pop = ce.generate(SPEC, 2)
    opt = cma.CmaEmitters(pop)
    before = [opt.state(e) for e in range(2)]
    b = refine.take(pop, np.array([0]))

    def up(arr):
        return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(opt.device)

    dn, db, dm, dg = up(b.nodes), up(b.bones), up(b.muscles), up(b.genomes)
    which = torch.tensor([7], dtype=torch.int32, device=opt.device)
    rej = torch.zeros(1, dtype=torch.int32, device=opt.device)
    pc = api.PopulationC(dn.data_ptr(), db.data_ptr(), dm.data_ptr(), dg.data_ptr(), 1, None)
    assert api.lib().ce_cma_recenter(C.byref(opt._c), C.byref(pc), which.data_ptr(), 1, rej.data_ptr(),
                                     opt._stream.cuda_stream) == ce.CE_OK
    assert int(rej.cpu()[0]) == 1
    for e in range(2):
        for x, y in zip(opt.state(e), before[e]):
            assert (np.asarray(x) == np.asarray(y)).all()
    with pytest.raises(ValueError):
        opt.recenter([5], b)
