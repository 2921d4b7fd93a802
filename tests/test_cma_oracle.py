"""The float32 restatement of the reference's CMA-ES emitters
(oracle/cma_ref.py), checked against the reference's own tests of them
(src/qd.rs:3033-3110) and of its random streams (src/evolution.rs:
3124-3160), and the host side of ce_cma_*: offsets and argument checks. No
GPU call is made."""
import ctypes as C

import numpy as np

import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import api, cma, refine
from oracle import cma_ref as R

SPEC = ce.GenSpecPy(seed=11, min_nodes=3, max_nodes=8, max_muscles=12)


def body(pop, i):
    g = pop.genomes[i]
    return (pop.nodes[g["node_start"]:g["node_start"] + g["node_count"]].copy(),
            pop.bones[g["bone_start"]:g["bone_start"] + g["bone_count"]].copy(),
            pop.muscles[g["muscle_start"]:g["muscle_start"] + g["muscle_count"]].copy())


def start_state(template):
    mean = R.parameters(*template)
    D = len(mean)
    return mean, np.ones(D, np.float32), np.zeros(D, np.float32), np.zeros(D, np.float32), np.float32(0.5)


def test_phase_dimensions_follow_bones_and_eight_value_muscles():
    # cma_phase_dimensions_follow_bones_and_eight_value_muscles (src/qd.rs:3053-3068).
    n, b = 4, 3
    start = 4 * n + 5 * b + 1
    assert not R.wraps(n, b, start - 1) and not R.wraps(n, b, start)
    assert R.wraps(n, b, start + 4) and R.wraps(n, b, start + 7) and R.wraps(n, b, start + 12)
    assert not R.wraps(n, b, start + 13)


def test_parameters_round_trip_through_a_creature():
    # cma_parameters_round_trip_through_a_creature (src/qd.rs:3097-3109):
    # apply(parameters) gives back the parameters. ln and exp are numpy's
    # here, so the log coordinates agree to an ulp; the rest exactly.
    pop = ce.generate(SPEC, 20)
    for i in range(len(pop)):
        t = body(pop, i)
        p = R.parameters(*t)
        back = R.parameters(*R.apply(*t, p, friction=(SPEC.friction_lo, SPEC.friction_hi)))
        n, b, m = len(t[0]), len(t[1]), len(t[2])
        logs = np.zeros(len(p), bool)
        logs[4 * n + 5 * b] = True
        logs[4 * n + 5 * b + 1 + 6::8] = True
        assert (back[~logs] == p[~logs]).all()
        np.testing.assert_allclose(back[logs], p[logs], rtol=2e-7, atol=2e-7)
        assert len(p) == cma.dims(pop.genomes[i:i + 1])[0]


def test_optimizer_moves_toward_its_faster_samples():
    # optimizer_moves_toward_its_faster_samples (src/qd.rs:3071-3094).
    t = body(ce.generate(SPEC, 1), 0)
    samples = []
    for shift in (0.05, -0.05, 0.04, -0.04):
        n = t[0].copy()
        n["x"] += np.float32(shift)
        samples.append((n, t[1], t[2]))
    state = start_state(t)
    fitness = np.array([4.0, 1.0, 3.0, 2.0], np.float32)
    out = R.tell(state, t, samples, fitness)
    assert out[0][0] > state[0][0]


def explore_state(template):
    mean = R.explore_parameters(*template)
    D = len(mean)
    return mean, np.ones(D, np.float32), np.zeros(D, np.float32), np.zeros(D, np.float32), np.float32(0.12)


@pytest.mark.parametrize("exploring", [True, False])
def test_feedback_ignores_candidates_with_changed_topology(exploring):
    # cma_feedback_ignores_candidates_with_changed_topology (src/qd.rs:3033-3050):
    # a CMA-ME emitter there; both modes here.
    t = body(ce.generate(SPEC, 1), 0)
    m = np.concatenate([t[2], t[2][:1]])
    state = explore_state(t) if exploring else start_state(t)
    out = R.tell(state, t, [(t[0], t[1], m)] * 2, np.array([2.0, 1.0], np.float32), exploring)
    assert (out[0] == state[0]).all() and out[4] == state[4]
    rewired = t[2].copy()
    rewired["bone_b"][0] = (rewired["bone_b"][0] + 1) % len(t[1])
    out = R.tell(state, t, [(t[0], t[1], rewired)] * 2, np.array([2.0, 1.0], np.float32), exploring)
    assert (out[0] == state[0]).all()
    # The same samples with the template's plan do move it.
    out = R.tell(state, t, [t] * 2, np.array([2.0, 1.0], np.float32), exploring)
    assert out[4] != state[4]


def test_phase_dimensions_of_a_cma_me_emitter():
    # is_phase_dimension (src/qd.rs:2480-2482): muscle field 5 after 4 a
    # node and 1 a bone.
    n, b = 4, 3
    start = 4 * n + b
    assert [d for d in range(start + 24) if R.phase_dimension(d, start)] == [start + 5, start + 13, start + 21]


def test_cma_me_emitter_moves_toward_its_better_samples():
    t = body(ce.generate(SPEC, 1), 0)
    state = explore_state(t)
    samples = []
    for shift in (0.05, -0.05, 0.04, -0.04):
        n = t[0].copy()
        n["x"] += np.float32(shift)
        samples.append((n, t[1], t[2]))
    out = R.tell(state, t, samples, np.array([4.0, 1.0, 3.0, 2.0], np.float32), True)
    assert out[0][0] > state[0][0]
    assert 0.005 <= out[4] <= 0.35 and (out[1] >= 0.0025).all() and (out[1] <= 4.0).all()


def test_twelve_uniform_gaussians_have_unit_variance():
    # twelve_uniform_gaussians_have_unit_variance (src/evolution.rs:3124-3139),
    # on 100k draws of each kind: the cursor's and a gene sub-stream's.
    key = R.stream_key(1, 2, 3, 4)
    genes = R.keyed(key, R.CURSOR, 0)
    cursor = [R.twelve_uniforms([R.keyed(key, R.CURSOR, 1 + 3 * i + k) for k in range(3)]) for i in range(100_000)]
    gene = [R.gene_gaussian(genes, g) for g in range(100_000)]
    for draw in (np.array(cursor, np.float64), np.array(gene, np.float64)):
        assert abs(draw.mean()) < 0.01 and abs(draw.var() - 1.0) < 0.02 and (np.abs(draw) <= 6.0).all()


def test_gene_noise_does_not_depend_on_other_draws():
    # gene_noise_does_not_depend_on_other_draws (src/evolution.rs:3141-3160),
    # its stream half: a gene's noise is keyed by its index.
    a = R.keyed(R.stream_key(5, 1, 2, 3), R.CURSOR, 0)
    forward = [R.gene_gaussian(a, g) for g in range(64)]
    backward = [R.gene_gaussian(a, g) for g in reversed(range(64))]
    assert forward == backward[::-1]
    other = R.keyed(R.stream_key(5, 1, 2, 4), R.CURSOR, 0)
    assert any(R.gene_gaussian(other, g) != forward[g] for g in range(64))


def test_failed_and_non_finite_samples_are_dropped():
    t = body(ce.generate(SPEC, 1), 0)
    state = start_state(t)
    same = [t] * 3
    out = R.tell(state, t, same, np.array([R.FAILED, np.nan, 1.0], np.float32))
    assert (out[0] == state[0]).all() and out[4] == state[4]  # one sample left: no update
    out = R.tell(state, t, same, np.array([R.FAILED, 2.0, 1.0], np.float32))
    assert out[4] != state[4]


def test_step_size_shrinks_when_most_samples_are_slow():
    # The fragile-gait rule (src/qd.rs:2468-2473): median below a quarter of
    # the best multiplies sigma by 0.6 after step-length control.
    t = body(ce.generate(SPEC, 1), 0)
    state = start_state(t)
    rng = np.random.default_rng(0)
    samples = []
    for _ in range(8):
        n = t[0].copy()
        n["x"] += rng.normal(0, 0.01, len(n)).astype(np.float32)
        samples.append((n, t[1], t[2]))
    fast = R.tell(state, t, samples, np.array([8, 7, 6, 5, 4, 3, 2, 1], np.float32))
    slow = R.tell(state, t, samples, np.array([8, 7, 6, 1, 1, 1, 1, 1], np.float32))
    assert slow[4] == max(np.float32(fast[4] * np.float32(0.6)), np.float32(0.01))
    for a, b in zip(fast[:4], slow[:4]):
        assert (a == b).all()


def test_offsets_and_argument_checks_without_a_gpu():
    pop = ce.generate(SPEC, 5)
    L = ce.lib()
    off = np.zeros(6, np.uint64)
    assert L.ce_cma_offsets(api._ptr(pop.genomes), None, 5, api._ptr(off)) == ce.CE_OK
    d = cma.dims(pop.genomes)
    assert (off == np.concatenate([[0], np.cumsum(d)])).all()
    mode = np.array([1, 0, 1, 1, 0], np.uint8)
    assert L.ce_cma_offsets(api._ptr(pop.genomes), api._ptr(mode), 5, api._ptr(off)) == ce.CE_OK
    d = cma.dims(pop.genomes, mode)
    assert (off == np.concatenate([[0], np.cumsum(d)])).all()
    for i in range(5):
        t = body(pop, i)
        assert d[i] == len(R.explore_parameters(*t) if mode[i] else R.parameters(*t))
    bad = pop.genomes.copy()
    bad["bone_count"][2] += 1
    assert L.ce_cma_offsets(api._ptr(bad), None, 5, api._ptr(off)) == ce.CE_ERR_INVALID
    assert b"template 2" in L.ce_last_error()
    assert L.ce_cma_init(None, None) == ce.CE_ERR_INVALID
    empty = api.CmaC()
    assert L.ce_cma_init(C.byref(empty), None) == ce.CE_ERR_INVALID
    draw = cma.CmaEmitters.draw()
    assert L.ce_cma_ask(C.byref(empty), C.byref(draw), 0, 1, None, None, None, None, None, None, 0, None) \
        == ce.CE_ERR_INVALID
    assert L.ce_cma_tell(C.byref(empty), None, None, 0, 1, None) == ce.CE_ERR_INVALID


def test_dims_match_the_parameter_vectors():
    pop = ce.generate(SPEC, 30)
    d = cma.dims(pop.genomes)
    for i in range(len(pop)):
        assert d[i] == len(R.parameters(*body(pop, i)))
    assert refine.take(pop, np.arange(3)).genomes["node_start"][0] == 0


def test_device_entry_points_check_their_arguments_without_a_gpu():
    # Each check returns before any CUDA call, so fake (never dereferenced)
    # device addresses stand in for real ones.
    L = ce.lib()
    fake = 4096
    pc = api.PopulationC(fake, fake, fake, fake, 4, None)
    c = api.CmaC(pc, None, fake, fake, fake, fake, fake, fake)
    # More than 4096 samples an emitter in one tell.
    assert L.ce_cma_tell(C.byref(c), C.byref(pc), fake, 0, 4 * 4096 + 1, None) == ce.CE_ERR_INVALID
    assert b"4096" in L.ce_last_error()
    # An empty diameter or friction range.
    bad = cma.CmaEmitters.draw(size=(0.12, 0.06))
    assert L.ce_cma_ask(C.byref(c), C.byref(bad), 0, 8, fake, fake, fake, None, fake, None, 0, None) \
        == ce.CE_ERR_INVALID
    bad = cma.CmaEmitters.draw(friction=(1.0, 0.5))
    assert L.ce_cma_ask(C.byref(c), C.byref(bad), 0, 8, fake, fake, fake, None, fake, None, 0, None) \
        == ce.CE_ERR_INVALID
    # Values asked for with no stride.
    ok = cma.CmaEmitters.draw()
    assert L.ce_cma_ask(C.byref(c), C.byref(ok), 0, 8, fake, fake, fake, None, fake, fake, 0, None) \
        == ce.CE_ERR_INVALID
    # Recentering needs its bodies and emitter list.
    assert L.ce_cma_recenter(C.byref(c), None, fake, 1, None, None) == ce.CE_ERR_INVALID
    assert L.ce_cma_recenter(C.byref(c), C.byref(pc), None, 1, None, None) == ce.CE_ERR_INVALID
    # The audit's scratch must hold ce_audit_scratch_bytes(count).
    need = L.ce_audit_scratch_bytes(1000)
    assert need >= 1000 * 4
    assert L.ce_audit_device(fake, fake, fake, fake, 1000, fake, need - 1, fake, None, 0, None) == ce.CE_ERR_INVALID
    assert b"scratch" in L.ce_last_error()
    assert L.ce_audit_device(None, fake, fake, fake, 1000, fake, need, fake, None, 0, None) == ce.CE_ERR_INVALID


def test_a_second_restatement_of_the_streams_agrees():
    # The breeding streams again, vectorised in numpy's wrapping uint64:
    # stream keys, the genes sub-stream and its Gaussians, for 2,000 slots x
    # 64 genes, equal to the restatement's integers and floats.
    u = np.uint64

    def fin(z):
        z = (z ^ (z >> u(30))) * u(0xbf58476d1ce4e5b9)
        z = (z ^ (z >> u(27))) * u(0x94d049bb133111eb)
        return z ^ (z >> u(31))

    def key_of(seed, gen, rnd, slots):
        with np.errstate(over="ignore"):
            k = fin(np.full(len(slots), u(seed), u) + u(0x632be59bd9b4e019))
            for w in (np.full(len(slots), u(gen), u), np.full(len(slots), u(rnd), u), slots.astype(u)):
                k = fin(k ^ (w * u(0xd1342543de82ef95)))
        return k

    def keyed_v(key, gene, draw):
        with np.errstate(over="ignore"):
            return fin(key + ((u(gene) << u(32)) | u(draw)) * u(0x9e3779b97f4a7c15))

    slots = np.arange(2000, dtype=np.int64)
    keys = key_of(7, 3, 2, slots)
    for g in (0, 999, 1999):
        assert int(keys[g]) == R.stream_key(7, 3, 2, g)
    genes = keyed_v(keys, 0xffffffff, 0)
    total = np.zeros((2000, 64), np.int64)
    for d in range(64):
        for k in range(3):
            w = keyed_v(genes, d, k)
            total[:, d] += ((w & u(0xffff)) + ((w >> u(16)) & u(0xffff)) + ((w >> u(32)) & u(0xffff)) +
                            (w >> u(48))).astype(np.int64)
    gauss = (total - 6 * 65535).astype(np.float32) * (np.float32(1.0) / np.float32(65535.0))
    for g in (0, 1, 500, 1999):
        want = [R.gene_gaussian(R.keyed(R.stream_key(7, 3, 2, g), R.CURSOR, 0), d) for d in range(64)]
        assert (gauss[g] == np.array(want, np.float32)).all()
    assert abs(gauss.mean()) < 0.01 and abs(gauss.std() - 1.0) < 0.01
