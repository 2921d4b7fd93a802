"""The physics checks of the reference's own GPU tests, re-expressed against
this engine (tests/cuda_physics.rs and tests/cuda_effects.rs in the
reference), on seeded synthetic bodies:

* a muscle frozen at its start length scores like one without stiffness
  (cuda_physics.rs:69-89);
* three nodes on one point joined by bones shorter than a node is wide
  score a finite distance (:93-130);
* on rough ground with a slope no node sinks more than 2 cm below its floor
  (:236-266);
* joints narrowed to 0.3 rad either way stay within 0.75 rad of their start
  angle until the fall (:279-341), and joints with the widest ranges never
  turn through a half turn (:343-377);
* bodies without muscle drive neither travel (:379-400) nor rise (:402-441);
* every world effect changes some body's distance, and no trial fails
  (cuda_effects.rs:21-168), with the reference's stored walker
  (tests/fixtures/warp_walker.json, converted by
  tests/golden/make_fixtures.py), whose muscles have touch sensors; its
  results also equal the reference kernel's to the bit in the calm world and
  with every effect on.
"""
from pathlib import Path

import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import api
from evolution_simulator_gpu_b200.configs import WORKLOADS
from oracle.ref import RefKernel

pytestmark = pytest.mark.gpu

FIXTURES = Path(__file__).resolve().parent / "golden" / "fixtures"
JOINT_LIMIT = np.float32(120.0 * np.pi / 180.0)


def population(creatures):
    """A population of (nodes, bones, muscles, id) tuples."""
    genomes = np.zeros(len(creatures), api.GENOME_DTYPE)
    an = ab = am = 0
    for k, (n, b, m, cid) in enumerate(creatures):
        genomes[k] = (an, len(n), ab, len(b), am, len(m), cid, 0, 0)
        an, ab, am = an + len(n), ab + len(b), am + len(m)
    return ce.Population(np.concatenate([c[0] for c in creatures]), np.concatenate([c[1] for c in creatures]),
                         np.concatenate([c[2] for c in creatures]), genomes)


def small(n):
    return ce.generate(WORKLOADS["small"].spec, n)


def target_at_start(m):
    """physics::target(muscle, 0) (src/physics.rs:298-306), in float32."""
    f = np.float32
    phase = np.float32(np.modf(f(0.0) / m["period"] + m["phase"])[0])
    if phase < m["duty"]:
        wave = f(0.5) + f(0.5) * f(np.cos(f(np.pi) * phase / m["duty"]))
    else:
        wave = f(0.5) - f(0.5) * f(np.cos(f(np.pi) * (phase - m["duty"]) / (f(1.0) - m["duty"])))
    return f(m["short"] + (m["long"] - m["short"]) * wave)


def test_frozen_muscles_behave_like_unpowered_muscles(engine):
    world = ce.make_world(duration=1.0)
    pop = small(32)
    for m in pop.muscles:
        t = target_at_start(m)
        m["short"] = t
        m["long"] = t
    frozen = ce.evaluate(engine, pop, world)
    pop.muscles["stiffness"] = 0.0
    unpowered = ce.evaluate(engine, pop, world)
    assert np.isfinite(frozen["fitness"]).all()
    worst = float(np.abs(frozen["fitness"] - unpowered["fitness"]).max())
    assert worst < 1e-5, f"frozen and unpowered muscles differ by {worst} m"


def test_overlapping_nodes_remain_finite(engine):
    nodes = np.zeros(3, api.NODE_DTYPE)
    nodes["diameter"], nodes["friction"] = 0.08, 0.5
    bones = np.zeros(2, api.BONE_DTYPE)
    bones[0] = (0, 1, 0.03, -JOINT_LIMIT, JOINT_LIMIT, 0.0, 0.5)
    bones[1] = (1, 2, 0.03, -JOINT_LIMIT, JOINT_LIMIT, 0.0, 0.5)
    muscles = np.zeros(1, api.MUSCLE_DTYPE)
    muscles[0] = (0, 1, 0.5, 0.5, 0.1, 0.2, 1.0, 0.0, 0.5, 80.0, 255, 0.0, 0.0)
    res = ce.evaluate(engine, population([(nodes, bones, muscles, 1)]), ce.make_world(duration=1.0))
    assert np.isfinite(res["fitness"]).all() and res["fitness"][0] > -1e19


def _radii_masses(wave, c):
    lf = wave.lanes.view(np.float32)
    n, ro = int(wave.heads[c, 0] & 255), int(wave.heads[c, 3])
    return (np.array([lf[ro + 6 * i + 1] for i in range(n)]), np.array([lf[ro + 6 * i] for i in range(n)]))


def test_nodes_stay_on_top_of_rough_ground(engine):
    world = ce.make_world(duration=3.0, terrain=3, slope=0.15)
    wave = ce.pack(small(16), world)
    frames, _ = engine.record(wave, world)
    settle = ce.settle_frames(world)
    worst = np.inf
    for c in range(len(wave)):
        radius, _ = _radii_masses(wave, c)
        n = len(radius)
        xy = frames[c, settle + 1:, :n]
        for i in range(n):
            for x, y in xy[:, i]:
                h, s = api.ground(float(x), 0.15, 0.15)
                floor = h + radius[i] * np.sqrt(1.0 + s * s)
                worst = min(worst, y - floor)
    assert worst >= -0.02, f"a node sank {-worst} m below its floor"


def _joints(wave, c):
    """(pivot, reference, child) of each joint of packed creature c: the
    pivot (hub) of bone j, the far end of its parent bone, and node j + 1."""
    lanes = wave.lanes
    n, ro = int(wave.heads[c, 0] & 255), int(wave.heads[c, 3])
    bone0 = ro + n * api.NODE_WORDS
    out = []
    for j in range(1, n - 1):
        q = bone0 + j * api.BONE_WORDS
        pivot, parent = int(lanes[q]), int(lanes[q + 2])
        if parent == 0xFFFFFFFF:
            continue
        parent_pivot = int(lanes[bone0 + parent * api.BONE_WORDS])
        far = parent + 1 if parent_pivot == pivot else parent_pivot
        out.append((pivot, far, j + 1))
    return out


def _angle(p, pivot, ref, child):
    u = p[..., ref, :] - p[..., pivot, :]
    v = p[..., child, :] - p[..., pivot, :]
    return np.arctan2(u[..., 0] * v[..., 1] - u[..., 1] * v[..., 0], u[..., 0] * v[..., 0] + u[..., 1] * v[..., 1])


def test_joints_stay_within_their_range(engine):
    world = ce.make_world(duration=10.0)
    pop = small(64)
    pop.bones["min_angle"], pop.bones["max_angle"] = -0.3, 0.3
    wave = ce.pack(pop, world)
    frames, res = engine.record(wave, world)
    settle = ce.settle_frames(world)
    worst = 0.0
    for c in range(len(wave)):
        end = frames.shape[1]
        if res["fall_time"][c] > 0:
            end = min(end, settle + int(np.round(res["fall_time"][c] * 60)) + 1)
        for pivot, ref, child in _joints(wave, c):
            rest = _angle(frames[c, 0], pivot, ref, child)
            turn = _angle(frames[c, :end], pivot, ref, child) - rest
            off = np.mod(turn + np.pi, 2 * np.pi) - np.pi
            worst = max(worst, float(np.abs(off).max()) - 0.3)
    assert worst < 0.75, f"a joint left its range by {worst} rad"


def test_full_joint_ranges_do_not_spin_through_a_half_turn(engine):
    world = ce.make_world(duration=10.0)
    pop = small(64)
    pop.bones["min_angle"], pop.bones["max_angle"] = -JOINT_LIMIT, JOINT_LIMIT
    wave = ce.pack(pop, world)
    frames, _ = engine.record(wave, world)
    widest = 0.0
    for c in range(len(wave)):
        for pivot, ref, child in _joints(wave, c):
            a = _angle(frames[c], pivot, ref, child)
            delta = np.mod(np.diff(a) + np.pi, 2 * np.pi) - np.pi
            widest = max(widest, float(np.abs(np.cumsum(delta)).max()))
    assert widest < np.pi, f"a joint turned {widest} rad"


def _undriven(n):
    pop = small(n)
    pop.muscles["short"] = pop.muscles["long"]
    return pop


def test_a_body_without_drive_does_not_travel(engine):
    res = ce.evaluate(engine, _undriven(32), ce.make_world(duration=5.0))
    worst = float(np.abs(res["fitness"]).max())
    assert worst < 0.5, f"a body drifted {worst} m with no muscle drive"


def test_a_passive_body_never_rises_above_its_start(engine):
    world = ce.make_world(duration=5.0)
    wave = ce.pack(_undriven(32), world)
    frames, _ = engine.record(wave, world)
    settle = ce.settle_frames(world)
    for c in range(len(wave)):
        _, mass = _radii_masses(wave, c)
        n = len(mass)
        height = (frames[c, settle + 1:, :n, 1] * mass[None, :]).sum(axis=1) / mass.sum()
        assert height.max() <= height[0] + 0.02, (c, float(height[0]), float(height.max()))


def _with_walkers(n, extra=()):
    d = np.load(FIXTURES / "warp_walker.npz")
    walker = (d["nodes"], d["bones"], d["muscles"])
    assert (walker[2]["sensor"] != 255).any(), "the stored walker's muscles have touch sensors"
    pop = small(n)
    mine = [pop.creature(i)[:3] + (int(pop.genomes["id"][i]),) for i in range(n)]
    return population(mine + [walker + (k,) for k in range(8)] + list(extra))


def _over_the_pit_edge(reach, cid):
    """A three-node body with no drive, two long bones from its middle
    node: one 1.95 m forward and one `reach` m back. Centred on its centre
    of mass, the back node starts about 1.77 m behind the start, over the
    ramp into the first pit of `gaps` 0.5 (pits 0.5 m wide every 4 m,
    centred at x = -2 and 2): with gaps its back bone droops into the pit
    and the body's centre moves back by several centimetres; without, it
    lies still."""
    nodes = np.zeros(3, api.NODE_DTYPE)
    nodes[0] = (0.0, 0.0, 0.08, 0.5)
    nodes[1] = (1.95, 0.0, 0.08, 0.5)
    nodes[2] = (-reach, 0.0, 0.08, 0.5)
    bones = np.zeros(2, api.BONE_DTYPE)
    bones[0] = (0, 1, 1.95, -JOINT_LIMIT, JOINT_LIMIT, 0.0, 0.5)
    bones[1] = (0, 2, reach, -JOINT_LIMIT, JOINT_LIMIT, 0.0, 0.5)
    muscles = np.zeros(1, api.MUSCLE_DTYPE)
    muscles[0] = (0, 1, 0.5, 0.5, 1.0, 1.0, 1.0, 0.0, 0.5, 0.0, 255, 0.0, 0.0)
    return nodes, bones, muscles, cid


EFFECTS = {"terrain": dict(terrain=2), "slope": dict(slope=0.1), "mud": dict(mud=0.06), "water": dict(water=0.35),
           "gaps": dict(gaps=0.5), "hurdles": dict(hurdles=0.1), "ice": dict(patches=0.95),
           "quake": dict(quake=0.05), "wind": dict(wind=2.0), "air": dict(air_retention=0.98),
           "gravity": dict(gravity=5.0), "grip": dict(ground_friction=0.5), "heat": dict(muscle_energy=0.3)}


def test_the_kernel_feels_every_effect(engine):
    """As the reference's test, 8 s trials from a calm world. The reference
    counts on its stored walkers getting over 5 m, which its own notes say
    they no longer do, and an effect placed away from the start (the pits of
    `gaps` begin 1.75 m out, the ice patches 0.9 m out) is not reached by
    bodies that stay within half a metre. So two undriven bodies that start
    with a node over a pit's edge join the population, and an effect that
    changes nothing from the calm world is checked again against a steep
    slope (0.6), down which the bodies slide across the track."""
    pop = _with_walkers(256, [_over_the_pit_edge(1.35, 100), _over_the_pit_edge(1.4, 101)])
    bases = [{}, dict(slope=0.6)]
    base_res = {}
    for k, base in enumerate(bases):
        base_res[k] = ce.evaluate(engine, pop, ce.make_world(duration=8.0, **base))
    assert (base_res[0]["fitness"] > -1e19).all(), "a calm trial failed"
    for name, kw in EFFECTS.items():
        for k, base in enumerate(bases):
            res = ce.evaluate(engine, pop, ce.make_world(duration=8.0, **dict(base, **kw)))
            assert (res["fitness"] > -1e19).all(), f"{name}: a trial failed"
            change = float(np.abs(res["fitness"] - base_res[k]["fitness"]).max())
            if change > 0.005:
                break
        assert change > 0.005, f"{name} changes no body's distance, from calm or on a slope"


@pytest.mark.parametrize("every_effect", [False, True])
def test_walkers_with_touch_sensors_match_the_reference_kernel(engine, every_effect):
    kw = dict(terrain=2, gravity=14.7, air_retention=0.985, ground_friction=1.0, slope=0.03, wind=-1.0, mud=0.05,
              brambles=3.0, water=0.12, patches=0.5, gaps=0.35, hurdles=0.08, quake=0.05) if every_effect else {}
    world = ce.make_world(duration=8.0, **kw)
    pop = _with_walkers(256)
    wave = ce.pack(pop, world)
    mine, _ = engine.run(wave, world)
    ref, _ = RefKernel(ce.world_flags(world)).run(wave, ce.make_params(world))
    assert (mine.view(np.uint32) == ref.view(np.uint32)).all()
