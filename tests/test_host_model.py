"""The host side of the path on the CPU: the ground functions, world flags,
launch parameters, packing, start pose, metrics and niche cells.

The ground tests restate the reference's own CPU tests of these functions
(src/physics.rs:727-919) on the engine's host restatement; the packing tests
follow src/kernel.rs:595-656 and the start-pose rules of
src/physics2.rs:371-399.
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import api
from evolution_simulator_gpu_b200.configs import WORKLOADS, effects_world_kw


def terrain(x, amp):
    return api.ground(x, amp)


def test_terrain_slope_matches_its_height():
    for i in range(200):
        x = np.float32(i * 0.037 - 3.0)
        _, slope = terrain(x, 0.05)
        h = 1e-3
        numeric = (terrain(x + h, 0.05)[0] - terrain(x - h, 0.05)[0]) / (2 * h)
        assert abs(slope - numeric) < 1e-2
        assert 0.0 <= terrain(x, 0.05)[0] <= 0.05 + 1e-6
    assert terrain(0.7, 0.0) == (0.0, 0.0)
    tilt = 0.15
    for i in range(200):
        x = i * 0.037 - 3.0
        height, slope = api.ground(x, 0.05, tilt)
        h = 1e-3
        numeric = (api.ground(x + h, 0.05, tilt)[0] - api.ground(x - h, 0.05, tilt)[0]) / (2 * h)
        assert abs(slope - numeric) < 1e-2
        assert abs(height - (terrain(x, 0.05)[0] + tilt * x)) < 1e-6
    assert api.ground(0.7, 0.0, 0.0) == (0.0, 0.0)
    assert api.ground(2.0, 0.0, 0.25) == (0.5, 0.25)


def test_gaps_carve_bounded_pits_every_spacing():
    width = 1.0
    spacing = 2.0 + 4.0 * width
    gaps = lambda x, w=width: api.ground(x, width=w)  # noqa: E731
    assert gaps(0.0) == (0.0, 0.0)
    assert gaps(0.6)[0] > -1e-6
    assert gaps(0.5 * spacing) == (-2.0, 0.0)
    for x in [0.01, 0.5, 1.4, 7.3, 15.9]:
        assert -2.0 - 1e-6 <= gaps(x)[0] <= 0.0
    prev = gaps(-spacing)[0]
    x = -spacing + 0.001
    while x <= 3 * spacing:
        cur = gaps(x)[0]
        assert abs(cur - prev) < 0.5
        prev = cur
        x += 0.001
    assert gaps(0.5, 0.0) == (0.0, 0.0)


def test_ground_slope_matches_its_height_with_pits():
    for i in range(400):
        x = i * 0.037 - 4.0
        _, slope = api.ground(x, 0.05, 0.15, 1.0)
        h = 1e-3
        numeric = (api.ground(x + h, 0.05, 0.15, 1.0)[0] - api.ground(x - h, 0.05, 0.15, 1.0)[0]) / (2 * h)
        assert abs(slope - numeric) < 1e-2


def test_hurdles_rise_and_stay_continuous():
    height = 0.3
    hur = lambda x, hh=height: api.ground(x, hurdle=hh)  # noqa: E731
    assert hur(0.0) == (0.0, 0.0)
    assert hur(1.5, 0.0) == (0.0, 0.0)
    assert hur(1.5) == (pytest.approx(height), 0.0)
    prev = hur(-3.0)[0]
    x = -3.0 + 0.0005
    while x <= 6.0:
        cur = hur(x)[0]
        assert abs(cur - prev) < 0.5
        assert 0.0 <= cur <= height + 1e-6
        prev = cur
        x += 0.0005
    for x in [0.2, 0.8, 1.5, 2.6]:
        lo, lo_s = hur(x, 0.1)
        hi, hi_s = hur(x, 0.2)
        assert abs(hi - 2 * lo) < 1e-6 and abs(hi_s - 2 * lo_s) < 1e-6


def test_ground_slope_matches_its_height_with_hurdles():
    for i in range(400):
        x = i * 0.0371 - 4.0
        _, slope = api.ground(x, 0.03, 0.05, 0.0, 0.25, 0.37)
        h = 1e-3
        numeric = (api.ground(x + h, 0.03, 0.05, 0.0, 0.25, 0.37)[0] -
                   api.ground(x - h, 0.03, 0.05, 0.0, 0.25, 0.37)[0]) / (2 * h)
        assert abs(slope - numeric) < 1e-2


def test_quake_streams_are_deterministic_and_spread():
    assert api.quake_hash(47300) == api.quake_hash(47300)
    phases, scales = set(), set()
    for i in range(1, 1001):
        h = api.quake_hash(i)
        phase = np.float32(h & 0xFFFF) * np.float32(1.0 / 65536.0)
        scale = np.float32(0.6) + np.float32((h >> 16) & 0xFFFF) * np.float32(0.8 / 65536.0)
        assert 0.0 <= phase < 1.0 and 0.6 <= scale <= 1.4
        phases.add(float(phase))
        scales.add(float(scale))
    assert len(phases) > 900 and len(scales) > 900


def test_world_flags_name_the_effects():
    assert ce.world_flags(ce.make_world()) == 0x001
    assert ce.world_flags(ce.make_world(**effects_world_kw())) == 0x797
    quake = ce.make_world(**dict(effects_world_kw(), terrain=1, quake=0.05))
    assert ce.world_flags(quake) == 0x7B7
    # Without ground the ground's effects are off; water and wind stay.
    w = ce.make_world(ground=0, slope=0.1, mud=0.05, water=0.3, wind=-1.0, hurdles=0.2)
    assert ce.world_flags(w) == (1 << 7) | (1 << 9)


def test_launch_parameters():
    w = ce.make_world(air_retention=0.985, screen=(5.0, 0.3))
    p = ce.make_params(w, 7, 11, 3)
    assert (p.base, p.count, p.stride, p.steps) == (7, 11, 3, 1200)
    assert p.screen_step == 299
    assert np.float32(p.air_sub) == np.float32(np.float32(0.985) ** np.float32(1.0 / 16.0))
    assert p.r1.bias == -np.inf and p.r2.bias == -np.inf
    assert ce.make_params(ce.make_world()).screen_step == 0xFFFFFFFF
    assert ce.make_params(ce.make_world(rate=120, duration=2.0)).steps == 240


def test_a_population_packs_every_creature_once_in_order():
    w = ce.make_world()
    pop = ce.generate(WORKLOADS["game"].spec, 3000)
    wave = ce.pack(pop, w)
    assert sorted(wave.slots.tolist()) == list(range(3000))
    key = [(int(h[1]), int(h[0] & 255), int(s)) for h, s in zip(wave.heads, wave.slots)]
    assert key == sorted(key)
    # Record offsets are contiguous and sized by each body.
    rl = ml = 0
    for h in wave.heads:
        n, m = int(h[0] & 255), int(h[1])
        assert int(h[3]) == rl and int(h[4]) == ml
        rl += n * 6 + (n - 1) * 6
        ml += m * 20
    assert rl == len(wave.lanes) and ml == len(wave.muscles)


def test_start_pose_sits_on_the_ground_over_the_origin():
    w = ce.make_world()
    pop = ce.generate(WORKLOADS["game"].spec, 300)
    wave = ce.pack(pop, w)
    f = wave.lanes.view(np.float32)
    for h in wave.heads:
        n = int(h[0] & 255)
        rec = f[int(h[3]):int(h[3]) + 6 * n].reshape(n, 6)
        mass, radius, x, y = rec[:, 0], rec[:, 1], rec[:, 3], rec[:, 4]
        total = np.float32(0)
        for m in mass:
            total = np.float32(total + m)
        assert np.uint32(h[5]) == total.view(np.uint32)
        assert abs(float(np.dot(mass, x) / mass.sum())) < 1e-5
        assert abs(float((y - radius).min())) < 1e-6
        assert y[0] >= y.max() - 1e-6, "the head starts highest"


def test_feet_end_legs_of_two_bones():
    # Head 0 - neck to 1; 1 -> 2 -> 3 (a leg of two bones); 1 -> 4 (one bone).
    nodes = np.zeros(5, api.NODE_DTYPE)
    nodes["x"] = [0.0, 0.0, 0.1, 0.2, -0.1]
    nodes["y"] = [1.0, 0.8, 0.5, 0.2, 0.6]
    nodes["diameter"] = 0.1
    nodes["friction"] = 0.5
    bones = np.zeros(4, api.BONE_DTYPE)
    for j, (a, b) in enumerate([(0, 1), (1, 2), (2, 3), (1, 4)]):
        bones[j] = (a, b, np.hypot(*(np.array([nodes["x"][b] - nodes["x"][a], nodes["y"][b] - nodes["y"][a]]))),
                    -2.0, 2.0, 0.0, 0.5)
    genomes = np.zeros(1, api.GENOME_DTYPE)
    genomes[0] = (0, 5, 0, 4, 0, 0, 1, 0, 0)
    pop = api.Population(nodes, bones, np.zeros(0, api.MUSCLE_DTYPE), genomes, np.zeros(0, np.float32))
    wave = ce.pack(pop, ce.make_world())
    feet = wave.lanes[:30].reshape(5, 6)[:, 5]
    assert feet.tolist() == [0, 0, 0, 1, 0]


def test_period_half_rounds_to_nearest_even():
    pop = ce.generate(WORKLOADS["small"].spec, 500)
    wave = ce.pack(pop, ce.make_world())
    for h, s in zip(wave.heads, wave.slots):
        g = pop.genomes[s]
        period = pop.muscles["period"][g["muscle_start"]] if g["muscle_count"] else np.float32(0)
        assert int(h[7]) & 0xFFFF == int(np.float16(period).view(np.uint16))
    pop.muscles["period"][pop.genomes["muscle_start"][0]] = 12.3
    wave = ce.pack(pop, ce.make_world(), [0])
    assert np.uint16(wave.heads[0, 7] & 0xFFFF).view(np.float16) == np.float16(12.296875)


def test_metrics_and_niche_cells_known_answers():
    w = ce.make_world()
    r = np.zeros(2, ce.RESULT_DTYPE)
    # A trial that fell at 2 s: 120 steps of a 4-node body.
    r[0]["fitness"] = 1.5
    r[0]["ground_contact"] = 240.0
    r[0]["vertical_oscillation"] = 0.05
    r[0]["gait_frequency"] = 1.2
    r[0]["height_sum"] = 36.0
    r[0]["fall_time"] = 2.0
    r[0]["lift_lo"] = np.array([0b1011], np.uint32).view(np.float32)[0]
    # A full trial with infinite oscillation (never finished counters).
    r[1]["fitness"] = -0.5
    r[1]["vertical_oscillation"] = np.inf
    r[1]["gait_frequency"] = np.nan
    r[1]["height_sum"] = 1200.0
    m = ce.to_metrics(r, np.array([4, 3]), w)
    assert m[0]["steps"] == 120 and m[1]["steps"] == 1200
    assert m[0]["ground_contact"] == np.float32(0.5)
    assert m[0]["mean_height"] == np.float32(0.3) and m[0]["feet"] == 3
    assert m[1]["vertical_oscillation"] == 0 and m[1]["gait_frequency"] == 0
    assert m[1]["mean_height"] == 1.0
    # Niche bytes by hand: contact 0.5 -> bin 3 of 6; cadence 1.2 Hz -> bin
    # 1 of 8 over 0-6 Hz; height 0.3 m -> log axis ln(2)/ln(8) = 1/3 -> bin 2
    # of 6; 3 feet -> byte 2; shape and size from the start pose.
    nodes = np.zeros(4, api.NODE_DTYPE)
    nodes["x"] = [0.0, 0.3, 0.6, 0.9]
    nodes["y"] = [0.5, 0.0, 0.2, 0.1]
    genomes = np.zeros(1, api.GENOME_DTYPE)
    genomes[0] = (0, 4, 0, 3, 0, 2, 1, 0, 0)
    pop = api.Population(nodes, np.zeros(3, api.BONE_DTYPE), np.zeros(2, api.MUSCLE_DTYPE), genomes)
    cell, niche = ce.niche(pop, 0, m[0], global_layout=True)
    # aspect 0.9/0.5 = 1.8 -> global shape 2 of 4; 4 nodes -> size 0 of 4.
    assert niche.tolist() == [3, 1, 2, 2, 2, 0]
    bins = [6, 8, 4, 6, 5, 4]
    idx = 0
    for a, b in zip(niche.tolist(), bins):
        idx = idx * b + a
    assert cell == idx
    assert ce.niche_cells(pop, m[:1])[0] == cell
    # Island layout: aspect edges 1.2, 2.0 -> shape 1 of 3.
    _, niche_i = ce.niche(pop, 0, m[0], global_layout=False)
    assert niche_i.tolist() == [3, 1, 1, 2, 2, 0]


def test_unsupported_bodies_are_rejected():
    pop = ce.generate(WORKLOADS["small"].spec, 2)
    pop.genomes["bone_count"][0] = 0
    with pytest.raises(ce.EngineError) as err:
        ce.pack(pop, ce.make_world())
    assert err.value.status == ce.CE_ERR_INVALID
