"""The step's contact tallies round exactly as the reference kernel's.

A node counts as touching when its height is at most its floor plus 2 mm
(shaders/creature.cu:1009-1014); `ground_contact` sums those counts over the
trial, so a floor one unit in the last place off changes a count now and
then. The probe creatures hold a test node that cannot move during a
one-step trial (no gravity or wind, no muscles, a mass of 1e30 so the bone
projections leave it in place) at heights swept one unit in the last place at
a time around its floor, on rough sloped ground with hurdles. The highest
height that still counts as touching is the threshold each kernel computes;
the engine's must equal the reference kernel's at every probed x. The second
test runs a large effects-world generation and checks every result to the
bit, where a tally rounding differently shows up as a ground_contact off by
one in a few creatures in 100,000.
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.api import WavePack
from evolution_simulator_gpu_b200.configs import WORKLOADS, effects_world_kw
from oracle.ref import RefKernel

pytestmark = pytest.mark.gpu

EFFECTS = 0x797  # terrain, slope, hurdles, water, ice, wind, thick air
SWEEP = 40
RADIUS = 0.05


def probe_world():
    kw = dict(effects_world_kw(), gravity=0.0, wind=0.0, duration=1.0 / 60.0)
    world = ce.make_world(**kw)
    p = ce.make_params(world)
    p.steps = 1
    return p


def floor_estimate(x: float, p) -> np.float32:
    t0 = x / 1.1
    u0 = t0 - np.floor(t0)
    w0 = u0 * (1 - u0)
    t1 = x / 0.43 + 0.3
    u1 = t1 - np.floor(t1)
    w1 = u1 * (1 - u1)
    h = p.terrain * (10.4 * w0 * w0 + 5.6 * w1 * w1) + p.slope * x
    s = p.terrain * (20.8 * w0 * (1 - 2 * u0) / 1.1 + 11.2 * w1 * (1 - 2 * u1) / 0.43) + p.slope
    r = x - np.floor(x / 3.0) * 3.0
    d = abs(r - 1.5)
    h += p.hurdles * (1.0 if d <= 0.6 else (0.0 if d >= 0.8 else (0.8 - d) / 0.2))
    if 0.6 < d < 0.8:
        s += p.hurdles * ((1.0 if r < 1.5 else -1.0) / 0.2)
    return np.float32(h + RADIUS * np.sqrt(1 + s * s) + 0.002)


def probe_wave(xs, p):
    f32 = np.float32
    cases = []
    for x in xs:
        x = f32(x)
        t = floor_estimate(float(x), p)
        for k in range(-SWEEP, SWEEP + 1):
            y = t
            for _ in range(abs(k)):
                y = np.nextafter(y, f32(np.inf if k > 0 else -np.inf))
            cases.append((x, y))
    n = len(cases)
    lanes = np.zeros(n * 30, np.uint32)
    lf = lanes.view(np.float32)
    heads = np.zeros((n, 8), np.uint32)
    total = f32(1.0) + f32(1.0) + f32(1e30)
    for c, (x, y) in enumerate(cases):
        o = 30 * c
        nodes = [(1.0, 0.05, x, 1.0), (1.0, 0.05, f32(x + 0.3), 0.8), (1e30, RADIUS, x, y)]
        for i, (m, r, px, py) in enumerate(nodes):
            lf[o + 6 * i:o + 6 * i + 5] = [m, r, 0.5, px, py]
        b = o + 18
        lanes[b:b + 6] = [0, f32(np.hypot(0.3, 0.2)).view(np.uint32), 0xFFFFFFFF,
                          f32(-10).view(np.uint32), f32(10).view(np.uint32), 0]
        lanes[b + 6:b + 12] = [1, f32(np.hypot(0.3, 0.8 - float(y))).view(np.uint32), 0,
                               f32(-10).view(np.uint32), f32(10).view(np.uint32), 0]
        heads[c] = [3, 0, 0, o, 0, total.view(np.uint32), (f32(1.0) / total).view(np.uint32), 0]
    wave = WavePack(lanes, np.zeros(4, np.float32), heads, np.arange(n, dtype=np.uint32), np.zeros((n, 4), np.uint32))
    return wave, cases


def thresholds(results, cases):
    touching = (np.ascontiguousarray(results["contact_lo"]).view(np.uint32) >> 2) & 1
    out = {}
    for (x, y), t in zip(cases, touching):
        out.setdefault(float(x), -np.inf)
        if t:
            out[float(x)] = max(out[float(x)], float(y))
    return out


def test_contact_threshold_matches_reference():
    torch = pytest.importorskip("torch")
    p = probe_world()
    xs = list(np.arange(-3.0, 4.6, 0.0637)) + list(np.arange(0.70, 0.90, 0.011)) + list(np.arange(2.10, 2.30, 0.011))
    wave, cases = probe_wave(xs, p)
    ref, _ = RefKernel(EFFECTS).run(wave, p)
    dev = torch.device("cuda", 0)
    with ce.Engine(0) as eng:
        d_l = torch.from_numpy(wave.lanes.view(np.int32)).to(dev)
        d_m = torch.zeros(4, device=dev)
        d_h = torch.from_numpy(wave.heads.view(np.int32).reshape(-1)).to(dev)
        d_r = torch.zeros(len(wave) * 19, device=dev)
        d_c = torch.zeros(16, dtype=torch.int32, device=dev)
        d_s = torch.empty(eng.scratch_bytes(EFFECTS, 60, 3, 0, len(wave)), dtype=torch.uint8, device=dev)
        p.count = len(wave)
        eng.advance_device(d_l.data_ptr(), d_m.data_ptr(), d_h.data_ptr(), d_r.data_ptr(), d_c.data_ptr(),
                           d_s.data_ptr(), p, EFFECTS, 60, 3, 0, torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize(dev)
        mine = d_r.cpu().numpy().view(ce.RESULT_DTYPE)
    t_ref, t_mine = thresholds(ref, cases), thresholds(mine, cases)
    assert all(np.isfinite(v) for v in t_ref.values()), "the sweep must bracket every threshold"
    diff = {x: (t_ref[x], t_mine[x]) for x in t_ref if t_ref[x] != t_mine[x]}
    assert not diff, f"{len(diff)} of {len(t_ref)} thresholds differ: {list(diff.items())[:4]}"


def test_effects_generation_matches_bits_at_scale(engine):
    world = ce.make_world(duration=5.0, **effects_world_kw())
    wave = ce.pack(ce.generate(WORKLOADS["effects"].spec, 200_000), world)
    mine, _ = engine.run(wave, world)
    ref, _ = RefKernel(ce.world_flags(world)).run(wave, ce.make_params(world))
    bad = (mine.view(np.uint32).reshape(len(mine), -1) != ref.view(np.uint32).reshape(len(ref), -1)).any(axis=1)
    assert not bad.any(), f"{int(bad.sum())} creatures differ"
