"""Generates the golden vectors of the creature path from the reference
itself.

Run on a machine with a B200 and the reference kernel built
(oracle/build_ref.py). It packs small seeded populations with the engine's
packer, runs the reference's own kernel (shaders/creature.cu, built for
sm_100a, oracle/_ref) on them and stores the packed inputs, the launch
parameters, the reference's results and, for a few creatures, the reference's
recorded frames, as tests/golden/<name>.npz. The CPU tests check the CPU
oracle and the host packing against these files.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import evolution_simulator_gpu_b200 as ce  # noqa: E402
from evolution_simulator_gpu_b200.configs import WORKLOADS, effects_world_kw  # noqa: E402
from oracle.ref import RefKernel  # noqa: E402

OUT = Path(__file__).resolve().parent
CASES = {
    # name: (workload spec, world overrides, creatures, recorded creatures)
    "calm_small": ("small", dict(duration=2.0), 96, 6),
    "calm_game": ("game", dict(duration=2.0), 96, 4),
    "effects": ("effects", dict(effects_world_kw(), duration=2.0), 96, 4),
    "every_effect": ("effects", dict(terrain=2, gravity=14.7, air_retention=0.985, ground_friction=1.0, slope=0.03,
                                     wind=-1.0, mud=0.05, brambles=3.0, water=0.12, patches=0.5, gaps=0.35,
                                     hurdles=0.08, quake=0.05, duration=2.0), 64, 4),
}


def make(name: str) -> Path:
    wl, kw, n, rec = CASES[name]
    spec = WORKLOADS[wl].spec
    world = ce.make_world(**kw)
    pop = ce.generate(spec, n)
    wave = ce.pack(pop, world)
    params = ce.make_params(world)
    flags = ce.world_flags(world)
    results, _ = RefKernel(flags).run(wave, params)
    frames = []
    per = ce.settle_frames(world) + ce.trial_steps(world) + 1
    recorder = RefKernel(flags, 60, record=True)
    for c in range(rec):
        one = wave.take([c])
        stride = ce.frame_stride(one.max_muscles)
        p = ce.make_params(world, 0, 1, stride)
        fr, _ = recorder.record_one(one, p, per, stride)
        nodes = int(one.heads[0, 0] & 255)
        pos = np.full((per, 32, 2), np.nan, np.float32)
        pos[:, :nodes] = fr[:, :nodes]
        frames.append(pos)
    path = OUT / f"{name}.npz"
    world_fields = {f: getattr(world, f) for f, _ in ce.World._fields_ if f != "rungs"}
    np.savez_compressed(
        path, lanes=wave.lanes, muscles=wave.muscles, heads=wave.heads, slots=wave.slots,
        params=np.frombuffer(bytes(params), np.uint8), flags=np.uint32(flags), results=results,
        frames=np.stack(frames), world=np.array([repr(world_fields)]),
        genomes=pop.genomes, nodes=pop.nodes, bones=pop.bones, pop_muscles=pop.muscles, strength=pop.strength)
    return path


def main() -> None:
    for name in CASES:
        print(make(name))


if __name__ == "__main__":
    main()
