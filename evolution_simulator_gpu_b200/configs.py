"""The workloads the engine is measured and checked on: seeded synthetic
populations and their worlds.

The reference measures on saved evolved populations that are not available,
so each workload is generated from a seed (see csrc/generator.cpp for the
body and muscle rules). The worlds use the reference's level tables
(src/environment.rs:121-160, src/physics.rs:523).

1. small: 4,096 creatures (seed 0), 3-6 nodes uniform, spanning muscles plus
   up to 3 extra, joints +-120 degrees, calm world. Replay frames of the
   first 16.
2. game scale: 3,000,000 creatures (seed 1), 3-10 nodes uniform, 2-24 muscles
   uniform, calm world.
3. effects: 3,000,000 creatures (seed 2), 3-24 nodes geometric with mean 7,
   joints +-U(30, 150) degrees, spanning plus up to 3 extra muscles; rough
   ground (0.08 m), 1.5 g, thick air, wet grip, 8% slope, strong headwind,
   shallows at 0.35 m, ice patches at 80%, low hurdles.
4. gradients: 65,536 creatures (seed 3), 4-12 nodes, 4-20 muscles, flat,
   Earth gravity, grippy.
5. refined search: 1,024 parents (seed 4) of 3-16 nodes in the effects world
   plus pebbles (terrain level 1) and tremors (quake 0.05).
"""
from __future__ import annotations

import dataclasses

from .api import GenSpecPy, World, make_world

# Level tables (src/environment.rs:121-160).
GRAVITY = [9.8, 14.7, 19.6, 29.4]
AIR = [1.0, 0.995, 0.985, 0.96]
GRIP = [3.0, 1.5, 1.0, 0.6, 0.3]
SLOPE = [0.0, 0.03, 0.08, 0.15, 0.25]
WIND = [0.0, -1.0, -3.0, -6.0]
WATER = [0.0, 0.12, 0.35, 0.9]
PATCHES = [0.0, 0.5, 0.8, 0.95]
HURDLES = [0.0, 0.08, 0.20, 0.35]
QUAKE = [0.0, 0.05, 0.12, 0.25]


@dataclasses.dataclass
class Workload:
    name: str
    count: int
    spec: GenSpecPy
    world_kw: dict

    def world(self, **over) -> World:
        kw = dict(self.world_kw)
        kw.update(over)
        return make_world(**kw)


def effects_world_kw() -> dict:
    return dict(terrain=2, gravity=GRAVITY[1], air_retention=AIR[2], ground_friction=GRIP[3], slope=SLOPE[2],
                wind=WIND[2], water=WATER[2], patches=PATCHES[2], hurdles=HURDLES[1])


WORKLOADS = {
    "small": Workload("small", 4096, GenSpecPy(seed=0, min_nodes=3, max_nodes=6, muscle_rule=0, max_extra=3), {}),
    "game": Workload("game", 3_000_000,
                     GenSpecPy(seed=1, min_nodes=3, max_nodes=10, muscle_rule=1, min_muscles=2, max_muscles=24), {}),
    "effects": Workload("effects", 3_000_000,
                        GenSpecPy(seed=2, min_nodes=3, max_nodes=24, node_dist=1, mean_nodes=7.0, muscle_rule=0,
                                  max_extra=3, joint_lo_deg=30.0, joint_hi_deg=150.0), effects_world_kw()),
    "gradients": Workload("gradients", 65_536,
                          GenSpecPy(seed=3, min_nodes=4, max_nodes=12, muscle_rule=1, min_muscles=4, max_muscles=20),
                          dict(ground_friction=GRIP[0])),
    "refine": Workload("refine", 1024,
                       GenSpecPy(seed=4, min_nodes=3, max_nodes=16, muscle_rule=0, max_extra=3, joint_lo_deg=30.0,
                                 joint_hi_deg=150.0),
                       dict(effects_world_kw(), terrain=1, quake=QUAKE[1])),
}
