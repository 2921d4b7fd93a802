"""A small, GPU-filling evaluation for profilers (ncu), and a timing check
of the engine against the reference kernel on the same case.

    python -m evolution_simulator_gpu_b200.profile_case --workload game \
        --creatures 300000 --seconds 1 [--reference]

It generates the workload, runs one submission through the engine (one
launch per size class) and prints the GPU seconds, the creature-substeps the
trials ran and the bytes of the packed records. With --reference it also
runs the reference's own kernel (oracle/_ref, built from its source) on the
same batch and prints whether the results are equal to the bit.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="game")
    ap.add_argument("--creatures", type=int, default=300_000)
    ap.add_argument("--seconds", type=float, default=1.0)
    ap.add_argument("--reference", action="store_true")
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="resident blocks per SM (0: the engine's choice)")
    args = ap.parse_args()
    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    w = WORKLOADS[args.workload]
    world = w.world(duration=args.seconds)
    pop = ce.generate(w.spec, args.creatures)
    wave = ce.pack(pop, world)
    with ce.Engine(0, ctas_per_sm=args.ctas_per_sm) as eng:
        mine, busy = eng.run(wave, world)
    out = {"workload": args.workload, "creatures": args.creatures, "seconds": args.seconds,
           "ctas_per_sm": args.ctas_per_sm, "engine_s": busy,
           "creature_substeps": ce.creature_substeps(mine, world),
           "record_bytes": int(wave.lanes.nbytes + wave.muscles.nbytes + wave.heads.nbytes)}
    if args.reference:
        sys.path.insert(0, str(ROOT))
        from oracle.ref import RefKernel
        ref, ms = RefKernel(ce.world_flags(world), world.rate or 60).run(wave, ce.make_params(world))
        out["reference_s"] = ms / 1e3
        out["bit_equal"] = bool((mine.view(np.uint32) == ref.view(np.uint32)).all())
    print(json.dumps(out))


if __name__ == "__main__":
    main()
