"""A small, GPU-filling evaluation for profilers (ncu): the bench's workloads
at sizes an ncu capture finishes in a minute or two.

    python profile_case.py --workload game \
        --creatures 300000 --seconds 1
    python profile_case.py --workload effects \
        --creatures 3000000 --seconds 20 --generations 10 --autotune

It generates the workload, runs one submission through the engine (one
launch per size class) and prints the GPU seconds, the creature-substeps the
trials ran and the bytes of the packed records.

With --generations K it packs K generations of the workload (disjoint
creature ranges), keeps them resident and runs them as one CUDA graph
(GenerationGraph), once to warm up and once timed; with --autotune the
engine's launch shape is first tuned on a sample of the workload: by
default a whole generation's worth of creatures on shorter trials
(--sample-seconds), since the best shape depends on how many creatures
share the GPU's lanes and how unevenly their trials end.

With --adjoint it runs the gradient path instead: one checkpointed forward
run (ce_forward) and one backward run (ce_backward) of the workload, and
prints both GPU times and the gradients per second.

With --refine it runs one gradient-refined search generation (refine.py):
--creatures samples of --parents parents, the --elites best refined by
--steps adjoint ascent steps, against plain resampling of the same elites
for the same GPU time, and prints the fitness gained per GPU-second of both.

    python profile_case.py --workload refine \
        --refine --creatures 1000000 --parents 1024 --elites 16384 --steps 5 --seconds 20
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="game")
    ap.add_argument("--creatures", type=int, default=300_000)
    ap.add_argument("--seconds", type=float, default=1.0)
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="resident blocks per SM (0: the engine's choice)")
    ap.add_argument("--generations", type=int, default=0, help="run K resident generations as one CUDA graph")
    ap.add_argument("--autotune", action="store_true", help="tune the launch shape on a sample first")
    ap.add_argument("--sample", type=int, default=0, help="creatures in the autotune sample (0: --creatures)")
    ap.add_argument("--sample-seconds", type=float, default=2.0, help="trial length of the autotune sample")
    ap.add_argument("--adjoint", action="store_true", help="time forward + backward of the gradient path")
    ap.add_argument("--refine", action="store_true", help="one gradient-refined search generation")
    ap.add_argument("--parents", type=int, default=1024)
    ap.add_argument("--elites", type=int, default=16_384)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--sampler", default="device", choices=["device", "host"], help="where the samples are drawn")
    ap.add_argument("--line-search", default="", help="step-size factors of a line-search ascent arm, e.g. 0.25,1,4,16")
    ap.add_argument("--cma", type=int, default=0, help="samples an elite a generation of a CMA-ES arm (0: no arm)")
    args = ap.parse_args()
    if args.generations:
        return generations(args)
    if args.adjoint:
        return adjoint(args)
    if args.refine:
        return refined(args)
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
    print(json.dumps(out))


def refined(args) -> None:
    """One refined search generation; under torchrun, over one GPU a rank
    (rank r draws and evaluates its share of the samples, the elites are
    chosen over all ranks and each rank refines its own)."""
    import os
    from datetime import timedelta

    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200 import refine
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    world_size, rank, local = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))
    device = None
    if world_size > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        device = torch.device("cuda", local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=device)
    w = WORKLOADS[args.workload]
    try:
        with ce.Engine(local) as eng:
            out = refine.search(eng, w.spec, w.world(duration=args.seconds), parents=args.parents,
                                count=args.creatures, elites=args.elites, steps=args.steps, sampler=args.sampler,
                                guided=True, rank=rank, world_size=world_size, device=device,
                                line_search=tuple(float(f) for f in args.line_search.split(",") if f),
                                cma_samples=args.cma)
    finally:
        if world_size > 1:
            dist.destroy_process_group()
    out.update(workload=args.workload, seconds=args.seconds)
    if rank == 0:
        print(json.dumps(out))


def adjoint(args) -> None:
    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    w = WORKLOADS[args.workload]
    world = w.world(duration=args.seconds)
    wave = ce.pack(ce.generate(w.spec, args.creatures), world)
    with ce.Engine(0) as eng, eng.forward(wave, world) as tape:
        g = tape.backward()
        fwd, bwd = tape.seconds
        rows, mm = tape.shape
    print(json.dumps({"workload": args.workload, "creatures": args.creatures, "seconds": args.seconds,
                      "rows": rows, "muscle_slots": mm, "forward_s": fwd, "backward_s": bwd,
                      "finite": float(np.isfinite(g).all(axis=1).mean()),
                      "gradients_per_s": args.creatures / (fwd + bwd)}))


def generations(args) -> None:
    import time
    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    w = WORKLOADS[args.workload]
    world = w.world(duration=args.seconds)
    out = {"workload": args.workload, "creatures": args.creatures, "seconds": args.seconds,
           "generations": args.generations}
    t0 = time.perf_counter()
    waves = [ce.pack(ce.generate(w.spec, args.creatures, first=k * args.creatures), world)
             for k in range(args.generations)]
    out["pack_s"] = time.perf_counter() - t0
    out["record_bytes"] = int(sum(v.lanes.nbytes + v.muscles.nbytes + v.heads.nbytes for v in waves))
    with ce.Engine(0, ctas_per_sm=args.ctas_per_sm) as eng:
        if args.autotune:
            short = w.world(duration=args.sample_seconds)
            sample = ce.pack(ce.generate(w.spec, args.sample or args.creatures, first=args.generations * args.creatures),
                             short)
            out["launch_shape"], out["autotune_best_s"] = eng.autotune(sample, short)
            del sample
        with ce.GenerationGraph(eng, waves, world) as g:
            out["warm_s"] = g.launch()
            out["graph_s"] = g.launch()
            subs = sum(ce.creature_substeps(g.results(k), world) for k in range(len(waves)))
        # One generation as a plain submission, for the per-launch comparison.
        _, out["plain_one_s"] = eng.run(waves[0], world)
    out["creature_substeps"] = subs
    out["creature_substeps_per_s"] = subs / out["graph_s"]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
