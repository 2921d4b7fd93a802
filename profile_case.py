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
    ap.add_argument("--cma-kernels", action="store_true",
                    help="time ce_cma_ask and ce_cma_tell: --creatures emitters, --cma samples an emitter")
    ap.add_argument("--exploring", action="store_true", help="with --cma-kernels: CMA-ME emitters")
    ap.add_argument("--audit", action="store_true", help="time ce_audit_device on --creatures synthetic results")
    args = ap.parse_args()
    if args.cma_kernels:
        return cma_kernels(args)
    if args.audit:
        return audit_case(args)
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


def _timed(torch, fn, reps: int) -> float:
    """Mean milliseconds of fn() over reps runs, CUDA events on the current
    stream, after two untimed runs."""
    for _ in range(2):
        fn()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / reps


def cma_kernels(args) -> None:
    """ce_cma_ask and ce_cma_tell at scale: --creatures emitters of the
    workload's bodies, --cma (default 16) samples an emitter a generation."""
    import torch

    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200.cma import CmaEmitters, dims
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    w = WORKLOADS[args.workload]
    E, per = args.creatures, args.cma or 16
    templates = ce.generate(w.spec, E)
    opt = CmaEmitters(templates, exploring=True if args.exploring else None)
    n = E * per
    state = {}

    # Device time of the kernels alone: CmaEmitters brackets each ce_cma_ask
    # and ce_cma_tell call with CUDA events (kernel_seconds).
    for _ in range(2):
        state["genes"], _ = opt.ask_device(n, seed=1, generation=0, first=0)
    opt.kernel_seconds()
    for _ in range(5):
        state["genes"], _ = opt.ask_device(n, seed=1, generation=0, first=0)
    ask_ms = opt.kernel_seconds() / 5 * 1e3
    on, ob, om, ost, og = state["genes"]
    keys = torch.randn(n, device=opt.device)
    for _ in range(2):
        opt.tell_device((on, ob, om, og), keys, 0, n)
    opt.kernel_seconds()
    for _ in range(5):
        opt.tell_device((on, ob, om, og), keys, 0, n)
    tell_ms = opt.kernel_seconds() / 5 * 1e3
    D = dims(templates.genomes, np.full(E, args.exploring) if args.exploring else None)
    gene_bytes = sum(int(t.numel()) for t in (on, ob, om, og) + ((ost,) if ost is not None else ()))
    state_bytes = int(D.sum()) * 4 * 4 + E * 4
    print(json.dumps({"case": "cma kernels", "workload": args.workload, "emitters": E, "samples": n,
                      "mode": "cma-me" if args.exploring else "optimizer", "mean_coordinates": float(D.mean()),
                      "ask_ms": ask_ms, "tell_ms": tell_ms, "samples_per_s": n / (ask_ms * 1e-3),
                      "ask_genes_bytes": gene_bytes, "ask_write_gbs": gene_bytes / (ask_ms * 1e-3) / 1e9,
                      "state_bytes": state_bytes,
                      "tell_bytes": state_bytes * 2 + gene_bytes,
                      "tell_gbs": (state_bytes * 2 + gene_bytes) / (tell_ms * 1e-3) / 1e9}))


def audit_case(args) -> None:
    """ce_audit_device on --creatures synthetic trials: random trace words,
    one creature in 128 an audit creature (rungs::AUDIT_ONE_IN), random
    screen positions and bars."""
    import ctypes as C

    import torch

    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200 import api
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    count = args.creatures
    rng = np.random.default_rng(5)
    pop = ce.generate(WORKLOADS[args.workload].spec, min(count, 65_536))
    reps = np.arange(count) % len(pop)
    genomes = pop.genomes[reps].copy()
    genomes["flags"] = np.where(rng.random(count) < 1 / 128, 1, 0).astype(np.uint32)
    words = rng.integers(0, 1 << 32, size=(count, 7), dtype=np.uint64).astype(np.uint32) & np.uint32(0x7bff7bff)
    words[:, 2] = (words[:, 2] & 0xffff) | (rng.integers(1, 1300, count).astype(np.uint32) << 16)
    res = np.zeros(count, ce.RESULT_DTYPE)
    for k, f in enumerate(("contact_hi", "lift_hi", "ground_hi", "previous_center_y", "vertical_extremum",
                           "vertical_trend", "gait_turns")):
        res[f] = words[:, k].view(np.float32)
    res["screen_x"] = rng.normal(2.0, 1.5, count).astype(np.float32)
    bars = rng.normal(2.0, 0.5, count).astype(np.float32)
    dev = torch.device("cuda", 0)

    def up(arr):
        return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(dev)

    dr, dg, dm, db = up(res), up(genomes), up(pop.muscles), up(bars)
    L = api.lib()
    scratch = torch.empty(int(L.ce_audit_scratch_bytes(count)), dtype=torch.uint8, device=dev)
    out = torch.empty(C.sizeof(api.AuditC), dtype=torch.uint8, device=dev)
    words_out = torch.empty(2 * 65_536 * 6, dtype=torch.int16, device=dev)
    stream = torch.cuda.current_stream(dev)

    def run():
        api._check(L.ce_audit_device(dr.data_ptr(), dg.data_ptr(), dm.data_ptr(), db.data_ptr(), count,
                                     scratch.data_ptr(), scratch.numel(), out.data_ptr(), words_out.data_ptr(),
                                     65_536, stream.cuda_stream), "ce_audit_device")

    ms = _timed(torch, run, 10)
    a = api.AuditC.from_buffer_copy(out.cpu().numpy().tobytes())
    once = count * (ce.RESULT_DTYPE.itemsize + api.GENOME_DTYPE.itemsize + 4)
    print(json.dumps({"case": "rung audit", "trials": count, "audit_rows": int(a.rows), "ms": ms,
                      "trials_per_s": count / (ms * 1e-3), "bytes_read_once": once,
                      "gbs_read_once": once / (ms * 1e-3) / 1e9}))


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
