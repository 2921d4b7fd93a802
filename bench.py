"""Benchmark: creature-substeps per second at game scale.

Workload (per GPU): one generation of 3,000,000 seeded synthetic creatures
(seed 1, 3-10 nodes, 2-24 muscles, calm world) in 20 s trials at 60 steps a
second and 16 substeps a step. A step of the benchmark evaluates the whole
generation. A creature-substep is one substep of one creature until its trial
ends (fall, screen or last step), as the reference counts creature-steps
(examples/p2_speed.rs:55-72) times 16.

Printed, one JSON line from rank 0:
  value   -- creature-substeps/s of all ranks with the packed records already
             in GPU memory (the device-level entry ce_advance_device), timed
             with CUDA events on the launching stream, max over ranks;
  e2e     -- the same through the public C ABI with host buffers
             (ce_submit + ce_poll: upload, kernel, result download);
  roofline, cpu_baseline, clocks -- see below.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Under torchrun each rank evaluates its own generation (weak scaling).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "creature-substeps/s at 3M creatures x 20 s; adjoint grads/s vs plain-path FD"
UNIT = "creature-substeps/s"
WORKLOAD = "game"
# Kernels of one device-entry call besides the creature kernel: the node-count
# bucketing (count, scan, scatter) that builds the claim queues.
BUCKET_KERNELS = 3
WORKLOAD_TEXT = ("3,000,000 seeded synthetic creatures (seed 1), 3-10 nodes, 2-24 muscles, calm flat world, "
                 "20 s trials at 60 steps/s x 16 substeps, FP32")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--creatures", type=int, default=3_000_000)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-adjoint", action="store_true", help="leave out the gradient measurement")
    ap.add_argument("--no-effects", action="store_true", help="leave out the effects-world measurement")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ distributed
def dist_setup(gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- workload
def build_workload(n: int, rank: int):
    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    w = WORKLOADS[WORKLOAD]
    world = w.world()
    pop = ce.generate(w.spec, n, first=rank * n)
    wave = ce.pack(pop, world)
    return world, pop, wave


def results_digest(res) -> str:
    """SHA-256 of a generation's result words in packed order: the engine arm
    and the reference arm print it for the same generation, so equal digests
    show the two kernels' results equal to the bit."""
    return hashlib.sha256(np.ascontiguousarray(res).view(np.uint8).tobytes()).hexdigest()


def op_counts() -> dict:
    path = ROOT / "profiles" / "op_counts.json"
    return json.loads(path.read_text()) if path.exists() else {}


def traffic_model():
    """(bytes per creature, bytes per creature-substep) of DRAM traffic of the
    creature kernel, from two ncu captures (profiles/traffic.json)."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None
    t = json.loads(path.read_text()).get(WORKLOAD, {})
    if "dram_bytes_per_substep" not in t:
        return None
    return t.get("dram_bytes_per_creature", 0.0), t["dram_bytes_per_substep"]


# ---------------------------------------------------------------- CPU baseline
def cpu_sample(wave, world, budget_s: float, phase: int = 0):
    """The CPU oracle (oracle/creature_oracle.cpp, FP32, all host threads) on a
    bounded sample of the generation: chunks of 64 creatures per thread taken
    from 64 evenly spread places of the packed order (which is sorted by size,
    so the sample spans every size), shifted by `phase` chunks so repeated
    samples differ, until `budget_s` seconds of oracle time. Returns
    (creature-substeps, seconds, creatures, threads)."""
    import evolution_simulator_gpu_b200 as ce
    from oracle.ref import Oracle
    oracle = Oracle()
    params = ce.make_params(world)
    flags = ce.world_flags(world)
    cores = os.cpu_count() or 1
    n = len(wave)
    chunk = min(64 * cores, n)
    starts = np.linspace(0, n - chunk, 64).astype(np.int64)
    starts = (starts + phase * chunk) % (n - chunk + 1)
    done = secs = 0.0
    creatures = 0
    for s in starts:
        res, t = oracle.run(wave, params, flags, world.rate or 60, int(s), chunk, threads=cores)
        secs += t
        done += ce.creature_substeps(res, world)
        creatures += chunk
        if secs > budget_s:
            break
    return done, secs, creatures, cores


def cpu_baseline(wave, world, budget_s: float) -> dict:
    done, secs, creatures, cores = cpu_sample(wave, world, budget_s)
    return {"value": done / secs, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{creatures} creatures of the same generation (chunks spread over the packed order), "
                      f"{done:.3g} creature-substeps in {secs:.1f} s"}


# ---------------------------------------------------------------- gradients
ADJOINT_TEXT = ("65,536 seeded synthetic creatures (seed 3), 4-12 nodes, 4-20 muscles, flat grippy calm world, "
                "20 s trials, FP32, checkpoints every 256 substeps; gradient = d fitness / d (short, long, strength, "
                "on time, off time of every muscle, friction of every node)")


def gradient_workload():
    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    w = WORKLOADS["gradients"]
    world = w.world()
    pop = ce.generate(w.spec, w.count)
    wave = ce.pack(pop, world)
    params = 5 * wave.heads[:, 1].astype(np.int64).sum() + (wave.heads[:, 0] & 255).astype(np.int64).sum()
    return world, pop, wave, float(params) / len(wave)


def adjoint_bench(eng) -> dict:
    """Full gradients per second of the adjoint (ce_forward + ce_backward,
    GPU time) against central finite differences on the plain kernel (2
    forward trials a parameter, GPU time of the plain submission)."""
    world, pop, wave, params = gradient_workload()
    eng.run(wave, world)
    _, plain_s = eng.run(wave, world)
    with eng.forward(wave, world) as tape:
        tape.backward()
    with eng.forward(wave, world) as tape:
        tape.backward()
        forward_s, backward_s = tape.seconds
    adjoint = len(wave) / (forward_s + backward_s)
    fd = len(wave) / (plain_s * 2.0 * params)
    return {"workload": ADJOINT_TEXT, "unit": "gradients/s", "value": adjoint, "fd_value": fd,
            "speedup_vs_fd": adjoint / fd, "params_per_creature": params, "forward_s": forward_s,
            "backward_s": backward_s, "plain_s": plain_s, "creatures": len(wave),
            "timing": "CUDA events around the kernels of one batch (forward with checkpoints, backward; "
                      "plain submission)"}


EFFECTS_TEXT = ("3,000,000 seeded synthetic creatures (seed 2), 3-24 nodes (geometric, mean 7), joint ranges "
                "+-U(30, 150) deg, rough ground 0.08 m, 1.5 g, thick air, wet grip, 8% slope, headwind, shallows "
                "0.35 m, ice patches, low hurdles; 20 s trials, FP32")


def effects_workload():
    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    w = WORKLOADS["effects"]
    world = w.world()
    return world, ce.pack(ce.generate(w.spec, w.count), world)


def effects_bench(eng) -> dict:
    """One generation of the effects workload through ce_submit (GPU-busy
    time of the second of two submissions)."""
    import evolution_simulator_gpu_b200 as ce
    world, wave = effects_workload()
    eng.run(wave, world)
    res, busy = eng.run(wave, world)
    units = ce.creature_substeps(res, world)
    return {"workload": EFFECTS_TEXT, "unit": UNIT, "value": units / busy, "seconds": busy,
            "creature_substeps": units,
            "timing": "CUDA events around one submission (bucketing and both size classes)"}


# ---------------------------------------------------------------- engine arm
def f3_bench(d_results, pop, wave, dev) -> dict:
    """Row f3 on this generation: the rung audit of its results (population
    order; audit creatures flagged as rungs::is_audit flags them, bars at the
    generation's median 5 s position) and a CMA ask and tell of 16,384
    optimizer emitters x 16 samples on the refine workload's bodies; CUDA
    events around the library calls, after two untimed calls."""
    import ctypes as C

    import torch

    import evolution_simulator_gpu_b200 as ce
    from evolution_simulator_gpu_b200 import api
    from evolution_simulator_gpu_b200.cma import CmaEmitters
    from evolution_simulator_gpu_b200.configs import WORKLOADS
    n = len(wave)
    inv = torch.from_numpy(np.argsort(wave.slots).astype(np.int64)).to(dev)
    d_res = d_results.view(n, 19).index_select(0, inv).contiguous()
    genomes = pop.genomes.copy()
    genomes["flags"] = api.audit_flags(1, 0, np.arange(n))
    screen_x = d_res[:, api.RESULT_FIELDS.index("screen_x")].cpu().numpy()
    bars = np.full(n, np.float32(np.median(screen_x)), np.float32)

    def up(arr):
        return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(dev)

    d_g, d_m, d_b = up(genomes), up(pop.muscles), up(bars)
    L = api.lib()
    scratch = torch.empty(int(L.ce_audit_scratch_bytes(n)), dtype=torch.uint8, device=dev)
    out = torch.empty(C.sizeof(api.AuditC), dtype=torch.uint8, device=dev)
    words = torch.empty(2 * 65_536 * 6, dtype=torch.int16, device=dev)
    stream = torch.cuda.current_stream(dev)

    def audit():
        api._check(L.ce_audit_device(d_res.data_ptr(), d_g.data_ptr(), d_m.data_ptr(), d_b.data_ptr(), n,
                                     scratch.data_ptr(), scratch.numel(), out.data_ptr(), words.data_ptr(), 65_536,
                                     stream.cuda_stream), "ce_audit_device")

    for _ in range(2):
        audit()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(10):
        audit()
    b.record(stream)
    b.synchronize()
    audit_ms = a.elapsed_time(b) / 10
    rows = int(api.AuditC.from_buffer_copy(out.cpu().numpy().tobytes()).rows)

    E, per = 16_384, 16
    opt = CmaEmitters(ce.generate(WORKLOADS["refine"].spec, E), device=dev.index)
    for _ in range(2):
        genes, _ = opt.ask_device(E * per, seed=1, first=0)
    keys = torch.randn(E * per, device=dev)
    opt.tell_device(genes[:3] + genes[4:], keys, 0, E * per)
    opt.kernel_seconds()
    for _ in range(5):
        genes, _ = opt.ask_device(E * per, seed=1, first=0)
    ask_ms = opt.kernel_seconds() / 5 * 1e3
    for _ in range(5):
        opt.tell_device(genes[:3] + genes[4:], keys, 0, E * per)
    tell_ms = opt.kernel_seconds() / 5 * 1e3
    return {"audit": {"trials": n, "audit_rows": rows, "ms": audit_ms, "trials_per_s": n / (audit_ms * 1e-3)},
            "cma": {"emitters": E, "samples": E * per, "ask_ms": ask_ms, "tell_ms": tell_ms,
                    "samples_per_s": E * per / (ask_ms * 1e-3)},
            "timing": "CUDA events around the library calls (ce_audit_device; ce_cma_ask, ce_cma_tell)"}


def run_engine(args):
    world_size, rank, local = dist_setup(args.gpus)
    import torch

    import evolution_simulator_gpu_b200 as ce
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    world, pop, wave = build_workload(args.creatures, rank)
    eng = ce.Engine(local)
    flags = ce.world_flags(world)
    rate = world.rate or 60
    max_nodes, max_muscles = wave.max_nodes, wave.max_muscles
    params = ce.make_params(world, 0, len(wave), 0)
    # Device-resident records (the inputs of the value measurement).
    d_lanes = torch.from_numpy(wave.lanes.view(np.int32)).to(dev)
    d_muscles = torch.from_numpy(wave.muscles).to(dev)
    d_heads = torch.from_numpy(wave.heads.view(np.int32).reshape(-1)).to(dev)
    d_results = torch.zeros(len(wave) * 19, dtype=torch.float32, device=dev)
    d_counter = torch.zeros(16, dtype=torch.int32, device=dev)
    d_scratch = torch.empty(eng.scratch_bytes(flags, rate, max_nodes, max_muscles, len(wave)), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def one_step():
        d_counter.zero_()
        eng.advance_device(d_lanes.data_ptr(), d_muscles.data_ptr(), d_heads.data_ptr(), d_results.data_ptr(),
                           d_counter.data_ptr(), d_scratch.data_ptr(), params, flags, rate, max_nodes, max_muscles,
                           stream.cuda_stream)

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize(dev)
    res = d_results.cpu().numpy().view(ce.RESULT_DTYPE)
    units = ce.creature_substeps(res, world)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world_size)
    torch.cuda.synchronize(dev)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launch_ms = []
    start.record(stream)
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one_step()
        e1.record(stream)
        launch_ms.append((e0, e1))
    stop.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world_size)
    clk = clocks.stop()
    ms = start.elapsed_time(stop)
    per_launch_ms = float(np.mean([a.elapsed_time(b) for a, b in launch_ms]))
    ms_max = max_over_ranks(ms, world_size)
    total_units = sum_over_ranks(units * args.steps, world_size)
    value = total_units / (ms_max / 1e3)

    # End to end through the C ABI with host buffers.
    e2e_launches = 0
    nodes = wave.heads[:, 0] & 255
    classes = int((nodes <= 16).any()) + int((nodes > 16).any())
    h2d = wave.lanes.nbytes + wave.muscles.nbytes + wave.heads.nbytes + 4 * len(wave)
    d2h = len(wave) * ce.RESULT_DTYPE.itemsize
    eng.run(wave, world)  # buffers sized, pinned staging allocated
    barrier(world_size)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out, busy = eng.run(wave, world)
        e2e_launches += BUCKET_KERNELS + classes
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world_size)
    e2e_value = sum_over_ranks(ce.creature_substeps(out, world) * args.steps, world_size) / e2e_s
    same = bool((out.view(np.uint32) == res.view(np.uint32)).all())

    if rank == 0:
        counts = op_counts().get(WORKLOAD, {})
        flops_per = counts.get("flops_per_substep")
        peak = ce.measure_fp32(local)
        achieved = flops_per * units / (per_launch_ms / 1e3) / 1e12 if flops_per else None
        tm = traffic_model()
        roofline = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak if achieved else None,
                    "traffic": tm[0] * len(wave) + tm[1] * units if tm else None,
                    "traffic_unit": "bytes per launch (ncu capture scaled by creatures and substeps)",
                    "peak_source": "measured: FP32 multiply-add calibration kernel (ce_measure_fp32) on this GPU",
                    "numerator": f"{flops_per:.0f} algorithmic FP32 operations per creature-substep "
                                 "(oracle op count, profiles/op_counts.json) x creature-substeps of the launch"
                    if flops_per else None}
        cpu = cpu_baseline(wave, world, args.cpu_seconds)
        adjoint = adjoint_bench(eng) if not args.no_adjoint else None
        effects = effects_bench(eng) if not args.no_effects else None
        f3 = f3_bench(d_results, pop, wave, dev)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD_TEXT, "creatures_per_gpu": len(wave),
                       "trial_steps": ce.trial_steps(world), "substeps_per_step": 16,
                       "mean_steps_run": units / 16.0 / len(wave),
                       "nominal_creature_substeps": len(wave) * ce.trial_steps(world) * 16,
                       "trials_ended_early": float(((res["fall_time"] > 0) | (res["screened"] > 0)).mean()),
                       "l2": "inputs larger than L2 (%.1f GB of packed records per GPU)" % (h2d / 1e9),
                       "parallelism": f"dp{world_size} (independent generations per GPU)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "seconds_per_step": e2e_s / args.steps, "timing": "host wall clock around ce_submit+ce_poll",
                    "results_equal_device_entry": same},
            "parity": {"results_sha256": results_digest(res),
                       "compare_with": "the reference arm's reference_gpu.results_sha256: the reference kernel's "
                                       "results for the same generation in the same packed order"},
            "gpu_launches": (BUCKET_KERNELS + 1) * args.steps, "gpu_launches_e2e": e2e_launches,
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "adjoint": adjoint, "effects": effects,
            "f3": f3,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference arm: the reference path has no CPU implementation of its
    own (its only physics is the CUDA kernel, src/physics.rs:3-6), so it is
    timed as the CPU restatement of that kernel (the oracle port) on all host
    cores, one bounded sample of the generation per step. The reference's own
    kernel, built from its source for this GPU, is timed beside it on the same
    generation (reference_gpu)."""
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import evolution_simulator_gpu_b200 as ce
    from oracle.ref import RefKernel
    world, pop, wave = build_workload(args.creatures, 0)
    params = ce.make_params(world)
    flags = ce.world_flags(world)
    per_step = max(args.cpu_seconds / 4.0, 2.0)
    phase = 0
    for _ in range(args.warmup):
        cpu_sample(wave, world, per_step, phase)
        phase += 1
    tot_units = tot_secs = 0.0
    tot_count = 0
    for _ in range(args.steps):
        u, s, c, cores = cpu_sample(wave, world, per_step, phase)
        phase += 1
        tot_units += u
        tot_secs += s
        tot_count += c
    value = tot_units / tot_secs
    ref_gpu = None
    try:
        kern = RefKernel(flags, world.rate or 60)
        kern.run(wave.take(np.arange(4096)), params)
        res, ms = kern.run(wave, params)
        ref_gpu = {"value": ce.creature_substeps(res, world) / (ms / 1e3), "unit": UNIT,
                   "results_sha256": results_digest(res),
                   "what": "the reference's own kernel (shaders/creature.cu) built for sm_100a with its NVRTC "
                           "options, launched with its engine's wave and grid rule, CUDA-event time of one "
                           "generation", "seconds": ms / 1e3}
        gworld, _, gwave, gparams = gradient_workload()
        gkern = RefKernel(ce.world_flags(gworld), gworld.rate or 60)
        gkern.run(gwave.take(np.arange(4096)), ce.make_params(gworld))
        _, gms = gkern.run(gwave, ce.make_params(gworld))
        ref_gpu["fd_gradients"] = {"unit": "gradients/s", "workload": ADJOINT_TEXT,
                                   "value": len(gwave) / (gms / 1e3 * 2.0 * gparams),
                                   "what": "central finite differences on the reference's kernel: 2 trials a "
                                           "parameter (the reference has no gradients)"}
        if not args.no_effects:
            eworld, ewave = effects_workload()
            ekern = RefKernel(ce.world_flags(eworld), eworld.rate or 60)
            ekern.run(ewave.take(np.arange(4096)), ce.make_params(eworld))
            eres, ems = ekern.run(ewave, ce.make_params(eworld))
            ref_gpu["effects"] = {"workload": EFFECTS_TEXT, "unit": UNIT, "seconds": ems / 1e3,
                                  "value": ce.creature_substeps(eres, eworld) / (ems / 1e3)}
    except Exception as exc:  # the reference kernel needs a GPU
        ref_gpu = {"unavailable": str(exc).splitlines()[0]}
    sample = (f"{tot_count} creatures of the generation (chunks spread over the packed order), "
              f"{tot_units:.3g} creature-substeps in {tot_secs:.1f} s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD_TEXT, "creatures_per_gpu": len(wave)},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
