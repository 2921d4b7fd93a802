"""Gradient-refined search generation: Gaussian samples of parent genomes,
one batched evaluation, adjoint gradient ascent on the best samples, and
plain resampling of the same elites for the same GPU time as the yardstick.

The samples move the optimizer's parameter vector of a body
(src/qd.rs:2700-2770, `parameters` / `write_parameters`): per node x, y,
diameter and friction; per bone rest length, joint range and organ; one log
period shared by the muscles; per muscle the anchors, short and long length,
phase, duty, log stiffness and reset phase. Coordinates go back to genes as
`apply_parameters` does (src/qd.rs:2773-2811: y at least 0, rest length in
[0.03, max bone], joint range within +-JOINT_LIMIT on its side, organ mass at
least 0 and its place in [0, 1], the period scaled by exp(log period) / the
first muscle's period within [min period, 10] s, anchors in [0, 1], short in
[0.01, 0.8 max stroke], long in [short, max stroke], phase and reset wrapped,
duty in [0.05, 0.95], stiffness exp(.) in [1, 120]), then the diameter and
friction are held to the workload's ranges as `repair` holds them to the
configured ones (src/evolution.rs:1230-1234). The topology never changes, so
the rest of `repair` has nothing to do. The samples carry the muscles'
strength factors of their parents unchanged (the parameter vector has none).

The ascent moves the coordinates the adjoint differentiates: per muscle short,
long, strength factor, phase and duty (phase = frac(-t_on / period), duty =
(t_off - t_on) / period), per node friction. A step adds, per coordinate,
`step` x gradient clipped to the coordinate's unit step of the optimizer's
layout (src/qd.rs:2620-2660: 0.02 x the body's mean bone length for lengths,
0.05 for phase and duty, 0.03 for friction; 0.05 for the strength factor),
then applies the same clamps. A creature keeps the best fitness it reached.
"""
from __future__ import annotations

import time

import numpy as np

from . import api, shard

MAX_BONE = 2.0            # physics::Limits::DEFAULT.max_bone (src/physics.rs:142-153)
MAX_STROKE = 2.0          # .max_stroke
MIN_PERIOD = 0.2          # .min_period
JOINT_LIMIT = float(np.float32(120.0 * np.pi / 180.0))  # src/evolution.rs:92
DIAMETER = (0.06, 0.12)   # the workloads' node diameters
FRICTION = (0.0, 1.0)     # the workloads' node friction
STRENGTH = (0.5, 1.5)     # the workloads' strength factors
UNIT = dict(length=0.02, phase=0.05, duty=0.05, friction=0.03, strength=0.05)
SAMPLE_BLOCK = 4096       # samples drawn from one random stream


def take(pop: api.Population, idx, ids=None) -> api.Population:
    """The creatures `idx` of `pop` (repeats allowed) as a population of
    their own, in that order, with genome ids `ids` (theirs by default)."""
    idx = np.asarray(idx, np.int64)
    g = pop.genomes[idx]

    def gather(start, count, arr):
        cnt = g[count].astype(np.int64)
        out_start = np.cumsum(cnt) - cnt
        src = np.repeat(g[start].astype(np.int64) - out_start, cnt) + np.arange(int(cnt.sum()))
        # Rows as plain 32-bit words: fancy indexing of a structured array
        # is several times slower.
        words = arr.view(np.uint32).reshape(len(arr), arr.dtype.itemsize // 4)
        return words[src].reshape(-1).view(arr.dtype), out_start, cnt, src

    nodes, ns, nc, _ = gather("node_start", "node_count", pop.nodes)
    bones, bs, bc, _ = gather("bone_start", "bone_count", pop.bones)
    muscles, ms, mc, msrc = gather("muscle_start", "muscle_count", pop.muscles)
    strength = None if pop.strength is None else pop.strength[msrc].copy()
    genomes = np.zeros(len(idx), api.GENOME_DTYPE)
    genomes["node_start"], genomes["node_count"] = ns, nc
    genomes["bone_start"], genomes["bone_count"] = bs, bc
    genomes["muscle_start"], genomes["muscle_count"] = ms, mc
    genomes["id"] = g["id"] if ids is None else np.asarray(ids, np.uint64)
    genomes["flags"] = g["flags"]
    return api.Population(nodes, bones, muscles, genomes, strength)


def _owner(pop: api.Population, start: str, count: str) -> np.ndarray:
    """The creature of each node, bone or muscle row."""
    return np.repeat(np.arange(len(pop.genomes)), pop.genomes[count].astype(np.int64))


def _size(pop: api.Population) -> np.ndarray:
    """Each creature's mean bone rest length within [0.05, 10] (1 without
    bones): the optimizer layout's length unit (src/qd.rs:2641-2655)."""
    owner = _owner(pop, "bone_start", "bone_count")
    total = np.bincount(owner, pop.bones["rest_length"].astype(np.float64), len(pop.genomes))
    cnt = pop.genomes["bone_count"].astype(np.float64)
    size = np.where(cnt > 0, total / np.maximum(cnt, 1.0), 1.0)
    return np.clip(size, 0.05, 10.0).astype(np.float32)


def concat(pops) -> api.Population:
    """Populations one after another as one population."""
    pops = list(pops)
    genomes = np.concatenate([p.genomes for p in pops])
    for field, rows in (("node_start", "nodes"), ("bone_start", "bones"), ("muscle_start", "muscles")):
        offsets = np.cumsum([0] + [len(getattr(p, rows)) for p in pops[:-1]])
        genomes[field] += np.repeat(offsets, [len(p.genomes) for p in pops]).astype(np.uint32)
    strength = None if pops[0].strength is None else np.concatenate([p.strength for p in pops])
    return api.Population(np.concatenate([p.nodes for p in pops]), np.concatenate([p.bones for p in pops]),
                          np.concatenate([p.muscles for p in pops]), genomes, strength)


def _perturb(pop: api.Population, sigma: float, rng) -> None:
    """Every parameter-vector coordinate of every creature of `pop` moved by
    sigma x N(0, 1), back to genes with the clamps (in place)."""
    f32 = np.float32

    def noise(n):
        return f32(sigma) * rng.standard_normal(n, dtype=f32)

    count = len(pop)
    n = pop.nodes
    n["x"] += noise(len(n))
    n["y"] = np.maximum(n["y"] + noise(len(n)), f32(0.0))
    n["diameter"] = np.clip(n["diameter"] + noise(len(n)), *DIAMETER)
    n["friction"] = np.clip(n["friction"] + noise(len(n)), *FRICTION)
    b = pop.bones
    b["rest_length"] = np.clip(b["rest_length"] + noise(len(b)), f32(0.03), f32(MAX_BONE))
    b["min_angle"] = np.clip(b["min_angle"] + noise(len(b)), f32(-JOINT_LIMIT), f32(0.0))
    b["max_angle"] = np.clip(b["max_angle"] + noise(len(b)), f32(0.0), f32(JOINT_LIMIT))
    b["organ_mass"] = np.maximum(b["organ_mass"] + noise(len(b)), f32(0.0))
    b["organ_at"] = np.clip(b["organ_at"] + noise(len(b)), f32(0.0), f32(1.0))
    m = pop.muscles
    owner = _owner(pop, "muscle_start", "muscle_count")
    first = pop.genomes["muscle_start"].astype(np.int64)
    has = pop.genomes["muscle_count"] > 0
    base = np.ones(count, f32)
    base[has] = np.maximum(m["period"][first[has]], f32(1e-3))
    log_period = np.log(base) + noise(count)
    scale = np.clip(np.exp(log_period), f32(MIN_PERIOD), f32(10.0)) / base
    m["anchor_a"] = np.clip(m["anchor_a"] + noise(len(m)), f32(0.0), f32(1.0))
    m["anchor_b"] = np.clip(m["anchor_b"] + noise(len(m)), f32(0.0), f32(1.0))
    m["short"] = np.clip(m["short"] + noise(len(m)), f32(0.01), f32(0.8 * MAX_STROKE))
    m["long"] = np.clip(m["long"] + noise(len(m)), m["short"], f32(MAX_STROKE))
    m["period"] = np.clip(m["period"] * scale[owner], f32(MIN_PERIOD), f32(10.0))
    m["phase"] = np.mod(m["phase"] + noise(len(m)), f32(1.0))
    m["duty"] = np.clip(m["duty"] + noise(len(m)), f32(0.05), f32(0.95))
    m["stiffness"] = np.clip(np.exp(np.log(np.maximum(m["stiffness"], f32(1e-3))) + noise(len(m))), f32(1.0),
                             f32(120.0))
    m["reset"] = np.mod(m["reset"] + noise(len(m)), f32(1.0))


def samples(parents: api.Population, count: int, sigma: float, seed: int, first_id: int = 1, first: int = 0):
    """Samples [first, first + count): sample i is a child of parent
    i mod len(parents) with every parameter-vector coordinate moved by
    sigma x N(0, 1) and id first_id + i. Its moves come from the random
    stream of its block of SAMPLE_BLOCK samples, seeded with (seed, block),
    so a sample is the same whichever range of samples a rank draws.
    Returns (population, parent of each sample)."""
    P = len(parents)
    parts = []
    blocks = range(first // SAMPLE_BLOCK, (first + count - 1) // SAMPLE_BLOCK + 1) if count > 0 else range(0)
    for blk in blocks:
        c0, c1 = blk * SAMPLE_BLOCK, (blk + 1) * SAMPLE_BLOCK
        idx = np.arange(c0, c1, dtype=np.int64)
        pop = take(parents, idx % P, first_id + idx.astype(np.uint64))
        _perturb(pop, sigma, np.random.default_rng([seed, blk]))
        lo, hi = max(first, c0) - c0, min(first + count, c1) - c0
        parts.append(pop if (lo, hi) == (0, SAMPLE_BLOCK) else take(pop, np.arange(lo, hi)))
    pop = concat(parts) if parts else take(parents, np.zeros(0, np.int64))
    return pop, np.arange(first, first + count, dtype=np.int64) % P


def samples_gpu(parents: api.Population, count: int, sigma: float, seed: int, first_id: int = 1, first: int = 0,
                device=None):
    """Samples [first, first + count) drawn on the GPU (ce_sample_device):
    the moves of `samples`, from a counter-based hash of (seed, sample, gene,
    field) instead of numpy's streams, on GPU `device` (the current one by
    default). Returns (population on the host, parent of each sample)."""
    import torch
    import ctypes as C
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    par = take(parents, np.arange(len(parents)))  # genes packed in order from row 0

    def up(arr):
        return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(dev)

    dn, db, dm, dg = up(par.nodes), up(par.bones), up(par.muscles), up(par.genomes)
    ds = None if par.strength is None else up(par.strength)
    rn, rb, rm = C.c_size_t(), C.c_size_t(), C.c_size_t()
    L = api.lib()
    api._check(L.ce_sample_rows(api._ptr(par.genomes), len(par), first, count, C.byref(rn), C.byref(rb), C.byref(rm)),
               "ce_sample_rows")

    def out(rows, dtype):
        return torch.empty(max(rows * dtype.itemsize, 1), dtype=torch.uint8, device=dev)

    on, ob, om = out(rn.value, api.NODE_DTYPE), out(rb.value, api.BONE_DTYPE), out(rm.value, api.MUSCLE_DTYPE)
    og, ost = out(count, api.GENOME_DTYPE), out(rm.value, np.dtype(np.float32))
    pc = api.PopulationC(dn.data_ptr(), db.data_ptr(), dm.data_ptr(), dg.data_ptr(), len(par),
                         None if ds is None else ds.data_ptr())
    stream = torch.cuda.current_stream(dev)
    api._check(L.ce_sample_device(C.byref(pc), first, count, sigma, seed, first_id, on.data_ptr(), ob.data_ptr(),
                                  om.data_ptr(), ost.data_ptr(), og.data_ptr(), stream.cuda_stream),
               "ce_sample_device")
    stream.synchronize()

    def back(t, rows, dtype):
        return t.cpu().numpy()[:rows * dtype.itemsize].view(dtype).copy()

    pop = api.Population(back(on, rn.value, api.NODE_DTYPE), back(ob, rb.value, api.BONE_DTYPE),
                         back(om, rm.value, api.MUSCLE_DTYPE), back(og, count, api.GENOME_DTYPE),
                         None if ds is None else back(ost, rm.value, np.dtype(np.float32)))
    return pop, np.arange(first, first + count, dtype=np.int64) % len(parents)


def ascend(pop: api.Population, muscle_grads: np.ndarray, node_grads: np.ndarray, step: float) -> api.Population:
    """One clipped gradient-ascent step on the differentiated coordinates
    (see the module docstring), from gene gradients (gene_gradients: per
    muscle d/d short, long, strength factor, t_on, t_off; per node d/d
    friction). Returns a new population."""
    out = api.Population(pop.nodes.copy(), pop.bones.copy(), pop.muscles.copy(), pop.genomes.copy(),
                         None if pop.strength is None else pop.strength.copy())
    f32 = np.float32
    gm = np.nan_to_num(np.asarray(muscle_grads, np.float64), nan=0.0, posinf=0.0, neginf=0.0)
    gn = np.nan_to_num(np.asarray(node_grads, np.float64), nan=0.0, posinf=0.0, neginf=0.0)
    m = out.muscles
    T = m["period"].astype(np.float64)
    length_unit = (UNIT["length"] * _size(out)[_owner(out, "muscle_start", "muscle_count")]).astype(np.float64)

    def move(g, unit):
        return np.clip(step * g, -unit, unit).astype(f32)

    m["short"] = np.clip(m["short"] + move(gm[:, 0], length_unit), f32(0.01), f32(0.8 * MAX_STROKE))
    m["long"] = np.clip(m["long"] + move(gm[:, 1], length_unit), m["short"], f32(MAX_STROKE))
    m["phase"] = np.mod(m["phase"] + move(-T * (gm[:, 3] + gm[:, 4]), UNIT["phase"]), f32(1.0))
    m["duty"] = np.clip(m["duty"] + move(T * gm[:, 4], UNIT["duty"]), f32(0.05), f32(0.95))
    if out.strength is not None:
        out.strength[:] = np.clip(out.strength + move(gm[:, 2], UNIT["strength"]), *STRENGTH)
    out.nodes["friction"] = np.clip(out.nodes["friction"] + move(gn, UNIT["friction"]), *FRICTION)
    return out


def pick(cands, choice: np.ndarray, fallback: api.Population) -> api.Population:
    """Per creature c the genes of cands[choice[c]] (-1: `fallback`'s). The
    candidates and the fallback share one layout (ascend keeps it)."""
    out = api.Population(fallback.nodes.copy(), fallback.bones.copy(), fallback.muscles.copy(),
                         fallback.genomes.copy(), None if fallback.strength is None else fallback.strength.copy())
    m_own = _owner(out, "muscle_start", "muscle_count")
    n_own = _owner(out, "node_start", "node_count")
    for j, cand in enumerate(cands):
        mrows = choice[m_own] == j
        out.muscles[mrows] = cand.muscles[mrows]
        if out.strength is not None:
            out.strength[mrows] = cand.strength[mrows]
        nrows = choice[n_own] == j
        out.nodes[nrows] = cand.nodes[nrows]
    return out


def _fitness(wave: api.WavePack, results: np.ndarray) -> np.ndarray:
    """Fitness in population order from results in packed order."""
    out = np.empty(len(wave), np.float32)
    out[wave.slots] = results["fitness"]
    return out


def _evaluate(engine, pop, world, chunk: int):
    """(fitness in population order, GPU-busy seconds), in chunks."""
    fit = np.empty(len(pop), np.float32)
    busy = 0.0
    for lo in range(0, len(pop), chunk):
        part = take(pop, np.arange(lo, min(lo + chunk, len(pop))))
        wave = api.pack(part, world)
        res, secs = engine.run(wave, world)
        fit[lo:lo + len(part)] = _fitness(wave, res)
        busy += secs
    return fit, busy


def search(engine, spec, world, parents: int = 1024, count: int = 1_000_000, sigma: float = 0.05,
           elites: int = 16_384, steps: int = 5, step: float = 1e-2, seed: int = 4, chunk: int = 2_000_000,
           resample: bool = True, rank: int = 0, world_size: int = 1, group=None, device=None,
           sampler: str = "host", guided: bool = False, ascent: str = "device", line_search=(),
           cma_samples: int = 0) -> dict:
    """One gradient-refined search generation and its resampling yardstick.

    1. `count` samples of `parents` parents (σ = sigma), evaluated in one
       batch; 2. the `elites` best get `steps` ascent steps, each a
       checkpointed forward run (which also scores the current genes) and a
       backward run, then a last evaluation; 3. plain resampling gives the
       same elites children (σ = sigma) for about the same GPU time, each
       elite keeping the best of itself and its children. Fitness gained is
       the elites' mean best fitness minus their mean sampled fitness; GPU
       seconds are the kernels' device time summed over ranks (host packing
       not included).

    Over several ranks (one GPU each, `group` a torch.distributed group):
    rank r draws and evaluates samples [count r / W, count (r + 1) / W), the
    elites are chosen once over all ranks (an all-gather of each rank's best
    (fitness, sample) pairs), and each rank refines and resamples the elites
    among its own samples; the report's figures are totals over the ranks,
    the same on every rank. `sampler` "device" draws the samples on the GPU
    (samples_gpu), "host" with numpy (samples). With `guided`, a third arm
    spends the same GPU time on one gradient of each elite (the
    refinement's first forward and backward run) and children drawn around
    the elite moved by one ascent step instead of around the elite.
    `ascent` "device" runs the ascent steps and the last scoring as one CUDA
    graph on the GPU (api.Ascent: no host round trip between the steps),
    "host" step by step through the host (packing, gene gradients and the
    step in numpy); both give the same fitness and genes. With
    `line_search` (step-size factors, e.g. (0.25, 1, 4, 16)), a further arm
    runs `steps` ascent steps whose size each creature chooses: per step one
    gradient (checkpointed forward and backward run), then one evaluation of
    each factor's step, and each creature moves to its best candidate if
    that beats where it stands; its GPU time counts every evaluation. With
    `cma_samples` > 0, a further arm gives every elite a separable CMA-ES
    optimizer (the reference's optimizer emitter, cma.CmaEmitters, its
    ask and tell on the GPU) and runs generations of `cma_samples` samples
    an elite for about the same GPU time, ask and tell kernels included;
    each elite keeps the best of itself and its optimizer's samples."""
    draw = samples if sampler == "host" else samples_gpu
    report = dict(parents=parents, samples=count, sigma=sigma, elites=elites, steps=steps, step=step,
                  ranks=world_size, sampler=sampler, ascent=ascent)
    lo, hi = count * rank // world_size, count * (rank + 1) // world_size
    t0 = time.perf_counter()
    base = api.generate(spec, parents)
    pop, _ = draw(base, hi - lo, sigma, seed, first=lo)
    report["host_sample_s"] = time.perf_counter() - t0
    fit, busy = _evaluate(engine, pop, world, chunk)
    valid = np.isfinite(fit) & (fit > -1e19)
    _, chosen = shard.global_top_k(np.where(valid, fit, -np.inf), lo + np.arange(hi - lo), elites, world_size, group,
                                   device)
    mine = np.sort(chosen[(chosen >= lo) & (chosen < hi)]) - lo
    elite = take(pop, mine)
    f0 = fit[mine].astype(np.float64)
    # Gradient refinement of this rank's elites.
    best = f0.copy()
    x = elite
    refine_s = 0.0
    first_equal = True
    stepped, grad_s = None, 0.0
    t0 = time.perf_counter()
    last_s = 0.0
    if ascent == "device" and len(mine) and steps:
        with api.Ascent(engine, elite, world, steps, step) as asc:
            refine_s = asc.launch()
            for k in range(steps + 1):
                fk = asc.fitness(k).astype(np.float64)
                if k == 0:
                    first_equal = bool(np.array_equal(fk, f0))
                best = np.maximum(best, np.where(fk > -1e19, fk, -np.inf))
        if guided:
            # The genes after one step, and that step's GPU time (a
            # one-step ascent: its forward and backward runs, the step and
            # one scoring of the moved genes).
            with api.Ascent(engine, elite, world, 1, step) as one:
                grad_s = one.launch()
                stepped = one.population()
    else:
        for k in range(steps if len(mine) else 0):
            wave = api.pack(x, world)
            with engine.forward(wave, world) as tape:
                fk = _fitness(wave, tape.results).astype(np.float64)
                g = tape.backward()
                shape = tape.shape
                fwd, bwd = tape.seconds
            refine_s += fwd + bwd
            if k == 0:
                # The elites' genes, scored again by the checkpointed forward run.
                first_equal = bool(np.array_equal(fk, f0))
            best = np.maximum(best, np.where(fk > -1e19, fk, -np.inf))
            mg, ng = api.gene_gradients(x, wave, world, g, shape)
            x = ascend(x, mg, ng, step)
            if k == 0:
                stepped, grad_s = x, fwd + bwd
        if len(mine):
            fk, last_s = _evaluate(engine, x, world, chunk)
            refine_s += last_s
            best = np.maximum(best, np.where(fk > -1e19, fk, -np.inf))
    host_refine = time.perf_counter() - t0
    tot = shard.all_sum([len(mine), f0.sum(), best.sum(), (best > f0).sum(), busy, refine_s,
                         0.0 if first_equal else 1.0, last_s], world_size, group, device)
    n_el = max(tot[0], 1.0)
    report["sample_gpu_s"] = tot[4]
    report["elite_mean_fitness"] = tot[1] / n_el
    gain = (tot[2] - tot[1]) / n_el
    report["refine"] = dict(first_equal=bool(tot[6] == 0.0), gpu_s=float(tot[5]), mean_best=tot[2] / n_el, gain=gain,
                            gain_per_gpu_s=gain / tot[5], improved=tot[3] / n_el, host_s=host_refine)

    def resample_around(centres, budget, stream):
        """Rounds of children around `centres` (one child per elite a round)
        until `budget` GPU seconds are spent: (best per elite, seconds,
        rounds)."""
        bestr = f0.copy()
        secs = 0.0
        per = 0
        rounds = max(1, min(chunk, 1 << 19) // max(len(mine), 1))
        while len(mine) and secs < budget:
            n = rounds * len(mine)
            # A stream of its own for every arm, rank and batch.
            kids, parent = draw(centres, n, sigma, (seed + stream) * 10 ** 6 + rank * 10 ** 3 + per // rounds)
            # Children keep their elite's id, so they see its tremor phase.
            kids.genomes["id"] = elite.genomes["id"][parent]
            fk, busy_r = _evaluate(engine, kids, world, chunk)
            secs += busy_r
            per += rounds
            np.maximum.at(bestr, parent, np.where(fk > -1e19, fk, -np.inf).astype(np.float64))
        return bestr, secs, per

    if resample:
        t0 = time.perf_counter()
        bestr, secs, per = resample_around(elite, refine_s, 1)
        tr = shard.all_sum([bestr.sum(), (bestr > f0).sum(), secs, per], world_size, group, device)
        gain_r = (tr[0] - tot[1]) / n_el
        report["resample"] = dict(children_per_elite=tr[3] / world_size, gpu_s=tr[2], mean_best=tr[0] / n_el,
                                  gain=gain_r, gain_per_gpu_s=gain_r / tr[2], improved=tr[1] / n_el,
                                  host_s=time.perf_counter() - t0)
    if line_search and len(mine):
        t0 = time.perf_counter()
        xl, fl = elite, f0.astype(np.float64)
        bestl, secs = f0.copy(), 0.0
        for k in range(steps):
            wave = api.pack(xl, world)
            with engine.forward(wave, world) as tape:
                g = tape.backward()
                shape = tape.shape
                fwd, bwd = tape.seconds
            secs += fwd + bwd
            mg, ng = api.gene_gradients(xl, wave, world, g, shape)
            cands, fits = [], []
            for f in line_search:
                cand = ascend(xl, mg, ng, step * f)
                fc, busy_c = _evaluate(engine, cand, world, chunk)
                secs += busy_c
                cands.append(cand)
                fits.append(np.where(fc > -1e19, fc, -np.inf).astype(np.float64))
            fits = np.stack(fits)
            j = np.argmax(fits, axis=0)
            better = fits[j, np.arange(len(j))] > fl
            choice = np.where(better, j, -1)
            xl = pick(cands, choice, xl)
            fl = np.where(better, fits[j, np.arange(len(j))], fl)
            bestl = np.maximum(bestl, fl)
        tl = shard.all_sum([bestl.sum(), (bestl > f0).sum(), secs], world_size, group, device)
        gain_l = (tl[0] - tot[1]) / n_el
        report["line"] = dict(factors=list(line_search), gpu_s=tl[2], mean_best=tl[0] / n_el, gain=gain_l,
                              gain_per_gpu_s=gain_l / max(tl[2], 1e-12), improved=tl[1] / n_el,
                              host_s=time.perf_counter() - t0)
    if cma_samples and len(mine):
        report["cma"] = _cma_arm(engine, world, elite, f0, cma_samples, refine_s, seed, rank, chunk,
                                 (spec.friction_lo, spec.friction_hi))
        tc = shard.all_sum([report["cma"].pop("best_sum"), report["cma"]["improved"], report["cma"]["gpu_s"],
                            report["cma"]["generations"]], world_size, group, device)
        gain_c = (tc[0] - tot[1]) / n_el
        report["cma"].update(gpu_s=tc[2], mean_best=tc[0] / n_el, gain=gain_c,
                             gain_per_gpu_s=gain_c / max(tc[2], 1e-12), improved=tc[1] / n_el,
                             generations=tc[3] / world_size)
    if guided:
        t0 = time.perf_counter()
        if stepped is None:
            bestg, secs, per = f0.copy(), 0.0, 0
        else:
            bestg, secs, per = resample_around(stepped, refine_s - grad_s, 2)
        tg = shard.all_sum([bestg.sum(), (bestg > f0).sum(), secs + grad_s, per], world_size, group, device)
        gain_g = (tg[0] - tot[1]) / n_el
        report["guided"] = dict(children_per_elite=tg[3] / world_size, gpu_s=tg[2], mean_best=tg[0] / n_el,
                                gain=gain_g, gain_per_gpu_s=gain_g / max(tg[2], 1e-12), improved=tg[1] / n_el,
                                host_s=time.perf_counter() - t0)
    return report


def _cma_arm(engine, world, elite: api.Population, f0: np.ndarray, per: int, budget: float, seed: int, rank: int,
             chunk: int, friction) -> dict:
    """Generations of a CMA-ES optimizer per elite until `budget` GPU
    seconds are spent (evaluations, asks and tells); `friction` is the
    range repair holds frictions to (the workload's). Returns this rank's
    sum of best fitness, the count improved, GPU seconds and generations."""
    import torch
    from .cma import CmaEmitters
    t0 = time.perf_counter()
    opt = CmaEmitters(elite)
    E = len(elite)
    best = f0.astype(np.float64).copy()
    secs, gens, kernel_s = 0.0, 0, 0.0
    owner = np.arange(per * E) % E
    while secs < budget:
        genes, _ = opt.ask_device(per * E, seed=seed + 3, generation=gens, round=rank, first=0, friction=friction)
        kids = opt.download(genes)
        # Samples keep their elite's id, so they see its tremor phase.
        kids.genomes["id"] = elite.genomes["id"][owner]
        fk, busy = _evaluate(engine, kids, world, chunk)
        # The samples' genes are still on the device: tell reads them there.
        keys = torch.as_tensor(fk).to(opt.device)
        opt.tell_device(genes[:3] + genes[4:], keys, 0, per * E)
        ks = opt.kernel_seconds()
        secs += busy + ks
        kernel_s += ks
        gens += 1
        np.maximum.at(best, owner, np.where(fk > -1e19, fk, -np.inf).astype(np.float64))
    sig = opt.sigma.cpu().numpy()
    return dict(samples_per_generation=per, generations=gens, gpu_s=secs, ask_tell_gpu_s=kernel_s,
                best_sum=float(best.sum()),
                improved=float((best > f0).sum()), sigma_median=float(np.median(sig)),
                host_s=time.perf_counter() - t0)
