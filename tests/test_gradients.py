"""Host-side checks of the gradient path: the gene chain rule and the FP64
dual-number tangent of the CPU oracle. No GPU is used.

* `ce_gene_gradients` maps record-field gradients (muscle fields, node
  friction, mass and start position) to gene gradients through the packing
  arithmetic
  (src/physics2.rs:190-350, src/physics.rs:203-296, src/kernel.rs:336-411).
  For random record gradients g and a random gene direction v it must give
  <g_gene, v> = <g, d records / d genes . v>, the right side taken by central
  differences of the packer.
* The oracle's FP64 tangent (forward-mode dual numbers through the restated
  kernel, shaders/creature.cu:130-742) must equal central differences of the
  FP64 oracle over trials short enough that the perturbation keeps every
  contact, friction and joint-limit mode.
"""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

# Record float index of each gradient field of a muscle (kernel record layout).
FIELDS = [8, 3, 4, 5, 10, 11, 12, 13, 14]


def _direction(pop, rng):
    """A gene direction (muscle genes x 5, node genes), zero where the chain
    rule has a kink: duty at its clamp, phase near its wrap."""
    vm = rng.normal(size=(len(pop.muscles), 5))
    vn = rng.normal(size=len(pop.nodes))
    duty = pop.muscles["duty"]
    phase = pop.muscles["phase"]
    bad = (duty <= 0.0501) | (duty >= 0.9499) | (phase < 0.01) | (phase > 0.99)
    vm[bad, 3:] = 0.0
    return vm, vn


def _moved(pop, vm, vn, h):
    m = pop.muscles.copy()
    n = pop.nodes.copy()
    T = m["period"].astype(np.float64)
    m["short"] = (m["short"] + h * vm[:, 0]).astype(np.float32)
    m["long"] = (m["long"] + h * vm[:, 1]).astype(np.float32)
    m["phase"] = (m["phase"] - h * vm[:, 3] / T).astype(np.float32)
    m["duty"] = (m["duty"] + h * (vm[:, 4] - vm[:, 3]) / T).astype(np.float32)
    n["friction"] = (n["friction"] + h * vn).astype(np.float32)
    strength = None if pop.strength is None else (pop.strength + h * vm[:, 2]).astype(np.float32)
    return ce.Population(n, pop.bones, m, pop.genomes, strength)


@pytest.mark.parametrize("workload,part", [("gradients", "all"), ("refine", "all"), ("gradients", "start"),
                                           ("refine", "start")])
def test_gene_chain_rule_matches_packer_differences(workload, part):
    """In the calm world and in the refined-search world (rough ground with
    hurdles, tremors and the other effects), where the start pose is also
    lowered onto the ground under its lowest node; `start` puts the record
    gradient on the start positions alone (the pose's shifts)."""
    w = WORKLOADS[workload]
    world = w.world(duration=1.0)
    pop = ce.generate(w.spec, 48)
    assert pop.strength is not None
    wave = ce.pack(pop, world)
    rows, mm = int((wave.heads[:, 0] & 255).max()), int(wave.heads[:, 1].max())
    rng = np.random.default_rng(0)
    g = rng.normal(size=(len(wave), 9 * mm + 4 * rows)).astype(np.float32)
    if part == "start":
        g[:, :9 * mm + 2 * rows] = 0.0
    mg, ng = ce.gene_gradients(pop, wave, world, g, (rows, mm))
    vm, vn = _direction(pop, rng)
    h = 1e-3
    wp, wm = ce.pack(_moved(pop, vm, vn, h), world), ce.pack(_moved(pop, vm, vn, -h), world)
    assert (wp.slots == wave.slots).all() and (wm.slots == wave.slots).all()

    def record_change(wa, wb, c):
        """<g_c, records(wa) - records(wb)> of creature c."""
        la, lb = wa.lanes.view(np.float32), wb.lanes.view(np.float32)
        M, N = int(wave.heads[c, 1]), int(wave.heads[c, 0] & 255)
        mo, ro = int(wave.heads[c, 4]), int(wave.heads[c, 3])
        out = 0.0
        for k in range(M):
            for f, fi in enumerate(FIELDS):
                out += float(g[c, 9 * k + f]) * (float(wa.muscles[mo + 20 * k + fi]) -
                                                 float(wb.muscles[mo + 20 * k + fi]))
        for i in range(N):
            out += float(g[c, 9 * mm + i]) * (float(la[ro + 6 * i + 2]) - float(lb[ro + 6 * i + 2]))
            out += float(g[c, 9 * mm + rows + i]) * (float(la[ro + 6 * i]) - float(lb[ro + 6 * i]))
            for axis in range(2):
                out += float(g[c, 9 * mm + 2 * rows + 2 * i + axis]) * (float(la[ro + 6 * i + 3 + axis]) -
                                                                        float(lb[ro + 6 * i + 3 + axis]))
        return out

    # Central differences over all creatures; for the start positions alone,
    # which are piecewise linear in the genes, only creatures where the
    # packer has no kink within [-h, h] along the direction (its one-sided
    # differences agree: no muscle's length crosses its span, no other node
    # becomes the lowest).
    lhs = rhs = 0.0
    kept = 0
    for c in range(len(wave)):
        up, down = record_change(wp, wave, c) / h, record_change(wave, wm, c) / h
        if part == "start" and abs(up - down) > 0.02 * max(abs(up), abs(down)) + 1e-4:
            continue
        kept += 1
        gs = pop.genomes[int(wave.slots[c])]
        ms, ns = slice(gs["muscle_start"], gs["muscle_start"] + gs["muscle_count"]), slice(
            gs["node_start"], gs["node_start"] + gs["node_count"])
        lhs += 0.5 * (up + down)
        rhs += float((mg[ms] * vm[ms]).sum() + (ng[ns] * vn[ns]).sum())
    assert kept >= 0.8 * len(wave), kept
    assert abs(lhs - rhs) <= 2e-3 * max(abs(rhs), 1.0), (lhs, rhs)


@pytest.mark.parametrize("workload,field", [("gradients", f) for f in range(13)] +
                         [("refine", f) for f in (0, 2, 4, 8, 9, 10, 11, 12)])
def test_fp64_tangent_matches_fp64_differences(workload, field):
    """One record field of muscle 0 (field < 9), the friction of node 1
    (field 9), the mass of node 1 (field 10, with 1 / total mass moving
    along) or the start x or y of node 1 (fields 11, 12) of 8 creatures,
    0.2 s trials, in the calm world and in the refined-search world (rough
    ground, hurdles, tremors, water, ice, wind, thick air)."""
    from oracle.ref import Oracle
    o = Oracle()
    w = WORKLOADS[workload]
    world = w.world(duration=0.2)
    pop = ce.generate(w.spec, 8)
    wave = ce.pack(pop, world)
    p, flags = ce.make_params(world), ce.world_flags(world)
    rows, mm = int((wave.heads[:, 0] & 255).max()), int(wave.heads[:, 1].max())
    n = len(wave)
    dm = np.zeros((n, mm, 9))
    dn = np.zeros((n, rows))
    dmass = np.zeros((n, rows))
    dstart = np.zeros((n, rows, 2))
    lf = wave.lanes.view(np.float32)
    for c in range(n):
        mo, ro = int(wave.heads[c, 4]), int(wave.heads[c, 3])
        if field < 9:
            dm[c, 0, field] = wave.muscles[mo + FIELDS[field]]
        elif field == 9:
            dn[c, 1] = lf[ro + 6 + 2]
        elif field == 10:
            dmass[c, 1] = lf[ro + 6]
        else:
            dstart[c, 1, field - 11] = 1.0
    tangent, _, _ = o.tangent(wave, p, flags, dm, dn, dmass=dmass, dstart=dstart)

    def run(eps):
        mus = wave.muscles.copy()
        lanes = wave.lanes.copy()
        heads = wave.heads.copy()
        lf2 = lanes.view(np.float32)
        for c in range(n):
            mo, ro = int(wave.heads[c, 4]), int(wave.heads[c, 3])
            if field < 9:
                mus[mo + FIELDS[field]] = np.float32(wave.muscles[mo + FIELDS[field]] * (1 + eps))
            elif field == 9:
                lf2[ro + 6 + 2] = np.float32(lf[ro + 6 + 2] * (1 + eps))
            elif field > 10:
                lf2[ro + 6 + 3 + field - 11] = np.float32(lf[ro + 6 + 3 + field - 11] + eps)
            else:
                dmass_c = float(lf[ro + 6]) * eps
                lf2[ro + 6] = np.float32(lf[ro + 6] + dmass_c)
                inv = np.float32(1.0 / (1.0 / float(np.uint32(wave.heads[c, 6]).view(np.float32)) + dmass_c))
                heads[c, 6] = inv.view(np.uint32)
        o.tangent(ce.WavePack(lanes, mus, heads, wave.slots, wave.info), p, flags, np.zeros_like(dm),
                  np.zeros_like(dn))
        return o.fitness64.copy()

    # A start position moves by an absolute 2^-20 m (exact in float32 for
    # positions below 8 m: the start pose rests a node exactly on the ground,
    # so larger moves change its contact mode), the other fields by 1e-3
    # relative.
    h = 2.0 ** -20 if field > 10 else 1e-3
    f0, fp, fm = run(0.0), run(h), run(-h)
    fd = (fp - fm) / (2 * h)
    # Mode-preserving perturbations only: the one-sided differences agree
    # (a perturbation that crosses a contact, friction, joint-limit or rhythm
    # branch shows as a jump between them).
    up, down = (fp - f0) / h, (f0 - fm) / h
    keep = np.abs(up - down) <= 0.05 * np.maximum(np.abs(up), np.abs(down)) + 1e-9
    assert keep.sum() >= n // 2, keep
    scale = max(np.abs(fd[keep]).max(), 1e-9)
    assert np.allclose(tangent[keep], fd[keep], rtol=2e-2, atol=2e-2 * scale), (tangent, fd, keep)
