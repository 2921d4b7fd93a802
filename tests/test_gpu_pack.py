"""The device packer (ce_pack_plan + ce_pack_device) against the host packer
(ce_pack), byte for byte: every record word, muscle record and head word, on
the game workload (3,000,000 creatures), the effects workload (3,000,000,
rough ground with hurdles: the start pose is lowered onto uneven ground) and
the refined-search world with tremors (200,000 creatures, each muscle's
strength scaled), whose quake phases and amplitudes enter the start pose.

The host packer restates the reference's host packing (physics2::Model::new,
start, kernel::fill_creature, pack_reusing); the device packer runs the same
arithmetic (csrc/packer.h) with IEEE division and square root and no fused
multiply-adds, and takes the C library's arctangent, sine and cosine from the
host's plan.
"""
import ctypes as C

import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import api
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def device_pack(pop, world):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    plan = ce.pack_plan(pop, world)

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).to(dev)

    d_nodes, d_bones, d_muscles, d_genomes = up(pop.nodes), up(pop.bones), up(pop.muscles), up(pop.genomes)
    d_strength = up(pop.strength) if pop.strength is not None else None
    dev_pop = api.PopulationC(d_nodes.data_ptr(), d_bones.data_ptr(), d_muscles.data_ptr(), d_genomes.data_ptr(),
                              len(pop), d_strength.data_ptr() if d_strength is not None else None)
    d_trig, d_order, d_rat, d_mat = up(plan.trig), up(plan.order), up(plan.record_at), up(plan.muscle_at)
    n = len(plan.order)
    d_lanes = torch.zeros(plan.lanes_len, dtype=torch.int32, device=dev)
    d_mus = torch.zeros(plan.muscles_len, dtype=torch.float32, device=dev)
    d_heads = torch.zeros(8 * n, dtype=torch.int32, device=dev)
    ce.pack_device(dev_pop, d_trig.data_ptr(), d_order.data_ptr(), d_rat.data_ptr(), d_mat.data_ptr(), n, world,
                   d_lanes.data_ptr(), d_mus.data_ptr(), d_heads.data_ptr(),
                   torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    return (plan, d_lanes.cpu().numpy().view(np.uint32), d_mus.cpu().numpy().view(np.uint32),
            d_heads.cpu().numpy().view(np.uint32).reshape(n, 8))


@pytest.mark.parametrize("name,count,strength", [("game", 3_000_000, False), ("effects", 3_000_000, False),
                                                 ("refine", 200_000, True)])
def test_device_packing_equals_host_packing(name, count, strength):
    w = WORKLOADS[name]
    world = w.world()
    pop = ce.generate(w.spec, count)
    if strength:
        rng = np.random.default_rng(5)
        pop.strength = rng.uniform(0.5, 1.5, len(pop.muscles)).astype(np.float32)
    wave = ce.pack(pop, world)
    plan, lanes, muscles, heads = device_pack(pop, world)
    assert (plan.order == wave.slots).all()
    assert len(lanes) == len(wave.lanes) and len(muscles) == len(wave.muscles)
    rows, cols = np.nonzero(heads != wave.heads)
    assert len(rows) == 0, (f"{len(np.unique(rows))} heads differ in words {np.unique(cols)}; first "
                            f"{rows[:2]}: device {heads[rows[0]]} host {wave.heads[rows[0]]}")
    bad = np.nonzero(lanes != wave.lanes)[0]
    assert len(bad) == 0, f"{len(bad)} record words differ, first at {bad[:4]}"
    bad = np.nonzero(muscles != wave.muscles.view(np.uint32))[0]
    assert len(bad) == 0, f"{len(bad)} muscle words differ, first at {bad[:4]}"
