"""Test infrastructure: counts the algorithmic FP32 operations of a creature
substep, the numerator of the creature kernel's roofline.

The CPU oracle runs sample creatures of each workload with a scalar type that
counts every floating-point operation (add/subtract, multiply, divide, square
root, cosine and arctangent, min/max, compare, floor/abs/copysign), and the
counts are divided by the substeps the trials ran. The result is written to
profiles/op_counts.json, which the benchmark reads.

    python oracle/count_ops.py [--sample 256]
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import evolution_simulator_gpu_b200 as ce  # noqa: E402
from evolution_simulator_gpu_b200.configs import WORKLOADS  # noqa: E402
from oracle.ref import Oracle  # noqa: E402

KINDS = ["add", "mul", "div", "sqrt", "transcendental", "minmax", "compare", "other"]


def count_workload(name: str, sample: int) -> dict:
    w = WORKLOADS[name]
    world = w.world()
    pop = ce.generate(w.spec, sample)
    wave = ce.pack(pop, world)
    params = ce.make_params(world)
    flags = ce.world_flags(world)
    oracle = Oracle()
    totals = np.zeros(8, np.float64)
    substeps = 0
    for c in range(len(wave)):
        res, counts = oracle.count(wave, params, flags, c, world.rate or 60)
        steps = int(np.array([res["ground_hi"]], np.float32).view(np.uint32)[0] >> 16)  # steps run
        substeps += 16 * steps
        totals += counts
    per = totals / max(substeps, 1)
    return {"sample": sample, "substeps": substeps, "ops_per_substep": float(per.sum()),
            "by_kind": {k: float(v) for k, v in zip(KINDS, per)},
            "flops_per_substep": float(per[:5].sum() + per[7])}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--sample", type=int, default=256)
    args = ap.parse_args()
    out = {name: count_workload(name, args.sample) for name in ["small", "game", "effects", "gradients"]}
    path = ROOT / "profiles" / "op_counts.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
