"""Converts the reference's test fixtures into this repository's gene arrays.

The reference's effect-sensitivity test (tests/cuda_effects.rs:21-48) scores
copies of a stored walker, tests/fixtures/warp_walker.json: a 6-node,
5-bone, 16-muscle creature whose muscles include touch sensors. This script
reads that JSON from the reference checkout (REFERENCE_DIR, else a checkout
called `reference` beside this repository) and writes its nodes, bones and
muscles with the engine's gene layouts (NODE_DTYPE, BONE_DTYPE,
MUSCLE_DTYPE) to tests/golden/fixtures/warp_walker.npz, which the GPU tests
load.

    python tests/golden/make_fixtures.py
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from evolution_simulator_gpu_b200 import api  # noqa: E402

OUT = Path(__file__).resolve().parent / "fixtures"
REFERENCE = Path(os.environ.get("REFERENCE_DIR") or ROOT.parent / "reference")


def convert(name: str) -> Path:
    data = json.loads((REFERENCE / "tests" / "fixtures" / f"{name}.json").read_text())
    nodes = np.zeros(len(data["nodes"]), api.NODE_DTYPE)
    for i, n in enumerate(data["nodes"]):
        nodes[i] = (n["x"], n["y"], n["diameter"], n["friction"])
    bones = np.zeros(len(data["bones"]), api.BONE_DTYPE)
    for i, b in enumerate(data["bones"]):
        bones[i] = (b["a"], b["b"], b["rest_length"], b["min_angle"], b["max_angle"], b["organ_mass"],
                    b["organ_at"])
    muscles = np.zeros(len(data["muscles"]), api.MUSCLE_DTYPE)
    for i, m in enumerate(data["muscles"]):
        muscles[i] = (m["bone_a"], m["bone_b"], m["anchor_a"], m["anchor_b"], m["short"], m["long"], m["period"],
                      m["phase"], m["duty"], m["stiffness"], m["sensor"], m["reset"], m["tendon"])
    OUT.mkdir(exist_ok=True)
    out = OUT / f"{name}.npz"
    np.savez_compressed(out, nodes=nodes, bones=bones, muscles=muscles, id=np.uint64(data["id"]))
    return out


if __name__ == "__main__":
    print(convert("warp_walker"))
