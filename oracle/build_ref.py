"""Test infrastructure: builds the reference kernel and the CPU oracle.

1. The reference kernel, from the reference's own source where it lies
   (shaders/creature.cu under the reference checkout), compiled ahead of
   time for sm_100a with the float options the reference passes to NVRTC
   (src/cuda_engine.rs:1450-1466) and the #define prelude its host writes
   (src/kernel.rs:268-332), one shared library per (world, step rate,
   recording) into oracle/_ref/. The reference's Rust host cannot be built
   here (no Rust toolchain); the launcher is oracle/ref_launch.cu.
2. The CPU oracle (oracle/creature_oracle.cpp) into oracle/_ref/liboracle.so.

    python oracle/build_ref.py [--reference PATH] [--force]

The reference checkout is found at --reference, else at the directory the
REFERENCE_DIR environment variable names, else at a checkout called
`reference` beside this repository's folder.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_REFERENCE = Path(os.environ.get("REFERENCE_DIR") or HERE.parent.parent / "reference")

FLAG_NAMES = ["GROUND", "TERRAIN", "SLOPE", "GAPS", "HURDLES", "QUAKE", "MUD", "WATER", "ICE", "WIND", "AIR",
              "BRAMBLES"]
# Worlds the tests and the benchmark compare on: calm, effects, effects with
# quakes, every effect.
WORLDS = [0x001, 0x797, 0x7B7, 0xFFF]
VARIANTS = [(f, 60, r) for f in WORLDS for r in (0, 1)] + [(0x001, 120, 0), (0x001, 120, 1)]

# The constants of the prelude, written as the reference's host writes them
# (Rust's shortest round-trip float text plus "f").
CONSTANTS = [
    ("MUSCLE_RECOVERY", "0.5f"), ("INV_JOINT_DAMPING", "10.0f"), ("JOINT_BREAK", "0.5f"),
    ("MUD_NORMAL", "2.0f"), ("MUD_GRIP", "2.0f"), ("MUD_DRAG", "2.0f"), ("MUD_FULL_DEPTH", "0.1f"),
    ("BRAMBLE_REACH", "0.01f"), ("AIR_DRAG", "0.6f"), ("WATER_DRAG", "100.0f"), ("WATER_ALONG", "0.25f"),
    ("WATER_BUOYANCY", "0.7f"), ("ICE_INV", "0.16666667f"), ("HEAD_SHAKE_LIMIT", "78.4f"),
    ("HEAD_SHAKE_WINDOW", "0.1f"), ("CONTACT_SLACK", "0.002f"), ("LIFT_CLEARANCE", "0.01f"),
    ("GAP_DEPTH", "2.0f"), ("GAP_RUN", "0.15f"), ("HURDLE_SPACING", "3.0f"), ("HURDLE_TOP", "1.2f"),
    ("HURDLE_RUN", "0.2f"),
]


def variant_name(flags: int, rate: int, record: int) -> str:
    return f"libref_{flags:03x}_{rate}_{record}.so"


def prelude(flags: int, rate: int, record: int) -> str:
    settle = (200 * rate + 119) // 120
    sample = max(rate // 30, 1)
    lines = [
        ("RATE", f"{rate:.1f}f"), ("SUBSTEPS", "16u"), ("SETTLE", f"{settle}u"), ("SAMPLE", f"{sample}u"),
        ("MAXN", "32u"), ("MAXM", "96u"), ("BLOCK", "128u"), ("MIN_BLOCKS", "3"), ("RECORD", str(record)),
    ]
    lines += [(name, "1" if flags >> bit & 1 else "0") for bit, name in enumerate(FLAG_NAMES)]
    lines += CONSTANTS
    return "".join(f"#define {k} {v}\n" for k, v in lines)


def nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


# The reference kernel's host stub is an extern "C" function called `advance`,
# a name the C library also exports (the old <regexp.h> advance); -Bsymbolic
# binds the launcher's launch to the stub in its own library.
def build_variant(reference: Path, flags: int, rate: int, record: int, force: bool) -> Path:
    out = OUT / variant_name(flags, rate, record)
    src = reference / "shaders" / "creature.cu"
    if out.exists() and not force and out.stat().st_mtime > max(src.stat().st_mtime,
                                                               (HERE / "ref_launch.cu").stat().st_mtime):
        return out
    pre = OUT / f"prelude_{flags:03x}_{rate}_{record}.h"
    pre.write_text(prelude(flags, rate, record))
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3", "--prec-div=false",
           "--prec-sqrt=false", "--fmad=true", "-extra-device-vectorization", "-Xcompiler", "-fPIC", "-shared", "-Xlinker", "-Bsymbolic",
           "-include", str(pre), f'-DREF_SOURCE="{src}"', str(HERE / "ref_launch.cu"), "-o", str(out)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"reference kernel build failed:\n{proc.stdout}{proc.stderr}")
    return out


def build_oracle(force: bool) -> Path:
    out = OUT / "liboracle.so"
    src = HERE / "creature_oracle.cpp"
    deps = [src, HERE / "creature_oracle.hpp"]
    if out.exists() and not force and out.stat().st_mtime > max(d.stat().st_mtime for d in deps if d.exists()):
        return out
    cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-march=x86-64-v2",
           str(src), "-o", str(out)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{proc.stdout}{proc.stderr}")
    return out


def build(reference: Path = DEFAULT_REFERENCE, force: bool = False) -> list[Path]:
    OUT.mkdir(exist_ok=True)
    built = []
    if (HERE / "creature_oracle.cpp").exists():
        built.append(build_oracle(force))
    if not (reference / "shaders" / "creature.cu").exists():
        # The reference checkout is not on this machine (the GPU box): the
        # libraries built next to it travel with the repository.
        return built
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        built += list(pool.map(lambda v: build_variant(reference, *v, force), VARIANTS))
    return built


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    for p in build(args.reference, args.force):
        print(p)


if __name__ == "__main__":
    sys.exit(main())
