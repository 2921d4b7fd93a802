"""Builds the engine library, libcreature_engine.so, in this package's folder.

The CUDA sources are compiled ahead of time for sm_100a only. The float
flags are those the reference passes to NVRTC for its kernel
(src/cuda_engine.rs:1450-1466): approximate division and square root,
contracted multiply-adds. The host model is built without contraction so its
single-precision arithmetic rounds like the reference's Rust host.

    python -m evolution_simulator_gpu_b200.build [--force] [-v]
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
CSRC = HERE / "csrc"
OUT = HERE / "libcreature_engine.so"
OBJ = HERE / "_build"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--prec-div=false", "--prec-sqrt=false", "--fmad=true",
    "-extra-device-vectorization", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
    # A host-only function called from device code has no device body: an
    # error, not a warning (the call would be undefined on the GPU).
    "-Werror", "cross-execution-space-call",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fopenmp"]

CUDA_SOURCES = ["advance.cu", "adjoint.cu", "bucket.cu", "engine.cu", "metrics.cu", "peak.cu", "noalloc.cu",
                "sample.cu", "pack.cu", "cma.cu", "audit.cu"]
# The device packer, gene gradients and ascent step, the CMA-ES emitters and
# the rung audit's sums round as their host counterparts: IEEE division and
# square root, no contraction of multiply-adds.
IEEE_SOURCES = {"pack.cu", "cma.cu", "audit.cu"}


def file_flags(name: str) -> list[str]:
    if name not in IEEE_SOURCES:
        return NVCC_FLAGS
    swap = {"--prec-div=false": "--prec-div=true", "--prec-sqrt=false": "--prec-sqrt=true", "--fmad=true": "--fmad=false"}
    return [swap.get(f, f) for f in NVCC_FLAGS]
CXX_SOURCES = ["host_model.cpp", "generator.cpp"]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the engine needs the CUDA toolkit to build")
    return found


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    return obj.stat().st_mtime < newest


def _run(cmd: list[str], log: Path) -> str:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    text = proc.stdout + proc.stderr
    log.write_text(text)
    if proc.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{text[-6000:]}")
    return text


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for name in CUDA_SOURCES:
        src, obj = CSRC / name, OBJ / (name + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append(([nvcc(), *ARCH, *file_flags(name), "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)],
                         OBJ / (name + ".log")))
    for name in CXX_SOURCES:
        src, obj = CSRC / name, OBJ / (name + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append((["g++", *CXX_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)],
                         OBJ / (name + ".log")))
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as pool:
            outs = list(pool.map(lambda j: _run(*j), jobs))
        if verbose:
            for o in outs:
                sys.stdout.write(o)
    if jobs or not OUT.exists():
        tmp = OUT.with_suffix(".so.tmp")
        _run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp", "-Xlinker", "-Bsymbolic"],
             OBJ / "link.log")
        os.replace(tmp, OUT)
    return OUT


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()
