"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a B200 and run the engine's CUDA kernels (and, as
the checker, the reference kernel built under oracle/_ref). The rest run on
the CPU: the host model, the CPU oracle against the golden vectors, the C ABI
exports and the multi-process host logic.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU")
    # A fresh checkout has no built libraries: build the engine and the
    # checkers (the reference kernel only where the reference checkout is).
    from evolution_simulator_gpu_b200 import api
    if not api.LIB_PATH.exists():
        from evolution_simulator_gpu_b200.build import build
        build()
    if not (ROOT / "oracle" / "_ref" / "liboracle.so").exists():
        from oracle.build_ref import build as build_checkers
        build_checkers()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def engine():
    if not gpu_available():
        pytest.skip("no GPU")
    import evolution_simulator_gpu_b200 as ce
    e = ce.Engine(0)
    yield e
    e.close()
