"""The CPU oracle against the golden vectors of the reference kernel.

tests/golden/*.npz hold packed populations, the reference kernel's results
and its recorded frames (made by tests/golden/make_golden.py from the
reference's own shaders/creature.cu on a B200). The CPU oracle
(oracle/creature_oracle.cpp) restates that kernel with IEEE division and
square root, the C library's cosine and arctangent and no fused
multiply-adds, so it agrees to a tolerance, not to the bit:
  * node positions within 2e-4 m over the first 10 steps and 2e-3 m over the
    first 30 (contact events make the difference grow later);
  * the same fall step for at least 90% of creatures, and a median relative
    fitness difference under 2e-3.
The packing of the stored populations must reproduce the stored records
byte for byte.
"""
from pathlib import Path

import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.api import Params, Population, WavePack
from oracle.ref import Oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    wave = WavePack(z["lanes"], z["muscles"], z["heads"], z["slots"], np.zeros((len(z["slots"]), 4), np.uint32))
    return z, wave, Params.from_buffer_copy(z["params"].tobytes()), int(z["flags"])


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def test_golden_cases_exist():
    assert set(CASES) >= {"calm_small", "calm_game", "effects", "every_effect"}


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("fp64", [False, True])
def test_oracle_tracks_reference_frames(oracle, name, fp64):
    z, wave, params, flags = load(name)
    settle = 100
    for c in range(len(z["frames"])):
        n = int(wave.heads[c, 0] & 255)
        res, trace = oracle.trace(wave, params, flags, c, 30, fp64=fp64)
        steps = int(np.array([res["ground_hi"]], np.float32).view(np.uint32)[0] >> 16)
        ref = z["frames"][c][settle + 1:settle + 31, :n]
        err = np.abs(trace[:, :n] - ref)
        k10, k30 = min(10, steps), min(30, steps)
        assert err[:k10].max(initial=0.0) < 2e-4, f"creature {c}: {err[:k10].max()} m in the first {k10} steps"
        assert err[:k30].max(initial=0.0) < 2e-3, f"creature {c}: {err[:k30].max()} m in the first {k30} steps"


@pytest.mark.parametrize("name", CASES)
def test_oracle_results_agree_with_reference(oracle, name):
    z, wave, params, flags = load(name)
    res, _ = oracle.run(wave, params, flags)
    ref = z["results"]
    assert (res["fall_time"] == ref["fall_time"]).mean() >= 0.9
    rel = np.abs(res["fitness"] - ref["fitness"]) / np.maximum(np.abs(ref["fitness"]), 1e-3)
    assert np.median(rel) < 2e-3
    # Fields the trajectory does not change stay equal: the rung trace's
    # step count of trials that end together.
    same = res["fall_time"] == ref["fall_time"]
    steps = lambda r: np.ascontiguousarray(r["ground_hi"]).view(np.uint32) >> 16  # noqa: E731
    assert (steps(res)[same] == steps(ref)[same]).all()


@pytest.mark.parametrize("name", CASES)
def test_packing_reproduces_golden_records(name):
    z, wave, _, _ = load(name)
    world = ce.make_world(**eval(str(z["world"][0])))
    pop = Population(z["nodes"], z["bones"], z["pop_muscles"], z["genomes"], z["strength"])
    again = ce.pack(pop, world)
    assert np.array_equal(again.lanes, z["lanes"])
    assert np.array_equal(again.muscles.view(np.uint32), z["muscles"].view(np.uint32))
    assert np.array_equal(again.heads, z["heads"])
    assert np.array_equal(again.slots, z["slots"])
