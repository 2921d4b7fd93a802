"""The rung audit on the device (ce_audit_device) against its restatement
(oracle/audit_ref.py): Audit::note's tallies, the audit rows and every
float64 sum of GenAudit::of equal to the bit, and class A's feature words
equal word for word; on random trace words (non-finite halves, empty traces
and exempt rows included) and on the results of real trials."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import api
from evolution_simulator_gpu_b200.configs import WORKLOADS
from oracle import audit_ref as A

pytestmark = pytest.mark.gpu


def periods_of(pop):
    g = pop.genomes
    has = g["muscle_count"] > 0
    out = np.zeros(len(pop), np.float32)
    out[has] = pop.muscles["period"][g["muscle_start"][has]]
    return out


def check(res, pop, bars):
    got = api.audit(res, pop, bars)
    flags = pop.genomes["flags"]
    n, steps, stops = A.note(res)
    rows, sums, a_rows = A.gen_audit(res, flags, periods_of(pop), bars)
    assert (got["creatures"], got["steps"], got["stops"], got["rows"]) == (n, steps, stops, rows)
    for r in range(2):
        for k in range(2):
            gn, gs, gx = got["sums"][r][k]
            wn, ws, wx = sums[r][k]
            assert gn == wn, (r, k)
            assert gs == ws, (r, k)          # float64, bit for bit
            assert gx == wx, (r, k)
        assert (got["a_words"][r] == a_rows[r]).all()
    return got


def test_audit_of_random_traces(engine):
    rng = np.random.default_rng(3)
    count = 60_000
    pop = ce.generate(WORKLOADS["game"].spec, count)
    words = rng.integers(0, 1 << 32, size=(count, 7), dtype=np.uint64).astype(np.uint32)
    # Mostly finite halves (exponent field below 31), a few infinities and NaNs.
    finite = rng.random((count, 7)) < 0.98
    words[finite] &= np.uint32(0x7bff7bff)
    steps = rng.integers(0, 1300, count).astype(np.uint32)
    steps[rng.random(count) < 0.05] = 0
    words[:, 2] = (words[:, 2] & 0xffff) | (steps << 16)
    res = np.zeros(count, ce.RESULT_DTYPE)
    for k, f in enumerate(A.TRACE_FIELDS):
        res[f] = words[:, k].view(np.float32)
    res["screen_x"] = rng.normal(2.0, 1.5, count).astype(np.float32)
    res["screened"] = np.where(rng.random(count) < 0.4, rng.uniform(1, 5, count), 0).astype(np.float32)
    flags = np.where(rng.random(count) < 0.2, A.AUDIT, 0) | np.where(rng.random(count) < 0.1, A.EXEMPT, 0)
    pop.genomes["flags"] = flags.astype(np.uint32)
    bars = rng.normal(2.0, 0.5, count).astype(np.float32)
    bars[rng.random(count) < 0.05] = np.nan
    got = check(res, pop, bars)
    assert got["rows"] > 10_000 and got["sums"][1][0][0] > 1000 and got["sums"][0][1][0] > 1000


def test_audit_of_real_trials(engine):
    w = WORKLOADS["effects"]
    pop = ce.generate(w.spec, 8192)
    pop.genomes["flags"] = np.where(np.arange(8192) % 8 == 0, A.AUDIT, 0).astype(np.uint32)
    res = ce.evaluate(engine, pop, w.world())
    bars = np.full(8192, np.float32(np.median(res["screen_x"])), np.float32)
    got = check(res, pop, bars)
    assert got["rows"] >= 1000  # one creature in 8, nearly all with a trace
    assert got["sums"][0][0][0] > 0 and got["sums"][0][1][0] > 0


def test_audit_of_an_empty_batch(engine):
    pop = ce.generate(WORKLOADS["game"].spec, 1)
    res = np.zeros(0, ce.RESULT_DTYPE)
    got = api.audit(res, api.Population(pop.nodes, pop.bones, pop.muscles, pop.genomes[:0], pop.strength),
                    np.zeros(0, np.float32))
    assert got["creatures"] == 0 and got["rows"] == 0 and got["sums"][0][0][0] == 0


def test_audit_words_stop_at_the_callers_capacity(engine):
    # Class A's feature words go to the first a_cap rows only (here fewer
    # than one chunk of 256 rows holds, and more than one); the sums count
    # every row.
    rng = np.random.default_rng(4)
    count = 20_000
    pop = ce.generate(WORKLOADS["game"].spec, count)
    words = rng.integers(0, 1 << 32, size=(count, 7), dtype=np.uint64).astype(np.uint32) & np.uint32(0x7bff7bff)
    words[:, 2] = (words[:, 2] & 0xffff) | (rng.integers(200, 1300, count).astype(np.uint32) << 16)
    res = np.zeros(count, ce.RESULT_DTYPE)
    for k, f in enumerate(A.TRACE_FIELDS):
        res[f] = words[:, k].view(np.float32)
    res["screen_x"] = rng.normal(2.0, 1.0, count).astype(np.float32)
    pop.genomes["flags"] = np.where(rng.random(count) < 0.1, A.AUDIT, 0).astype(np.uint32)
    bars = np.full(count, 1.5, np.float32)
    _, sums, a_rows = A.gen_audit(res, pop.genomes["flags"], periods_of(pop), bars)
    assert len(a_rows[0]) > 600
    for cap in (37, 300):
        got = api.audit(res, pop, bars, a_cap=cap)
        for r in range(2):
            assert got["sums"][r][0][0] == sums[r][0][0]
            assert (got["a_words"][r] == a_rows[r][:cap]).all() and len(got["a_words"][r]) == cap
