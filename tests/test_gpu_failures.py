"""Failure paths of the engine, made on the host (no GPU fault).

The reference's scheduler recovers a failed GPU by reopening its engine and
submitting the unfinished units again with their exact inputs, which gives
the same results (src/scheduler.rs:725-806); out-of-memory submissions are
retried after idle buffers are freed (MemoryBackoff, src/engine.rs:534-650);
a poll that finds nothing finished in time is not an error. Here:

* ce_inject_fault makes the chosen submission fail with the chosen status
  (the device-lost and out-of-memory statuses), nothing is queued for it,
  and the engine then takes a fresh submission of the same batch whose
  results equal the first run's to the bit;
* ce_poll and ce_wait with a short timeout return CE_ERR_TIMEOUT while a
  batch still runs, and the batch's results come back on a later poll;
* a poll into a result buffer that is too small fails without losing the
  submission;
* an engine closed with work in flight and opened again gives the same
  results for the same batch (the reopen-and-resubmit path).
"""
import ctypes as C

import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(scope="module")
def batch():
    w = WORKLOADS["game"]
    world = w.world(duration=2.0)
    return world, ce.pack(ce.generate(w.spec, 4096), world)


@pytest.mark.parametrize("status", [ce.CE_ERR_DEVICE, ce.CE_ERR_OOM])
def test_injected_fault_fails_one_submission_then_the_engine_recovers(batch, status):
    world, wave = batch
    with ce.Engine(0) as eng:
        first, _ = eng.run(wave, world)
        eng.inject_fault(2, status)
        t1 = eng.submit(wave, world)  # the first submission after arming goes through
        with pytest.raises(ce.EngineError) as err:
            eng.submit(wave, world)
        assert err.value.status == status
        assert err.value.out_of_memory == (status == ce.CE_ERR_OOM)
        assert b"injected" in ce.lib().ce_last_error()
        got = eng.poll(600.0)
        assert got is not None and got[0] == t1
        assert eng.poll(0.0) is None, "the failed submission left nothing in flight"
        if status == ce.CE_ERR_OOM:
            eng.release_idle()  # what the reference's backoff does before a retry
        again, _ = eng.run(wave, world)
    assert (bits(got[1]) == bits(first)).all()
    assert (bits(again) == bits(first)).all()


def test_poll_and_wait_time_out_while_a_batch_runs(batch):
    world, _ = batch
    w = WORKLOADS["game"]
    long_world = w.world(duration=20.0)
    wave = ce.pack(ce.generate(w.spec, 300_000), long_world)
    with ce.Engine(0) as eng:
        assert eng.poll(0.0) is None, "nothing in flight"
        t = eng.submit(wave, long_world)
        # 300,000 creatures x 20 s take hundreds of milliseconds on a B200.
        assert eng.poll(0.0) is None
        assert eng.wait(0.0) is False
        st = ce.lib().ce_wait(eng.handle, 1000)
        assert st == ce.CE_ERR_TIMEOUT
        assert eng.wait(600.0) is True
        got = eng.poll(600.0)
        assert got is not None and got[0] == t and len(got[1]) == len(wave)
        assert eng.free_slots() == 4


def test_poll_into_a_small_buffer_keeps_the_submission(batch):
    world, wave = batch
    with ce.Engine(0) as eng:
        t = eng.submit(wave, world)
        assert eng.wait(600.0)
        small = np.zeros(len(wave) - 1, ce.RESULT_DTYPE)
        tk, n, busy = C.c_uint64(), C.c_size_t(), C.c_double()
        st = ce.lib().ce_poll(eng.handle, 0, C.byref(tk), small.ctypes.data, len(small), C.byref(n), C.byref(busy))
        assert st == ce.CE_ERR_INVALID
        assert b"too small" in ce.lib().ce_last_error()
        got = eng.poll(0.0)
        assert got is not None and got[0] == t and len(got[1]) == len(wave)


def test_reopened_engine_gives_the_same_results(batch):
    world, wave = batch
    eng = ce.Engine(0)
    first, _ = eng.run(wave, world)
    eng.submit(wave, world)
    eng.submit(wave, world)
    eng.close()  # with two submissions in flight: the close waits for them and frees everything
    with ce.Engine(0) as eng2:
        again, _ = eng2.run(wave, world)
    assert (bits(again) == bits(first)).all()
