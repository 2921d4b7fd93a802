"""The restatement of the rung audit (oracle/audit_ref.py) on traces built
the way the reference's rung tests build them (src/rungs/tests.rs:14-55):
the features it reads, which trials are audit rows, which rows each rung's
classes take, and Audit::note's tallies. No GPU call is made."""
import numpy as np

import evolution_simulator_gpu_b200 as ce
from oracle import audit_ref as A


def h(v):
    return int(np.float32(v).astype(np.float16).view(np.uint16))


def pair(lo, hi):
    return h(lo) | h(hi) << 16


def trace_words(d60, d150, d300, steps, bands=(0, 0), code=0):
    """The reference tests' `trace`: speed equals distance at each rung,
    every node touched, energy 0.5, head shake 1.0."""
    c = bands[0] << 8 | bands[1] << 11 | code
    return [pair(d60, d150), pair(d300, d300), c | steps << 16, pair(d60, d150), pair(1.0, 0.5), pair(1.0, 0.5),
            pair(1.0, 1.0)]


def results_of(words, screen_x=None, screened=None):
    r = np.zeros(len(words), ce.RESULT_DTYPE)
    w = np.array(words, np.uint32).reshape(-1, 7)
    for k, f in enumerate(A.TRACE_FIELDS):
        r[f] = w[:, k].view(np.float32)
    if screen_x is not None:
        r["screen_x"] = screen_x
    if screened is not None:
        r["screened"] = screened
    return r


def test_features_read_the_trace_words():
    w = trace_words(1.25, 3.5, 8.0, 1200)
    assert A.features(w, 0, 0.25) == [1.25, 1.25, 1.0, 1.0, 0.5, 0.25]
    assert A.features(w, 1, 0.3) == [3.5, 3.5, 1.0, 1.0, 0.5, float(np.float16(0.3))]
    assert A.steps_of(w) == 1200


def test_rows_classes_and_sums():
    # The reference tests' `row`: pass3 rows are further along at 2.5 s.
    words, flags, bars, sx = [], [], [], []
    for i, (pass3, exempt) in enumerate([(True, False), (False, False), (True, True), (False, False), (True, False)]):
        d150 = (3.0 if pass3 else 0.5) + 0.01 * i
        words.append(trace_words(d150 * 0.4, d150, 8.0 if pass3 else 1.0, 1200))
        flags.append(A.AUDIT | (A.EXEMPT if exempt else 0))
        bars.append(5.0)
        sx.append(8.0 if pass3 else 1.0)
    # Not an audit creature; an audit creature with no trace; no bar; dead
    # before R2.
    words += [trace_words(1, 1, 1, 1200), trace_words(1, 1, 1, 0), trace_words(1, 1, 1, 1200),
              trace_words(0.2, 0.0, 0.0, 100)]
    flags += [0, A.AUDIT, A.AUDIT, A.AUDIT]
    bars += [5.0, 5.0, np.nan, 5.0]
    sx += [1.0, 1.0, 1.0, 0.1]
    res = results_of(words, sx)
    periods = np.full(len(words), 0.25, np.float32)
    flags = np.array(flags, np.uint32)
    rows, sums, a_rows = A.gen_audit(res, flags, periods, np.array(bars, np.float32))
    assert A.rows(res, flags) == [0, 1, 2, 3, 4, 7, 8]
    assert rows == 7
    (a0, b0), (a1, b1) = sums
    assert (a0[0], b0[0], a1[0], b1[0]) == (2, 3, 2, 2)  # the dead-before-R2 row counts at R1 only
    d150 = [float(np.float16(x)) for x in (3.0, 3.04)]
    assert a1[1][0] == d150[0] + d150[1]
    assert a1[2][0][0] == d150[0] * d150[0] + d150[1] * d150[1]
    assert len(a_rows[1]) == 2 and (a_rows[1][:, 5] == h(0.25)).all()


def test_note_counts_trials_steps_and_stops():
    # End code bits 6-7: the rung that stopped the trial (1 R1, 2 R2, else
    # the 5 s screen).
    words = [trace_words(1, 1, 1, 60, code=1 << 6), trace_words(1, 1, 1, 150, code=2 << 6),
             trace_words(1, 1, 1, 300, code=0), trace_words(1, 1, 1, 1200, code=1 << 6)]
    res = results_of(words, screened=[1.0, 2.5, 5.0, 0.0])
    assert A.note(res) == (4, 60 + 150 + 300 + 1200, [1, 1, 1])


def test_one_in_128_slots_are_audit_creatures():
    # one_in_128_slots_are_audit_creatures (src/rungs/tests.rs:56-70).
    n = 2_000_000
    share = ce.api.audit_flags(5051, 7, np.arange(n)).mean()
    assert abs(share - 1 / 128) < 5e-4
    a = ce.api.audit_flags(1, 2, np.arange(4096))
    assert (a == ce.api.audit_flags(1, 2, np.arange(4096))).all()
    assert (a != ce.api.audit_flags(1, 3, np.arange(4096))).any()


def test_audit_flags_follow_the_hash():
    # is_audit's hash (src/rungs.rs:157-168) for one slot, in Python integers.
    def is_audit(seed, round_, slot):
        m = (1 << 64) - 1
        x = seed ^ (round_ * 0x9e3779b97f4a7c15 & m) ^ (slot * 0xd1342543de82ef95 & m)
        x = (x + 0x9e3779b97f4a7c15) & m
        x = ((x ^ (x >> 30)) * 0xbf58476d1ce4e5b9) & m
        x = ((x ^ (x >> 27)) * 0x94d049bb133111eb) & m
        return (x ^ (x >> 31)) % 128 == 0
    slots = np.arange(50_000)
    want = np.array([is_audit(77, 5, int(k)) for k in slots])
    assert (ce.api.audit_flags(77, 5, slots).astype(bool) == want).all() and want.sum() > 300


def test_a_second_restatement_agrees():
    # GenAudit::of written again, vectorised: the same rows, classes, counts
    # and class A words exactly; the float64 sums within rounding of the
    # summation order (np.sum pairs its terms).
    rng = np.random.default_rng(8)
    n = 20_000
    words = rng.integers(0, 1 << 32, size=(n, 7), dtype=np.uint64).astype(np.uint32)
    finite = rng.random((n, 7)) < 0.97
    words[finite] &= np.uint32(0x7bff7bff)
    words[:, 2] = (words[:, 2] & 0xffff) | (rng.integers(0, 1300, n).astype(np.uint32) << 16)
    res = results_of(words.tolist(), rng.normal(2.0, 1.5, n).astype(np.float32))
    flags = (np.where(rng.random(n) < 0.3, A.AUDIT, 0) | np.where(rng.random(n) < 0.1, A.EXEMPT, 0)).astype(np.uint32)
    periods = rng.uniform(0.2, 3.0, n).astype(np.float32)
    bars = rng.normal(2.0, 0.5, n).astype(np.float32)
    bars[rng.random(n) < 0.05] = np.nan
    rows, sums, a_rows = A.gen_audit(res, flags, periods, bars)

    def halves(w):
        return (w & 0xffff).astype(np.uint16).view(np.float16).astype(np.float64), \
            (w >> 16).astype(np.uint16).view(np.float16).astype(np.float64)

    steps = words[:, 2] >> 16
    is_row = ((flags & A.AUDIT) != 0) & (steps != 0)
    assert rows == int(is_row.sum())
    counted = is_row & ((flags & A.EXEMPT) == 0) & np.isfinite(bars)
    with np.errstate(invalid="ignore"):
        pass3 = res["screen_x"] >= bars
    lo, hi = zip(*[halves(words[:, k]) for k in range(7)])
    ph = periods.astype(np.float16).astype(np.float64)
    for r in range(2):
        f = np.stack([hi[0] if r else lo[0], hi[3] if r else lo[3], lo[4 + r], hi[6] if r else lo[6], hi[4 + r], ph], 1)
        ok = counted & (steps > (150 if r else 60)) & np.isfinite(f).all(1)
        for k, cls in enumerate((ok & pass3, ok & ~pass3)):
            x = f[cls]
            assert sums[r][k][0] == len(x)
            np.testing.assert_allclose(sums[r][k][1], x.sum(0), rtol=1e-12)
            np.testing.assert_allclose(np.array(sums[r][k][2]), x.T @ x, rtol=1e-12)
        assert (a_rows[r] == f[ok & pass3].astype(np.float16).view(np.uint16)).all()
