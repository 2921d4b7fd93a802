"""Test infrastructure: a restatement of the reference's rung audit over one
batch of trials, the checker of the device's ce_audit_device. Only tests/
use it.

* ``note``: Audit::note for every trial (src/rungs.rs:510-525): trials,
  steps and the stops of R1, R2 and the 5 s screen.
* ``rows``: the audit rows record_rungs files (src/storage.rs:672-708): the
  trials of creatures flagged AUDIT whose trace is not empty, in batch order.
* ``gen_audit``: GenAudit::of (src/rungs.rs:319-345) with Sums::add
  (src/rungs.rs:286-299) and features (src/rungs.rs:224-235): per rung the
  sums of class A (reached the 5 s bar) and class B, in float64, added in row
  order as the reference adds them, and class A's feature words.

The trace is the seven words a result carries (RungTrace, src/
creature_kernel.rs:120-218): the bits of contact_hi, lift_hi, ground_hi,
previous_center_y, vertical_extremum, vertical_trend and gait_turns.
"""
from __future__ import annotations

import numpy as np

AUDIT, EXEMPT = 1, 2
RUNG_STEPS = (60, 150)
FEATURES = 6
TRACE_FIELDS = ("contact_hi", "lift_hi", "ground_hi", "previous_center_y", "vertical_extremum", "vertical_trend",
                "gait_turns")


def trace_words(results: np.ndarray) -> np.ndarray:
    """[n, 7] uint32: each result's trace words."""
    return np.stack([results[f].astype(np.float32).view(np.uint32) for f in TRACE_FIELDS], axis=1)


def half(w: int, high: bool) -> float:
    return float(np.uint16((int(w) >> 16) if high else (int(w) & 0xffff)).view(np.float16))


def to_half(x: float) -> float:
    """f16_to_f32(f32_to_f16(x)): numpy's float16 rounds to nearest even, as
    the reference's conversion does."""
    return float(np.float32(x).astype(np.float16))


def features(words, r: int, period: float):
    """features (src/rungs.rs:224-235): distance, speed, touched, head shake,
    energy at rung r, and the rhythm period in half precision."""
    return [half(words[r // 2], r % 2 == 1), half(words[3], r == 1), half(words[4 + r], False),
            half(words[6], r == 1), half(words[4 + r], True), to_half(period)]


def steps_of(words) -> int:
    return int(words[2]) >> 16


def stopped_by(words) -> int:
    return (int(words[2]) & 0xffff) >> 6 & 3


def note(results: np.ndarray):
    """(trials, steps, [R1, R2, screen] stops) of Audit::note over the batch."""
    w = trace_words(results)
    stops = [0, 0, 0]
    for i in range(len(results)):
        if results["screened"][i] > 0:
            k = stopped_by(w[i])
            stops[0 if k == 1 else 1 if k == 2 else 2] += 1
    return len(results), int(sum(steps_of(x) for x in w)), stops


def rows(results: np.ndarray, flags: np.ndarray):
    """Indices of the audit rows, in batch order."""
    w = trace_words(results)
    return [i for i in range(len(results)) if int(flags[i]) & AUDIT and steps_of(w[i]) != 0]


def gen_audit(results: np.ndarray, flags: np.ndarray, periods: np.ndarray, bars: np.ndarray):
    """GenAudit::of over the batch's audit rows. Returns (rows, sums, a_rows):
    sums[r][k] = (n, sum[6], xx[6][6]) for rung r and class k (0: A, 1: B),
    a_rows[r] the class A rows' features as half words."""
    w = trace_words(results)
    idx = rows(results, flags)
    sums = [[[0, [0.0] * FEATURES, [[0.0] * FEATURES for _ in range(FEATURES)]] for _ in range(2)] for _ in range(2)]
    a_rows = [[], []]
    for i in idx:
        bar = float(bars[i])
        if int(flags[i]) & EXEMPT or not np.isfinite(bar):
            continue
        pass3 = float(results["screen_x"][i]) >= bar
        for r in range(2):
            if not steps_of(w[i]) > RUNG_STEPS[r]:
                continue
            f = features(w[i], r, float(periods[i]))
            if not all(np.isfinite(f)):
                continue
            s = sums[r][0 if pass3 else 1]
            s[0] += 1
            for a in range(FEATURES):
                s[1][a] += f[a]
                for b in range(FEATURES):
                    s[2][a][b] += f[a] * f[b]
            if pass3:
                a_rows[r].append(np.array(f, np.float32).astype(np.float16).view(np.uint16))
    return len(idx), sums, [np.array(a, np.uint16).reshape(-1, FEATURES) for a in a_rows]
