"""Generation dump rows on the host (ce_dump_rows) against the byte layout
of the reference's dump rows (src/storage/dump.rs:76-113, written by
Dump::write_rows at 409-455): each field at its offset, the behaviour cell
as dump::cell makes it from the result's niche (storage/dump.rs:151-158),
the screened bit from the result, the rung trace words in the order of
GpuResult::rung_trace (src/creature_kernel.rs:100-118). No GPU is used."""
import numpy as np

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

TRACE = ["contact_hi", "lift_hi", "ground_hi", "previous_center_y", "vertical_extremum", "vertical_trend",
         "gait_turns"]


def _heads(n, rng):
    h = np.zeros(n, ce.DUMP_HEAD_DTYPE)
    h["parent"] = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    h["parent"][::7] = np.iinfo(np.uint64).max
    h["slot"] = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    h["op"] = rng.integers(0, 0x1000, n)
    h["op"][::5] = 0xFFF
    h["parent_cell"] = rng.integers(0, 2 ** 16, n)
    h["cma"] = rng.integers(0, 2 ** 16, n)
    h["period"] = rng.integers(0, 2 ** 16, n)
    h["emitter"] = rng.integers(0, 256, n)
    h["flags"] = rng.integers(0, 256, n) & 0xEF  # every bit but SCREENED, which the result sets
    h["kind"] = rng.integers(0, 16, n)
    for f in ("nodes", "muscles", "parent_nodes", "parent_muscles"):
        h[f] = rng.integers(0, 256, n)
    return h


def test_host_rows_follow_the_reference_layout():
    w = WORKLOADS["small"]
    world = w.world(duration=4.0)
    pop = ce.generate(w.spec, 256)
    wave = ce.pack(pop, world)
    rng = np.random.default_rng(5)
    n = len(wave)
    res = np.zeros(n, ce.RESULT_DTYPE)
    for f in ce.RESULT_DTYPE.names:
        res[f] = rng.normal(size=n).astype(np.float32)
    res["ground_contact"] = rng.uniform(0, 240 * 6, n)
    res["gait_frequency"] = rng.uniform(0, 8, n)
    res["height_sum"] = rng.uniform(0, 240 * 1.5, n)
    res["lift_lo"] = rng.integers(0, 64, n).astype(np.uint32).view(np.float32)
    res["fall_time"] = np.where(rng.random(n) < 0.5, rng.uniform(0.1, 4.0, n), 0.0)
    res["screened"] = np.where(rng.random(n) < 0.3, rng.uniform(0.1, 4.0, n), 0.0)
    heads = _heads(n, rng)
    archive = rng.normal(size=n).astype(np.float32)
    for af in (None, archive):
        rows = ce.dump_rows(res, wave, heads, world, af)
        assert rows.shape == (n, 64)
        metrics = ce.to_metrics(res, (wave.heads[:, 0] & 255).astype(np.uint32), world)
        for c in range(n):
            b = rows[c].tobytes()
            h, r = heads[c], res[c]
            assert int.from_bytes(b[0:4], "little") == h["slot"]
            assert b[4] == h["emitter"] and b[5] == int(h["op"]) & 0xFF
            assert b[6] == int(h["flags"]) | (16 if r["screened"] > 0 else 0)
            assert b[7] == int(h["kind"]) | ((int(h["op"]) >> 8) & 15) << 4
            assert int.from_bytes(b[8:16], "little") == h["parent"]
            assert int.from_bytes(b[16:18], "little") == h["parent_cell"]
            _, niche = ce.niche(pop, int(wave.slots[c]), metrics[c])
            cell = ((int(niche[0]) * 8 + int(niche[1])) * 6 + int(niche[3])) * 5 + int(niche[4])
            assert int.from_bytes(b[18:20], "little") == cell
            assert int.from_bytes(b[20:22], "little") == h["cma"]
            assert list(b[22:26]) == [h["nodes"], h["muscles"], h["parent_nodes"], h["parent_muscles"]]
            assert int.from_bytes(b[26:28], "little") == h["period"]
            assert b[28:32] == r["fitness"].tobytes()
            assert b[32:36] == (r["fitness"] if af is None else af[c]).tobytes()
            assert b[36:64] == b"".join(np.float32(r[f]).tobytes() for f in TRACE)
