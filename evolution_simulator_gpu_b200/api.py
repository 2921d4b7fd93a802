"""Python host side of the creature engine: a ctypes binding of the C ABI in
include/creature_engine.h.

It mirrors the reference's engine surface for this path:

* ``Engine`` is ``trait Engine`` (src/engine.rs:163-199): ``submit``,
  ``poll``, ``wait``, ``free_slots``, ``allocated_bytes``, plus ``record``
  (``record_on_gpu``, src/engine.rs:71-92) and ``release_idle``.
* ``evaluate`` is ``Gpu::evaluate`` (src/gpu.rs:46-57): results in population
  order.
* ``pack`` is ``kernel::pack`` (src/kernel.rs:429-593) and ``make_params`` is
  ``kernel::params`` (src/kernel.rs:212-251).
* ``to_metrics`` and ``niche`` are ``scheduler::to_metrics``
  (src/scheduler.rs:890-923) and ``Descriptor::niche_in`` with ``cell_index``
  (src/qd.rs:762-846, 988-999).

Every call runs the compiled library; there is no Python or CPU stand-in for
the GPU path. A missing library or a missing GPU is an error.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libcreature_engine.so"

# ------------------------------------------------------------------ status
CE_OK, CE_ERR_INVALID, CE_ERR_OOM, CE_ERR_TIMEOUT, CE_ERR_DEVICE, CE_ERR_UNSUPPORTED, CE_ERR_BUSY = range(7)
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "OOM", 3: "TIMEOUT", 4: "DEVICE", 5: "UNSUPPORTED", 6: "BUSY"}

MAX_NODES = 32
MAX_MUSCLES = 96
NODE_WORDS = 6
BONE_WORDS = 6
MUSCLE_FIELDS = 20
SUBSTEPS = 16
NO_SENSOR = 255

FLAG_NAMES = ["GROUND", "TERRAIN", "SLOPE", "GAPS", "HURDLES", "QUAKE", "MUD", "WATER", "ICE", "WIND", "AIR",
              "BRAMBLES"]


class EngineError(RuntimeError):
    """A failed engine call; ``status`` is the ce_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status

    @property
    def out_of_memory(self) -> bool:
        return self.status == CE_ERR_OOM


# ------------------------------------------------------------- structures
class Rung(C.Structure):
    _fields_ = [("w", C.c_float * 6), ("bias", C.c_float), ("off", C.c_uint32)]


class World(C.Structure):
    _fields_ = [
        ("ground", C.c_uint32), ("terrain", C.c_uint32),
        ("gravity", C.c_float), ("air_retention", C.c_float), ("ground_friction", C.c_float),
        ("muscle_energy", C.c_float), ("muscle_recovery", C.c_float),
        ("slope", C.c_float), ("wind", C.c_float), ("mud", C.c_float), ("brambles", C.c_float),
        ("water", C.c_float), ("patches", C.c_float), ("gaps", C.c_float), ("hurdles", C.c_float),
        ("quake", C.c_float), ("duration", C.c_float), ("rate", C.c_uint32),
        ("has_screen", C.c_uint32), ("screen_seconds", C.c_float), ("screen_bar", C.c_float),
        ("screen_bar_young", C.c_float), ("screen_bar_reshaped", C.c_float),
        ("has_rungs", C.c_uint32), ("rungs", Rung * 2),
    ]


PARAM_FIELDS = ["count", "base", "steps", "screen_step", "stride", "gravity", "air", "friction", "terrain",
                "muscle_energy", "muscle_recovery", "slope", "wind", "mud", "gaps", "hurdles", "quake",
                "screen_bar", "screen_bar_young", "screen_bar_reshaped", "water", "patches", "air_sub",
                "inv_muscle_energy", "brambles"]


class Params(C.Structure):
    _fields_ = [(n, C.c_uint32 if i < 5 else C.c_float) for i, n in enumerate(PARAM_FIELDS)] + [
        ("r1", Rung), ("r2", Rung)]


RESULT_FIELDS = ["fitness", "ground_contact", "vertical_oscillation", "gait_frequency", "previous_center_y",
                 "vertical_extremum", "vertical_trend", "gait_turns", "height_sum", "contact_lo", "contact_hi",
                 "lift_lo", "lift_hi", "ground_lo", "ground_hi", "fall_time", "head_shake", "screen_x",
                 "screened"]
RESULT_DTYPE = np.dtype([(n, "<f4") for n in RESULT_FIELDS])
NODE_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("diameter", "<f4"), ("friction", "<f4")])
BONE_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("rest_length", "<f4"), ("min_angle", "<f4"),
                       ("max_angle", "<f4"), ("organ_mass", "<f4"), ("organ_at", "<f4")])
MUSCLE_DTYPE = np.dtype([("bone_a", "<u4"), ("bone_b", "<u4"), ("anchor_a", "<f4"), ("anchor_b", "<f4"),
                         ("short", "<f4"), ("long", "<f4"), ("period", "<f4"), ("phase", "<f4"),
                         ("duty", "<f4"), ("stiffness", "<f4"), ("sensor", "<u4"), ("reset", "<f4"),
                         ("tendon", "<f4")])
DUMP_HEAD_DTYPE = np.dtype([("parent", "<u8"), ("slot", "<u4"), ("op", "<u2"), ("parent_cell", "<u2"),
                            ("cma", "<u2"), ("period", "<u2"), ("emitter", "u1"), ("flags", "u1"), ("kind", "u1"),
                            ("nodes", "u1"), ("muscles", "u1"), ("parent_nodes", "u1"), ("parent_muscles", "u1"),
                            ("reserved", "u1")], align=True)
DUMP_ROW_BYTES = 64
GENOME_DTYPE = np.dtype([("node_start", "<u4"), ("node_count", "<u4"), ("bone_start", "<u4"),
                         ("bone_count", "<u4"), ("muscle_start", "<u4"), ("muscle_count", "<u4"),
                         ("id", "<u8"), ("flags", "<u4"), ("reserved", "<u4")])
METRICS_DTYPE = np.dtype([("fitness", "<f4"), ("ground_contact", "<f4"), ("vertical_oscillation", "<f4"),
                          ("gait_frequency", "<f4"), ("mean_height", "<f4"), ("feet", "<f4"),
                          ("screen_x", "<f4"), ("screened", "<u4"), ("steps", "<u4")])


class PopulationC(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("bones", C.c_void_p), ("muscles", C.c_void_p), ("genomes", C.c_void_p),
                ("count", C.c_size_t), ("strength_scale", C.c_void_p)]


class CmaC(C.Structure):
    _fields_ = [("templates", PopulationC), ("exploring", C.c_void_p), ("offsets", C.c_void_p),
                ("mean", C.c_void_p), ("covariance", C.c_void_p), ("path_c", C.c_void_p),
                ("path_sigma", C.c_void_p), ("sigma", C.c_void_p)]


class CmaDraw(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("generation", C.c_uint32), ("reserved", C.c_uint32), ("round", C.c_uint64),
                ("first_id", C.c_uint64), ("strength", C.c_float), ("min_size", C.c_float),
                ("max_size", C.c_float), ("min_friction", C.c_float), ("max_friction", C.c_float)]


class AuditSumsC(C.Structure):
    _fields_ = [("n", C.c_uint64), ("sum", C.c_double * 6), ("xx", (C.c_double * 6) * 6)]


class AuditC(C.Structure):
    _fields_ = [("creatures", C.c_uint64), ("steps", C.c_uint64), ("stops", C.c_uint64 * 3), ("rows", C.c_uint32),
                ("reserved", C.c_uint32), ("a", AuditSumsC * 2), ("b", AuditSumsC * 2)]


class WavePackC(C.Structure):
    _fields_ = [("lanes", C.c_void_p), ("lanes_len", C.c_size_t), ("muscles", C.c_void_p),
                ("muscles_len", C.c_size_t), ("heads", C.c_void_p), ("count", C.c_size_t)]


class GenSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("min_nodes", C.c_uint32), ("max_nodes", C.c_uint32),
                ("node_dist", C.c_uint32), ("mean_nodes", C.c_float), ("min_muscles", C.c_uint32),
                ("max_muscles", C.c_uint32), ("muscle_rule", C.c_uint32), ("max_extra", C.c_uint32),
                ("joint_lo_deg", C.c_float), ("joint_hi_deg", C.c_float), ("friction_lo", C.c_float),
                ("friction_hi", C.c_float), ("first_id", C.c_uint64)]


class Options(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("warps_per_cta", C.c_uint32),
                ("chunk_k", C.c_uint32), ("small_body", C.c_uint32), ("reserved", C.c_uint32 * 3)]


# --------------------------------------------------------------- library
_LIB: Optional[C.CDLL] = None


def _bind(lib: C.CDLL) -> None:
    P = C.POINTER
    sigs = {
        "ce_world_flags": (C.c_uint32, [P(World)]),
        "ce_make_params": (C.c_int, [P(World), C.c_uint32, C.c_uint32, C.c_uint32, P(Params)]),
        "ce_pack_size": (C.c_int, [P(PopulationC), C.c_void_p, C.c_size_t, P(C.c_size_t), P(C.c_size_t)]),
        "ce_pack": (C.c_int, [P(PopulationC), C.c_void_p, C.c_size_t, P(World), C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_frame_stride": (C.c_uint32, [C.c_uint32]),
        "ce_generate_size": (C.c_int, [P(GenSpec), C.c_size_t, C.c_size_t, P(C.c_size_t), P(C.c_size_t),
                                       P(C.c_size_t)]),
        "ce_generate": (C.c_int, [P(GenSpec), C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
        "ce_to_metrics": (C.c_int, [C.c_void_p, C.c_uint32, P(World), C.c_void_p]),
        "ce_niche": (C.c_int64, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_int, C.c_void_p]),
        "ce_open": (C.c_int, [C.c_int, P(Options), P(C.c_void_p)]),
        "ce_close": (C.c_int, [C.c_void_p]),
        "ce_last_error": (C.c_char_p, []),
        "ce_submit": (C.c_int, [C.c_void_p, P(WavePackC), P(World), P(C.c_uint64)]),
        "ce_poll": (C.c_int, [C.c_void_p, C.c_int64, P(C.c_uint64), C.c_void_p, C.c_size_t, P(C.c_size_t),
                              P(C.c_double)]),
        "ce_wait": (C.c_int, [C.c_void_p, C.c_int64]),
        "ce_free_slots": (C.c_int, [C.c_void_p]),
        "ce_allocated_bytes": (C.c_size_t, [C.c_void_p]),
        "ce_release_idle": (C.c_int, [C.c_void_p]),
        "ce_record": (C.c_int, [C.c_void_p, P(WavePackC), P(World), C.c_void_p, C.c_size_t, C.c_void_p]),
        "ce_advance_scratch_bytes": (C.c_size_t, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                                  C.c_uint32]),
        "ce_advance_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, P(Params), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.c_void_p]),
        "ce_advance_device_cells": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p, P(Params), P(World), C.c_uint32, C.c_uint32,
                                              C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_pack_plan": (C.c_int, [P(PopulationC), C.c_void_p, C.c_size_t, P(World), C.c_size_t, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_pack_device": (C.c_int, [P(PopulationC), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                     P(World), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_ascent_open": (C.c_int, [C.c_void_p, P(PopulationC), P(World), C.c_uint32, C.c_double, C.c_size_t,
                                     C.c_size_t, C.c_size_t, P(C.c_void_p)]),
        "ce_ascent_launch": (C.c_int, [C.c_void_p, P(C.c_double)]),
        "ce_ascent_fitness": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t]),
        "ce_ascent_genes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_ascent_close": (C.c_int, [C.c_void_p]),
        "ce_inject_fault": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int]),
        "ce_measure_fp32": (C.c_int, [C.c_int, P(C.c_double), P(C.c_double)]),
        "ce_ground": (None, [C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, P(C.c_float),
                             P(C.c_float)]),
        "ce_quake_hash": (C.c_uint32, [C.c_uint64]),
        "ce_advance_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, P(Params),
                                                C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]),
        "ce_noalloc_scratch_bytes": (C.c_size_t, []),
        "ce_to_metrics_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, P(World), C.c_void_p]),
        "ce_niche_batch": (C.c_int, [P(PopulationC), C.c_void_p, C.c_size_t, C.c_void_p, C.c_int, C.c_void_p]),
        "ce_forward": (C.c_int, [C.c_void_p, P(WavePackC), P(World), C.c_uint32, P(C.c_void_p)]),
        "ce_graph_open": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, P(World), P(C.c_void_p)]),
        "ce_autotune": (C.c_int, [C.c_void_p, P(WavePackC), P(World), P(Options), P(C.c_double)]),
        "ce_graph_launch": (C.c_int, [C.c_void_p, P(C.c_double)]),
        "ce_graph_results": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t]),
        "ce_graph_close": (C.c_int, [C.c_void_p]),
        "ce_metrics_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, P(World), C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_shape_classes": (C.c_int, [P(PopulationC), C.c_void_p, C.c_size_t, C.c_void_p, C.c_int, C.c_void_p]),
        "ce_sample_rows": (C.c_int, [C.c_void_p, C.c_size_t, C.c_uint64, C.c_size_t, P(C.c_size_t), P(C.c_size_t),
                                     P(C.c_size_t)]),
        "ce_sample_device": (C.c_int, [P(PopulationC), C.c_uint64, C.c_size_t, C.c_float, C.c_uint64, C.c_uint64,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_cma_offsets": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
        "ce_cma_init": (C.c_int, [P(CmaC), C.c_void_p]),
        "ce_cma_ask": (C.c_int, [P(CmaC), P(CmaDraw), C.c_uint64, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
        "ce_cma_tell": (C.c_int, [P(CmaC), P(PopulationC), C.c_void_p, C.c_uint64, C.c_size_t, C.c_void_p]),
        "ce_cma_recenter": (C.c_int, [P(CmaC), P(PopulationC), C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
        "ce_audit_scratch_bytes": (C.c_size_t, [C.c_size_t]),
        "ce_audit_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                      C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
        "ce_dump_rows": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, P(World), C.c_void_p]),
        "ce_dump_rows_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, P(World),
                                          C.c_void_p, C.c_void_p]),
        "ce_height_bin_edges": (None, [C.c_void_p]),
        "ce_replay_decode": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_tape_results": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
        "ce_tape_grad_floats": (C.c_uint32, [C.c_void_p]),
        "ce_tape_shape": (C.c_int, [C.c_void_p, P(C.c_uint32), P(C.c_uint32)]),
        "ce_tape_seconds": (C.c_int, [C.c_void_p, P(C.c_double), P(C.c_double)]),
        "ce_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]),
        "ce_backward_checked": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
        "ce_tape_free": (C.c_int, [C.c_void_p]),
        "ce_tangent": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ce_tape_checkpoints": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, P(C.c_uint32)]),
        "ce_gene_gradients": (C.c_int, [P(PopulationC), C.c_void_p, C.c_size_t, P(World), C.c_void_p, C.c_void_p,
                                        C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


def lib() -> C.CDLL:
    """The engine library, loaded once. Raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m evolution_simulator_gpu_b200.build")
        _LIB = C.CDLL(str(LIB_PATH))
        _bind(_LIB)
    return _LIB


EXPORTED = ["ce_world_flags", "ce_make_params", "ce_pack_size", "ce_pack", "ce_frame_stride", "ce_generate_size",
            "ce_generate", "ce_to_metrics", "ce_niche", "ce_open", "ce_close", "ce_last_error", "ce_submit",
            "ce_poll", "ce_wait", "ce_free_slots", "ce_allocated_bytes", "ce_release_idle", "ce_record",
            "ce_advance_scratch_bytes", "ce_advance_device", "ce_advance_device_cells", "ce_pack_plan", "ce_pack_device", "ce_ascent_open", "ce_ascent_launch",
            "ce_ascent_fitness", "ce_ascent_genes", "ce_ascent_close", "ce_inject_fault", "ce_measure_fp32",
            "ce_to_metrics_batch", "ce_niche_batch", "ce_ground", "ce_quake_hash", "ce_advance_device_noalloc",
            "ce_noalloc_scratch_bytes", "ce_forward", "ce_tape_results", "ce_tape_grad_floats", "ce_tape_shape",
            "ce_tape_seconds", "ce_backward", "ce_backward_checked", "ce_tape_free", "ce_tangent", "ce_gene_gradients", "ce_tape_checkpoints",
            "ce_replay_decode", "ce_sample_rows", "ce_sample_device", "ce_dump_rows", "ce_dump_rows_device", "ce_metrics_device", "ce_shape_classes", "ce_height_bin_edges", "ce_graph_open",
            "ce_graph_launch", "ce_graph_results", "ce_graph_close", "ce_autotune", "ce_cma_offsets", "ce_cma_init",
            "ce_cma_ask", "ce_cma_tell", "ce_cma_recenter", "ce_audit_scratch_bytes", "ce_audit_device"]


def _check(status: int, what: str) -> None:
    if status != CE_OK:
        msg = lib().ce_last_error().decode(errors="replace")
        raise EngineError(status, f"{what}: {msg}")


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


# ------------------------------------------------------------------ worlds
def make_world(**kw) -> World:
    """A world with the reference's default settings (src/config.rs:119-161):
    flat calm ground, 9.8 m/s^2, grip 1.5, 20 s trials at 60 steps a second,
    no screen and no rungs. Keyword arguments override fields."""
    w = World()
    w.ground = 1
    w.terrain = 0
    w.gravity = 9.8
    w.air_retention = 1.0
    w.ground_friction = 1.5
    w.muscle_energy = 1.0
    w.muscle_recovery = 1.0
    w.duration = 20.0
    w.rate = 60
    for k, v in kw.items():
        if k == "rungs":
            w.has_rungs = 1
            for i, r in enumerate(v):
                w.rungs[i].w[:] = list(r[0])
                w.rungs[i].bias = r[1]
                w.rungs[i].off = r[2]
        elif k == "screen":
            seconds, bar = v[0], v[1]
            young = v[2] if len(v) > 2 else bar
            reshaped = v[3] if len(v) > 3 else bar
            w.has_screen = 1
            w.screen_seconds, w.screen_bar, w.screen_bar_young, w.screen_bar_reshaped = seconds, bar, young, reshaped
        else:
            setattr(w, k, v)
    return w


def world_flags(w: World) -> int:
    return int(lib().ce_world_flags(C.byref(w)))


def make_params(w: World, base: int = 0, count: int = 0, stride: int = 0) -> Params:
    p = Params()
    _check(lib().ce_make_params(C.byref(w), base, count, stride, C.byref(p)), "ce_make_params")
    return p


def settle_frames(w: World) -> int:
    rate = w.rate or 60
    return (200 * rate + 119) // 120


def trial_steps(w: World) -> int:
    return int(np.round(np.float32(w.duration) * np.float32(w.rate or 60)))


def creature_substeps(results: np.ndarray, w: World) -> float:
    """Substeps the trials of `results` ran: a creature stops at its fall
    (fall_time) or at the screen (screened), else runs the whole trial, 16
    substeps a step (shaders/creature.cu:1063, 1159, 1182)."""
    rate = w.rate or 60
    total = trial_steps(w)
    t = np.where(results["fall_time"] > 0, results["fall_time"] * rate,
                 np.where(results["screened"] > 0, results["screened"] * rate, total))
    return float(SUBSTEPS * np.minimum(np.round(t), total).sum())


# -------------------------------------------------------------- population
@dataclasses.dataclass
class Population:
    """An arena-packed population (src/evolution.rs:440-453)."""
    nodes: np.ndarray
    bones: np.ndarray
    muscles: np.ndarray
    genomes: np.ndarray
    strength: Optional[np.ndarray] = None

    def __len__(self) -> int:
        return len(self.genomes)

    def c(self) -> PopulationC:
        return PopulationC(_ptr(self.nodes), _ptr(self.bones), _ptr(self.muscles), _ptr(self.genomes),
                           len(self.genomes), _ptr(self.strength))

    def creature(self, i: int):
        g = self.genomes[i]
        n = self.nodes[g["node_start"]:g["node_start"] + g["node_count"]]
        b = self.bones[g["bone_start"]:g["bone_start"] + g["bone_count"]]
        m = self.muscles[g["muscle_start"]:g["muscle_start"] + g["muscle_count"]]
        s = None if self.strength is None else self.strength[g["muscle_start"]:g["muscle_start"] + g["muscle_count"]]
        return n, b, m, s

    def subset(self, idx) -> "Population":
        """The creatures at `idx`, in that order, as a population of their own."""
        parts = [self.creature(int(i)) for i in idx]
        nodes = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, NODE_DTYPE)
        bones = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0, BONE_DTYPE)
        muscles = np.concatenate([p[2] for p in parts]) if parts else np.zeros(0, MUSCLE_DTYPE)
        strength = None
        if self.strength is not None:
            strength = np.concatenate([p[3] for p in parts]).astype(np.float32) if parts else np.zeros(0, np.float32)
        genomes = np.zeros(len(parts), GENOME_DTYPE)
        an = ab = am = 0
        for k, (i, p) in enumerate(zip(idx, parts)):
            g = self.genomes[int(i)]
            genomes[k] = (an, len(p[0]), ab, len(p[1]), am, len(p[2]), g["id"], g["flags"], 0)
            an += len(p[0])
            ab += len(p[1])
            am += len(p[2])
        return Population(nodes, bones, muscles, genomes, strength)


@dataclasses.dataclass
class GenSpecPy:
    seed: int
    min_nodes: int = 3
    max_nodes: int = 6
    node_dist: int = 0  # 0 uniform, 1 geometric
    mean_nodes: float = 7.0
    min_muscles: int = 2
    max_muscles: int = 24
    muscle_rule: int = 0  # 0 spanning + extras, 1 count uniform in [min, max]
    max_extra: int = 3
    joint_lo_deg: float = 120.0
    joint_hi_deg: float = 120.0
    friction_lo: float = 0.0
    friction_hi: float = 1.0
    first_id: int = 1

    def c(self) -> GenSpec:
        return GenSpec(self.seed, self.min_nodes, self.max_nodes, self.node_dist, self.mean_nodes,
                       self.min_muscles, self.max_muscles, self.muscle_rule, self.max_extra, self.joint_lo_deg,
                       self.joint_hi_deg, self.friction_lo, self.friction_hi, self.first_id)


def generate(spec: GenSpecPy, count: int, first: int = 0) -> Population:
    """`count` seeded synthetic creatures; creature i is a function of
    (spec.seed, first + i) only."""
    L = lib()
    cs = spec.c()
    nn, nb, nm = C.c_size_t(), C.c_size_t(), C.c_size_t()
    _check(L.ce_generate_size(C.byref(cs), first, count, C.byref(nn), C.byref(nb), C.byref(nm)),
           "ce_generate_size")
    nodes = np.zeros(nn.value, NODE_DTYPE)
    bones = np.zeros(nb.value, BONE_DTYPE)
    muscles = np.zeros(nm.value, MUSCLE_DTYPE)
    strength = np.zeros(nm.value, np.float32)
    genomes = np.zeros(count, GENOME_DTYPE)
    _check(L.ce_generate(C.byref(cs), first, count, _ptr(nodes), _ptr(bones), _ptr(muscles), _ptr(strength),
                         _ptr(genomes)), "ce_generate")
    return Population(nodes, bones, muscles, genomes, strength)


# --------------------------------------------------------------- packing
@dataclasses.dataclass
class WavePack:
    """Packed records of a batch (src/kernel.rs:56-72), sorted by (muscles,
    nodes, population index). `slots[c]` is the position in the packed
    indices of packed creature c; `info` holds node, bone and muscle counts
    and the quake hash."""
    lanes: np.ndarray
    muscles: np.ndarray
    heads: np.ndarray
    slots: np.ndarray
    info: np.ndarray

    def __len__(self) -> int:
        return len(self.slots)

    def c(self) -> WavePackC:
        return WavePackC(_ptr(self.lanes), len(self.lanes), _ptr(self.muscles), len(self.muscles),
                         _ptr(self.heads), len(self.slots))

    def take(self, packed_positions) -> "WavePack":
        """A batch of its own with the packed creatures at `packed_positions`
        (their record offsets rewritten), in that order."""
        pos = np.asarray(packed_positions, dtype=np.int64)
        lanes, muscles, heads = [], [], np.zeros((len(pos), 8), np.uint32)
        rl = ml = 0
        for k, c in enumerate(pos):
            h = self.heads[c].copy()
            n, m = int(h[0] & 255), int(h[1])
            r0, m0 = int(h[3]), int(h[4])
            rlen = n * NODE_WORDS + (n - 1) * BONE_WORDS
            lanes.append(self.lanes[r0:r0 + rlen])
            muscles.append(self.muscles[m0:m0 + m * MUSCLE_FIELDS])
            h[3], h[4] = rl, ml
            heads[k] = h
            rl += rlen
            ml += m * MUSCLE_FIELDS
        lanes_a = np.concatenate(lanes) if lanes else np.zeros(1, np.uint32)
        mus_a = np.concatenate(muscles) if muscles and ml else np.zeros(1, np.float32)
        return WavePack(np.ascontiguousarray(lanes_a, np.uint32), np.ascontiguousarray(mus_a, np.float32),
                        heads, self.slots[pos].copy(), self.info[pos].copy())

    @property
    def max_muscles(self) -> int:
        return int(self.heads[:, 1].max()) if len(self) else 0

    @property
    def max_nodes(self) -> int:
        return int((self.heads[:, 0] & 255).max()) if len(self) else 0


def pack(pop: Population, world: World, indices=None) -> WavePack:
    L = lib()
    pc = pop.c()
    idx = None if indices is None else np.ascontiguousarray(indices, np.uint32)
    n = len(pop) if idx is None else len(idx)
    rl, ml = C.c_size_t(), C.c_size_t()
    _check(L.ce_pack_size(C.byref(pc), _ptr(idx), n, C.byref(rl), C.byref(ml)), "ce_pack_size")
    lanes = np.zeros(rl.value, np.uint32)
    muscles = np.zeros(ml.value, np.float32)
    heads = np.zeros((n, 8), np.uint32)
    slots = np.zeros(n, np.uint32)
    info = np.zeros((n, 4), np.uint32)
    _check(L.ce_pack(C.byref(pc), _ptr(idx), n, C.byref(world), _ptr(lanes), _ptr(muscles), _ptr(heads),
                     _ptr(slots), _ptr(info)), "ce_pack")
    return WavePack(lanes, muscles, heads, slots, info)


@dataclasses.dataclass
class PackPlan:
    """The host half of a device packing (ce_pack_plan): packed order
    (population indices), record and muscle offsets, 3 floats per bone gene
    (direction, sine, cosine), and the sizes of the packed arrays."""
    order: np.ndarray
    record_at: np.ndarray
    muscle_at: np.ndarray
    trig: np.ndarray
    lanes_len: int
    muscles_len: int


def pack_plan(pop: Population, world: World, indices=None) -> PackPlan:
    L = lib()
    pc = pop.c()
    idx = None if indices is None else np.ascontiguousarray(indices, np.uint32)
    n = len(pop) if idx is None else len(idx)
    rl, ml = C.c_size_t(), C.c_size_t()
    _check(L.ce_pack_size(C.byref(pc), _ptr(idx), n, C.byref(rl), C.byref(ml)), "ce_pack_size")
    order = np.zeros(n, np.uint32)
    rat = np.zeros(n, np.uint32)
    mat = np.zeros(n, np.uint32)
    trig = np.zeros(3 * max(len(pop.bones), 1), np.float32)
    _check(L.ce_pack_plan(C.byref(pc), _ptr(idx), n, C.byref(world), len(pop.bones), _ptr(order), _ptr(rat),
                          _ptr(mat), _ptr(trig)), "ce_pack_plan")
    return PackPlan(order, rat, mat, trig, rl.value, ml.value)


def pack_device(dev_pop: PopulationC, trig: int, order: int, record_at: int, muscle_at: int, n: int, world: World,
                lanes: int, muscles: int, heads: int, stream: int = 0) -> None:
    """ce_pack_device on device pointers: `dev_pop` is a PopulationC whose
    pointers are device addresses (asynchronous on `stream`)."""
    _check(lib().ce_pack_device(C.byref(dev_pop), trig, order, record_at, muscle_at, n, C.byref(world), lanes,
                                muscles, heads, stream or None), "ce_pack_device")


def frame_stride(max_muscles: int) -> int:
    return int(lib().ce_frame_stride(max_muscles))


# ----------------------------------------------------------------- engine
class Engine:
    """One GPU's engine (the reference's ThreadedEngine surface)."""

    def __init__(self, device: int = 0, slots: int = 0, ctas_per_sm: int = 0, chunk_k: int = 0,
                 small_body: int = 0):
        """`ctas_per_sm` (0: as many as fit), `chunk_k` (creatures a warp
        claims per queue visit, 0: 64) and `small_body` (largest node count run
        as a small body, 0: 12) are the launch shape; `autotune` picks them."""
        h = C.c_void_p()
        opts = Options(slots, ctas_per_sm, 0, chunk_k, small_body)
        _check(lib().ce_open(device, C.byref(opts), C.byref(h)), "ce_open")
        self._h = h
        self.device = device

    def autotune(self, sample: WavePack, world: World) -> tuple[dict, float]:
        """Time `sample` under each launch shape (CTAs per SM x claim chunk x
        small-body bound) and keep the fastest for later submissions:
        ({ctas_per_sm, chunk_k, small_body}, its GPU-busy seconds). Results do
        not depend on the launch shape."""
        best, secs = Options(), C.c_double()
        _check(lib().ce_autotune(self.handle, C.byref(sample.c()), C.byref(world), C.byref(best), C.byref(secs)),
               "ce_autotune")
        return {"ctas_per_sm": best.ctas_per_sm, "chunk_k": best.chunk_k, "small_body": best.small_body}, secs.value

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise EngineError(CE_ERR_INVALID, "engine is closed")
        return self._h

    def close(self) -> None:
        if self._h:
            lib().ce_close(self._h)
            self._h = C.c_void_p()

    def __enter__(self) -> "Engine":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def name(self) -> str:
        return f"b200-cuda:{self.device}"

    def max_nodes(self) -> int:
        return MAX_NODES

    def submit(self, wave: WavePack, world: World) -> int:
        t = C.c_uint64()
        _check(lib().ce_submit(self.handle, C.byref(wave.c()), C.byref(world), C.byref(t)), "ce_submit")
        self._pending = getattr(self, "_pending", {})
        self._pending[t.value] = len(wave)
        return t.value

    def poll(self, timeout_s: float = 0.0):
        """(ticket, results in packed order, GPU-busy seconds) of the oldest
        finished submission, or None when nothing finished in time."""
        pending = getattr(self, "_pending", {})
        if not pending:
            return None
        cap = max(pending.values())
        out = np.empty(cap, RESULT_DTYPE)  # the library fills the first n
        t, n, busy = C.c_uint64(), C.c_size_t(), C.c_double()
        st = lib().ce_poll(self.handle, int(timeout_s * 1e6), C.byref(t), _ptr(out), cap, C.byref(n), C.byref(busy))
        if st == CE_ERR_TIMEOUT:
            return None
        _check(st, "ce_poll")
        pending.pop(t.value, None)
        return t.value, (out if n.value == cap else out[:n.value].copy()), busy.value

    def wait(self, timeout_s: float) -> bool:
        st = lib().ce_wait(self.handle, int(timeout_s * 1e6))
        if st == CE_ERR_TIMEOUT:
            return False
        _check(st, "ce_wait")
        return True

    def free_slots(self) -> int:
        return int(lib().ce_free_slots(self.handle))

    def allocated_bytes(self) -> int:
        return int(lib().ce_allocated_bytes(self.handle))

    def release_idle(self) -> None:
        _check(lib().ce_release_idle(self.handle), "ce_release_idle")

    def inject_fault(self, after: int, status: int) -> None:
        _check(lib().ce_inject_fault(self.handle, after, status), "ce_inject_fault")

    def run(self, wave: WavePack, world: World, timeout_s: float = 600.0):
        """Submit and wait: (results in packed order, busy seconds)."""
        t = self.submit(wave, world)
        while True:
            got = self.poll(timeout_s)
            if got is None:
                raise EngineError(CE_ERR_TIMEOUT, "submission did not finish")
            if got[0] == t:
                return got[1], got[2]

    def forward(self, wave: WavePack, world: World, checkpoint_every: int = 256) -> "Tape":
        """The batch's trials kept for gradients (ce_forward); see Tape."""
        return forward(self, wave, world, checkpoint_every)

    def record(self, wave: WavePack, world: World):
        """Every frame of each creature of `wave` (at most 65,536): an array
        [creature, frame, slot, 2] in the reference's frame layout
        (src/creature_kernel.rs:312-326), and the results in packed order."""
        k = len(wave)
        stride = frame_stride(wave.max_muscles)
        frames_per = settle_frames(world) + trial_steps(world) + 1
        frames = np.zeros((k, frames_per, stride, 2), np.float32)
        res = np.zeros(k, RESULT_DTYPE)
        _check(lib().ce_record(self.handle, C.byref(wave.c()), C.byref(world), _ptr(frames), frames.size,
                               _ptr(res)), "ce_record")
        return frames, res

    def scratch_bytes(self, flags: int, rate: int, max_nodes: int, max_muscles: int, count: int) -> int:
        """Bytes of the scratch of advance_device for `count` creatures."""
        return int(lib().ce_advance_scratch_bytes(self.handle, flags, rate, max_nodes, max_muscles, count))

    def advance_device(self, records: int, muscles: int, heads: int, results: int, counter: int, scratch: int,
                       params: Params, flags: int, rate: int, max_nodes: int, max_muscles: int,
                       stream: int = 0) -> None:
        """The kernel ABI on device pointers (asynchronous on `stream`)."""
        _check(lib().ce_advance_device(self.handle, records, muscles, heads, results, counter, scratch,
                                       C.byref(params), flags, rate, max_nodes, max_muscles, stream or None),
               "ce_advance_device")

    def advance_device_cells(self, records: int, muscles: int, heads: int, results: int, counter: int, scratch: int,
                             params: Params, world: World, max_nodes: int, max_muscles: int, shapes: int,
                             cells: int, metrics: int = 0, stream: int = 0, global_layout: bool = True) -> None:
        """advance_device with the niche epilogue in the creature kernel:
        each trial's metrics row (METRICS_DTYPE at `metrics`, 0 for none)
        and dense niche cell (int64 at `cells`) are stored with its result;
        `shapes` holds shape_classes() of the packed batch (asynchronous)."""
        _check(lib().ce_advance_device_cells(self.handle, records, muscles, heads, results, counter, scratch,
                                             C.byref(params), C.byref(world), max_nodes, max_muscles, shapes,
                                             1 if global_layout else 0, metrics or None, cells, stream or None),
               "ce_advance_device_cells")


# ------------------------------------------------------------------ ascent
class Ascent:
    """A population's gradient ascent kept on the GPU (ce_ascent_open):
    `launch()` runs `steps` checkpointed forward + backward runs, gene
    gradients, clipped ascent steps and device repacking, then scores the
    last genes, as one CUDA graph, and returns its GPU seconds;
    `fitness(k)` is step k's fitness in population order (k = steps: the
    last genes); `population()` the genes after the steps."""

    def __init__(self, engine: "Engine", pop: Population, world: World, steps: int, step: float):
        self._pop = pop
        self.steps = steps
        h = C.c_void_p()
        _check(lib().ce_ascent_open(engine.handle, C.byref(pop.c()), C.byref(world), steps, step, len(pop.nodes),
                                    len(pop.bones), len(pop.muscles), C.byref(h)), "ce_ascent_open")
        self._h = h

    def launch(self) -> float:
        s = C.c_double()
        _check(lib().ce_ascent_launch(self._h, C.byref(s)), "ce_ascent_launch")
        return s.value

    def fitness(self, step: int) -> np.ndarray:
        out = np.zeros(len(self._pop), np.float32)
        _check(lib().ce_ascent_fitness(self._h, step, _ptr(out), len(out)), "ce_ascent_fitness")
        return out

    def population(self) -> Population:
        p = self._pop
        nodes, muscles = p.nodes.copy(), p.muscles.copy()
        strength = None if p.strength is None else p.strength.copy()
        _check(lib().ce_ascent_genes(self._h, _ptr(nodes), _ptr(muscles), _ptr(strength)), "ce_ascent_genes")
        return Population(nodes, p.bones.copy(), muscles, p.genomes.copy(), strength)

    def close(self) -> None:
        if self._h:
            lib().ce_ascent_close(self._h)
            self._h = C.c_void_p()

    def __enter__(self) -> "Ascent":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ graphs
class GenerationGraph:
    """Several packed generations resident on the device and run as one CUDA
    graph (ce_graph_open): `launch()` runs them all and returns the GPU
    seconds; `results(k)` reads generation k's results (packed order)."""

    def __init__(self, engine: "Engine", waves, world: World):
        self._waves = list(waves)  # the packs stay alive while the graph is open
        arr = (WavePackC * len(self._waves))(*[w.c() for w in self._waves])
        h = C.c_void_p()
        _check(lib().ce_graph_open(engine.handle, arr, len(self._waves), C.byref(world), C.byref(h)), "ce_graph_open")
        self._h = h

    def launch(self) -> float:
        secs = C.c_double()
        _check(lib().ce_graph_launch(self._h, C.byref(secs)), "ce_graph_launch")
        return secs.value

    def results(self, k: int) -> np.ndarray:
        out = np.zeros(len(self._waves[k]), RESULT_DTYPE)
        _check(lib().ce_graph_results(self._h, k, _ptr(out), len(out)), "ce_graph_results")
        return out

    def close(self) -> None:
        if self._h:
            lib().ce_graph_close(self._h)
            self._h = None

    def __enter__(self) -> "GenerationGraph":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ replay
def replay_decode(bones: np.ndarray, muscles: int, frames: np.ndarray) -> dict:
    """One recorded creature's frames [frame, slot, 2] (Engine.record) in its
    own node numbering (engine::recorded, src/engine.rs:1062-1127):
    positions [frame, node, 2] and, when the frames carry them, energy and
    pull [frame, muscle], ground and friction [frame, node], broken [frame]."""
    bones = np.ascontiguousarray(bones, BONE_DTYPE)
    nodes = len(bones) + 1
    fr = np.ascontiguousarray(frames, np.float32)
    count, stride = fr.shape[0], fr.shape[1]
    out = {"positions": np.zeros((count, nodes, 2), np.float32)}
    forces = stride > MAX_NODES + muscles + nodes
    if forces:
        out.update(energy=np.zeros((count, muscles), np.float32), pull=np.zeros((count, muscles), np.float32),
                   ground=np.zeros((count, nodes), np.float32), friction=np.zeros((count, nodes), np.float32),
                   broken=np.zeros(count, np.uint64))
    g = out.get
    _check(lib().ce_replay_decode(_ptr(bones), nodes, muscles, _ptr(fr), count, stride, _ptr(out["positions"]),
                                  _ptr(g("energy")), _ptr(g("pull")), _ptr(g("ground")), _ptr(g("friction")),
                                  _ptr(g("broken"))), "ce_replay_decode")
    return out


# ---------------------------------------------------------------- gradients
GRAD_MUSCLE_FIELDS = ["amplitude", "hill", "cap", "inv_capacity", "phase", "duty", "inv_duty", "inv_complement",
                      "stiffness"]
GENE_MUSCLE_FIELDS = ["short", "long", "strength", "t_on", "t_off"]


class Tape:
    """A forward run kept for its backward pass, shaped like an autograd
    function: `Engine.forward` saves (checkpoints every 256 substeps),
    `backward` consumes. Calm world only."""

    def __init__(self, handle: C.c_void_p, count: int):
        self._h = handle
        self.count = count

    def _handle(self) -> C.c_void_p:
        if not self._h:
            raise EngineError(CE_ERR_INVALID, "the tape is freed")
        return self._h

    @property
    def results(self) -> np.ndarray:
        out = np.zeros(self.count, RESULT_DTYPE)
        _check(lib().ce_tape_results(self._handle(), _ptr(out), self.count), "ce_tape_results")
        return out

    @property
    def shape(self):
        """(node rows, muscle slots) of the gradient records."""
        rows, mm = C.c_uint32(), C.c_uint32()
        _check(lib().ce_tape_shape(self._handle(), C.byref(rows), C.byref(mm)), "ce_tape_shape")
        return rows.value, mm.value

    @property
    def seconds(self):
        """GPU seconds of the forward run and of the last backward pass."""
        f, b = C.c_double(), C.c_double()
        _check(lib().ce_tape_seconds(self._handle(), C.byref(f), C.byref(b)), "ce_tape_seconds")
        return f.value, b.value

    def backward(self, dl_dfitness=None, check: bool = False):
        """d(sum_c dl_dfitness[c] fitness_c) / d(record fields), one row per
        creature in packed order: 9 floats a muscle slot (GRAD_MUSCLE_FIELDS),
        then per node row its friction, then its mass, then its start
        position as (x, y) pairs. With `check`, (gradients, mismatches):
        ce_backward_checked's per-creature bits of reruns that did not
        reproduce the forward run (0: none)."""
        per = int(lib().ce_tape_grad_floats(self._handle()))
        out = np.zeros((self.count, per), np.float32)
        w = None if dl_dfitness is None else np.ascontiguousarray(dl_dfitness, np.float32)
        if w is not None and len(w) != self.count:
            raise ValueError("one weight a creature")
        if check:
            bad = np.zeros(self.count, np.uint32)
            _check(lib().ce_backward_checked(self._handle(), _ptr(w), _ptr(out), out.size, _ptr(bad)),
                   "ce_backward_checked")
            return out, bad
        _check(lib().ce_backward(self._handle(), _ptr(w), _ptr(out), out.size), "ce_backward")
        return out

    def tangent(self, dstart=None, dmuscle=None, dfriction=None, dmass=None) -> np.ndarray:
        """d fitness of each creature along a direction of its record fields
        by the tangent-linear run on the forward run's FP32 trajectory (the
        worlds `forward` takes): `dstart` [creature, rows, 2] start positions, `dmuscle`
        [creature, muscle slots, 9], `dfriction` and `dmass` [creature, rows], packed
        order, laid out as `backward`'s rows (each None for 0). The adjoint's
        check: <backward row, direction> = tangent."""
        rows, mm = self.shape
        def arr(x, width):
            return None if x is None else np.ascontiguousarray(x, np.float32).reshape(self.count, width)
        ds, dm, df = arr(dstart, 2 * rows), arr(dmuscle, len(GRAD_MUSCLE_FIELDS) * mm), arr(dfriction, rows)
        dn = arr(dmass, rows)
        out = np.zeros(self.count, np.float32)
        _check(lib().ce_tangent(self._handle(), _ptr(ds), _ptr(dm), _ptr(df), _ptr(dn), _ptr(out)), "ce_tangent")
        return out

    def checkpoints(self, steps: int) -> np.ndarray:
        """The forward run's checkpoints [creature, checkpoint, rows x 4 +
        muscle slots] (a trial of `steps` steps has ceil(steps / 16)):
        positions and velocities as (x, y) pairs, then energy stores, every
        16 steps."""
        rows, mm = self.shape
        n_ck = (steps + 15) // 16
        out = np.zeros((self.count, n_ck, 4 * rows + mm), np.float32)
        per = C.c_uint32()
        _check(lib().ce_tape_checkpoints(self._handle(), _ptr(out), out.size, C.byref(per)), "ce_tape_checkpoints")
        if per.value != n_ck:
            raise ValueError(f"the tape holds {per.value} checkpoints a creature, not {n_ck}")
        return out

    def free(self) -> None:
        if self._h:
            lib().ce_tape_free(self._h)
            self._h = None

    def __enter__(self) -> "Tape":
        return self

    def __exit__(self, *exc) -> None:
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def forward(engine: "Engine", wave: WavePack, world: World, checkpoint_every: int = 256) -> Tape:
    h = C.c_void_p()
    wc = wave.c()
    _check(lib().ce_forward(engine.handle, C.byref(wc), C.byref(world), checkpoint_every, C.byref(h)),
           "ce_forward")
    return Tape(h, len(wave))


def gene_gradients(pop: Population, wave: WavePack, world: World, grads: np.ndarray, shape, indices=None):
    """Gene gradients from record gradients (Tape.backward): an (muscle genes,
    5) array of d/d (GENE_MUSCLE_FIELDS) and a (node genes,) array of
    d/d friction, float64; creatures outside the batch stay 0. `indices` are
    those the batch was packed with."""
    rows, mm = shape
    pc = pop.c()
    idx = None if indices is None else np.ascontiguousarray(indices, np.uint32)
    g = np.ascontiguousarray(grads, np.float32)
    mg = np.zeros((len(pop.muscles), 5), np.float64)
    ng = np.zeros(len(pop.nodes), np.float64)
    _check(lib().ce_gene_gradients(C.byref(pc), _ptr(idx), len(wave), C.byref(world), _ptr(wave.slots), _ptr(g),
                                   rows, mm, _ptr(mg), _ptr(ng)), "ce_gene_gradients")
    return mg, ng


def evaluate(engine: Engine, pop: Population, world: World, indices=None) -> np.ndarray:
    """Results in population (or `indices`) order, as Gpu::evaluate gives them."""
    wave = pack(pop, world, indices)
    res, _ = engine.run(wave, world)
    out = np.zeros(len(wave), RESULT_DTYPE)
    out[wave.slots] = res
    return out


# ---------------------------------------------------------------- metrics
def to_metrics(results: np.ndarray, node_counts: np.ndarray, world: World) -> np.ndarray:
    """scheduler::to_metrics for every result (src/scheduler.rs:890-923)."""
    out = np.zeros(len(results), METRICS_DTYPE)
    res = np.ascontiguousarray(results, RESULT_DTYPE)
    nc = np.ascontiguousarray(node_counts, np.uint32)
    _check(lib().ce_to_metrics_batch(res.ctypes.data, nc.ctypes.data, len(res), C.byref(world), out.ctypes.data),
           "ce_to_metrics_batch")
    return out


def niche_cells(pop: Population, metrics: np.ndarray, indices=None, global_layout: bool = True) -> np.ndarray:
    """Dense niche cells (src/qd.rs:762-846, 988-999) of creatures `indices`
    (default: all, in order) with their metrics rows."""
    n = len(metrics)
    idx = None if indices is None else np.ascontiguousarray(indices, np.uint32)
    m = np.ascontiguousarray(metrics, METRICS_DTYPE)
    cells = np.zeros(n, np.int64)
    pc = pop.c()
    _check(lib().ce_niche_batch(C.byref(pc), _ptr(idx), n, m.ctypes.data, 1 if global_layout else 0,
                                cells.ctypes.data), "ce_niche_batch")
    return cells


def shape_classes(pop: Population, wave: "WavePack", indices=None, global_layout: bool = True) -> np.ndarray:
    """The niche's shape class (aspect axis) of each packed creature, for
    metrics_device."""
    out = np.zeros(len(wave), np.uint8)
    idx = None if indices is None else np.ascontiguousarray(indices, np.uint32)
    pc = pop.c()
    _check(lib().ce_shape_classes(C.byref(pc), _ptr(idx), len(wave), _ptr(wave.slots), 1 if global_layout else 0,
                                  _ptr(out)), "ce_shape_classes")
    return out


def audit_flags(seed: int, round_: int, slots) -> np.ndarray:
    """rungs::is_audit (src/rungs.rs:153-168) for each ring slot of breeding
    round `round_`: rungs::AUDIT (1) on one slot in 128, picked by a hash of
    (seed, round, slot), else 0."""
    s = np.asarray(slots, np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) ^ (np.uint64(round_) * np.uint64(0x9e3779b97f4a7c15)) ^ (s * np.uint64(0xd1342543de82ef95))
        x = x + np.uint64(0x9e3779b97f4a7c15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
        x = x ^ (x >> np.uint64(31))
    return (x % np.uint64(128) == 0).astype(np.uint32)


def audit(results: np.ndarray, pop: "Population", bars: np.ndarray, a_cap: int = 1 << 16, device=None) -> dict:
    """The rung audit of a batch on the GPU (ce_audit_device): `results` in
    population order, `pop` the batch's genomes (flags, first muscle's
    period), bars[i] the screen bar of creature i's block (NaN: none).
    Returns Audit::note's tallies, the audit row count and, per rung, class
    A and class B sums and class A's feature words."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)

    def up(arr):
        return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(dev)

    n = len(results)
    L = lib()
    dr, dg, dm = up(results), up(pop.genomes), up(pop.muscles if len(pop.muscles) else np.zeros(1, MUSCLE_DTYPE))
    db = up(np.ascontiguousarray(bars, np.float32))
    scratch = torch.empty(int(L.ce_audit_scratch_bytes(n)), dtype=torch.uint8, device=dev)
    out = torch.empty(C.sizeof(AuditC), dtype=torch.uint8, device=dev)
    words = torch.empty(2 * a_cap * 6, dtype=torch.int16, device=dev)
    stream = torch.cuda.current_stream(dev)
    _check(L.ce_audit_device(dr.data_ptr(), dg.data_ptr(), dm.data_ptr(), db.data_ptr(), n, scratch.data_ptr(),
                             scratch.numel(), out.data_ptr(), words.data_ptr(), a_cap, stream.cuda_stream),
           "ce_audit_device")
    stream.synchronize()
    a = AuditC.from_buffer_copy(out.cpu().numpy().tobytes())

    def sums(s):
        return int(s.n), list(s.sum), [list(row) for row in s.xx]

    w = words.cpu().numpy().view(np.uint16).reshape(2, a_cap, 6)
    return dict(creatures=int(a.creatures), steps=int(a.steps), stops=list(a.stops), rows=int(a.rows),
                sums=[[sums(a.a[r]), sums(a.b[r])] for r in range(2)],
                a_words=[w[r, :min(int(a.a[r].n), a_cap)].copy() for r in range(2)])


def height_bin_edges() -> np.ndarray:
    """The mean heights where the niche's height bin steps up."""
    out = np.zeros(5, np.float32)
    lib().ce_height_bin_edges(_ptr(out))
    return out


def metrics_device(results: int, heads: int, shapes: int, count: int, world: World, metrics: int, cells: int,
                   stream: int = 0, global_layout: bool = True) -> None:
    """The metrics epilogue on device pointers (asynchronous on `stream`):
    metrics rows (METRICS_DTYPE, `metrics` 0 to skip) and dense cells (int64)
    of `count` results, equal to to_metrics and niche_cells to the bit."""
    _check(lib().ce_metrics_device(results, heads, shapes, count, C.byref(world), 1 if global_layout else 0,
                                   metrics or None, cells, stream or None), "ce_metrics_device")


def dump_rows(results: np.ndarray, wave: WavePack, heads: np.ndarray, world: World,
              archive_fitness: Optional[np.ndarray] = None) -> np.ndarray:
    """The 64-byte generation dump rows (storage/dump.rs) of results in
    packed order, on the host: a (count, 64) uint8 array."""
    res = np.ascontiguousarray(results, RESULT_DTYPE)
    dh = np.ascontiguousarray(heads, DUMP_HEAD_DTYPE)
    af = None if archive_fitness is None else np.ascontiguousarray(archive_fitness, np.float32)
    assert len(res) == len(wave) == len(dh)
    out = np.zeros((len(res), DUMP_ROW_BYTES), np.uint8)
    _check(lib().ce_dump_rows(_ptr(res), _ptr(wave.heads), _ptr(dh), _ptr(af), len(res), C.byref(world), _ptr(out)),
           "ce_dump_rows")
    return out


def dump_rows_device(results: int, heads: int, dump_heads: int, archive_fitness: int, count: int, world: World,
                     rows: int, stream: int = 0) -> None:
    """dump_rows on device pointers (asynchronous on `stream`; `rows` 16-byte
    aligned, `archive_fitness` 0 for the results' fitness)."""
    _check(lib().ce_dump_rows_device(results, heads, dump_heads, archive_fitness or None, count, C.byref(world), rows,
                                     stream or None), "ce_dump_rows_device")


def ground(x: float, amplitude: float = 0.0, tilt: float = 0.0, width: float = 0.0, hurdle: float = 0.0,
           phase: float = 0.0):
    """(height, slope) of the ground under x (physics::ground)."""
    h, s = C.c_float(), C.c_float()
    lib().ce_ground(x, amplitude, tilt, width, hurdle, phase, C.byref(h), C.byref(s))
    return h.value, s.value


def quake_hash(creature_id: int) -> int:
    return int(lib().ce_quake_hash(creature_id))


def measure_fp32(device: int = 0) -> float:
    """The FP32 multiply-add rate of the GPU in TFLOP/s (calibration kernel)."""
    t, s = C.c_double(), C.c_double()
    _check(lib().ce_measure_fp32(device, C.byref(t), C.byref(s)), "ce_measure_fp32")
    return t.value


def niche(pop: Population, i: int, metrics_row: np.ndarray, global_layout: bool = True):
    """(dense cell index or -1, the six niche bytes) of creature i."""
    n, _, m, _ = pop.creature(i)
    nodes = np.ascontiguousarray(n)
    row = np.ascontiguousarray(np.asarray(metrics_row, METRICS_DTYPE).reshape(1))
    out = np.zeros(6, np.uint8)
    cell = lib().ce_niche(nodes.ctypes.data, len(n), len(m), row.ctypes.data, 1 if global_layout else 0,
                          out.ctypes.data)
    return int(cell), out
