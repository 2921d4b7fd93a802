"""Test infrastructure: bindings of the checkers in oracle/_ref/.

* ``RefKernel`` runs the reference's own kernel (shaders/creature.cu, built
  by oracle/build_ref.py) on the GPU with the reference engine's launch rule.
  It is the bit-level oracle for the engine's kernel and the GPU baseline.
* ``Oracle`` runs the CPU restatement of the kernel (oracle/creature_oracle.cpp).

Only tests/, the smoke check and the benchmark's reference arm use this.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"

RESULT_DTYPE = np.dtype([(n, "<f4") for n in [
    "fitness", "ground_contact", "vertical_oscillation", "gait_frequency", "previous_center_y",
    "vertical_extremum", "vertical_trend", "gait_turns", "height_sum", "contact_lo", "contact_hi", "lift_lo",
    "lift_hi", "ground_lo", "ground_hi", "fall_time", "head_shake", "screen_x", "screened"]])


def variant_path(flags: int, rate: int = 60, record: bool = False) -> Path:
    return REF / f"libref_{flags:03x}_{rate}_{int(record)}.so"


class RefKernel:
    """The reference kernel for one world, step rate and recording switch."""

    def __init__(self, flags: int, rate: int = 60, record: bool = False):
        path = variant_path(flags, rate, record)
        if not path.exists():
            raise FileNotFoundError(f"{path} is missing: build it with python oracle/build_ref.py")
        self.lib = C.CDLL(str(path))
        self.lib.ref_run.restype = C.c_int
        self.lib.ref_run.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_float),
                                     C.c_char_p, C.c_size_t]
        assert self.lib.ref_result_size() == RESULT_DTYPE.itemsize
        self.params_size = self.lib.ref_params_size()
        self.record = record

    def run(self, wave, params):
        """(results in packed order, GPU milliseconds) for the packed batch."""
        assert C.sizeof(params) == self.params_size, (C.sizeof(params), self.params_size)
        n = len(wave)
        out = np.zeros(n, RESULT_DTYPE)
        ms = C.c_float()
        err = C.create_string_buffer(512)
        rc = self.lib.ref_run(wave.lanes.ctypes.data, len(wave.lanes), wave.muscles.ctypes.data,
                              len(wave.muscles), wave.heads.ctypes.data, n, C.byref(params), out.ctypes.data,
                              None, 0, C.byref(ms), err, 512)
        if rc != 0:
            raise RuntimeError(f"reference kernel failed: {err.value.decode()}")
        return out, ms.value

    def record_one(self, wave1, params, frames: int, stride: int):
        """Every frame of the one creature of `wave1`: [frame, slot, 2]."""
        assert len(wave1) == 1
        out = np.zeros(1, RESULT_DTYPE)
        fr = np.zeros((frames, stride, 2), np.float32)
        ms = C.c_float()
        err = C.create_string_buffer(512)
        rc = self.lib.ref_run(wave1.lanes.ctypes.data, len(wave1.lanes), wave1.muscles.ctypes.data,
                              len(wave1.muscles), wave1.heads.ctypes.data, 1, C.byref(params), out.ctypes.data,
                              fr.ctypes.data, fr.size, C.byref(ms), err, 512)
        if rc != 0:
            raise RuntimeError(f"reference kernel failed: {err.value.decode()}")
        return fr, out


class Oracle:
    """The CPU oracle (oracle/creature_oracle.cpp): the reference kernel's
    per-creature simulation restated on the host, FP32 or FP64."""

    def __init__(self):
        path = REF / "liboracle.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} is missing: build it with python oracle/build_ref.py")
        self.lib = C.CDLL(str(path))
        self.lib.oracle_run.restype = C.c_double
        self.lib.oracle_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p,
                                        C.c_uint32, C.c_int, C.c_int, C.c_void_p, C.c_int]
        self.lib.oracle_trace.restype = None
        self.lib.oracle_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_uint32,
                                          C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_size_t]
        self.lib.oracle_tangent.restype = C.c_double
        self.lib.oracle_tangent.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p,
                                            C.c_uint32, C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        self.lib.oracle_tangent_along.restype = C.c_double
        self.lib.oracle_tangent_along.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t,
                                                  C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p,
                                                  C.c_uint32, C.c_uint32, C.c_void_p, C.c_size_t, C.c_uint32,
                                                  C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                  C.c_void_p]
        self.lib.oracle_count.restype = None
        self.lib.oracle_count.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_uint32,
                                          C.c_int, C.c_void_p, C.c_void_p]

    def run(self, wave, params, flags: int, rate: int = 60, first: int = 0, n: int = None, fp64: bool = False,
            threads: int = 0):
        """(results of packed creatures [first, first + n), wall seconds)."""
        n = len(wave) - first if n is None else n
        out = np.zeros(n, RESULT_DTYPE)
        secs = self.lib.oracle_run(wave.lanes.ctypes.data, wave.muscles.ctypes.data, wave.heads.ctypes.data, first,
                                   n, C.byref(params), flags, rate, 1 if fp64 else 0, out.ctypes.data, threads)
        return out, secs

    def trace(self, wave, params, flags: int, cidx: int, steps: int, rate: int = 60, fp64: bool = False):
        """(result, node positions after every step [steps, 32, 2]) of packed creature `cidx`."""
        out = np.zeros(1, RESULT_DTYPE)
        tr = np.full((steps, 32, 2), np.nan, np.float32)
        self.lib.oracle_trace(wave.lanes.ctypes.data, wave.muscles.ctypes.data, wave.heads.ctypes.data, cidx,
                              C.byref(params), flags, rate, 1 if fp64 else 0, out.ctypes.data, tr.ctypes.data, steps)
        return out[0], tr

    def count(self, wave, params, flags: int, cidx: int, rate: int = 60):
        """(result, arithmetic counts: add, mul, div, sqrt, transcendental,
        min/max, compare, other) of packed creature `cidx`'s trial."""
        out = np.zeros(1, RESULT_DTYPE)
        counts = np.zeros(8, np.uint64)
        self.lib.oracle_count(wave.lanes.ctypes.data, wave.muscles.ctypes.data, wave.heads.ctypes.data, cidx,
                              C.byref(params), flags, rate, out.ctypes.data, counts.ctypes.data)
        return out[0], counts

    def tangent(self, wave, params, flags: int, dmuscle, dnode, rate: int = 60, first: int = 0, threads: int = 0,
                dmass=None, dstart=None):
        """FP64 forward-mode tangents of the fitness of packed creatures
        [first, first + n): creature c's record fields move along
        dmuscle[c] (muscle slots x 9: amplitude, hill, cap, 1/capacity, phase,
        duty, 1/duty, 1/(1-duty), stiffness) and dnode[c] (node rows:
        friction) and dmass[c] (node rows: mass; None for none) and
        dstart[c] (node rows x 2: start x, y; None for none). Returns
        (d fitness [n], FP64 results, wall seconds); the FP64 fitness itself
        is left in `self.fitness64`."""
        dm = np.ascontiguousarray(dmuscle, np.float64)
        dn = np.ascontiguousarray(dnode, np.float64)
        n, mm = dm.shape[0], dm.shape[1]
        rows = dn.shape[1]
        out = np.zeros(n, RESULT_DTYPE)
        dfit = np.zeros(n, np.float64)
        fit = np.zeros(n, np.float64)
        secs = self.lib.oracle_tangent(wave.lanes.ctypes.data, wave.muscles.ctypes.data, wave.heads.ctypes.data,
                                       first, n, C.byref(params), flags, rate, dm.ctypes.data, dn.ctypes.data, rows,
                                       mm, dfit.ctypes.data, fit.ctypes.data, out.ctypes.data, threads,
                                       None if dmass is None else np.ascontiguousarray(dmass, np.float64).ctypes.data,
                                       None if dstart is None else np.ascontiguousarray(dstart, np.float64).ctypes.data)
        self.fitness64 = fit
        return dfit, out, secs

    def tangent_along(self, wave, params, flags: int, dmuscle, dnode, checkpoints, rate: int = 60,
                      threads: int = 0, every: int = 256, dmass=None):
        """As tangent, for packed creatures [0, n), with the FP64 state's
        values reset every `every` substeps to another run's `checkpoints`
        [creature, checkpoint, rows x 4 + muscle slots] (a GPU forward run's):
        the FP64 tangent along that run's trajectory."""
        dm = np.ascontiguousarray(dmuscle, np.float64)
        dn = np.ascontiguousarray(dnode, np.float64)
        ck = np.ascontiguousarray(checkpoints, np.float32)
        n, mm = dm.shape[0], dm.shape[1]
        rows = dn.shape[1]
        assert ck.shape[0] >= n and ck.shape[2] == 4 * rows + mm
        out = np.zeros(n, RESULT_DTYPE)
        dfit = np.zeros(n, np.float64)
        secs = self.lib.oracle_tangent_along(wave.lanes.ctypes.data, wave.muscles.ctypes.data,
                                             wave.heads.ctypes.data, 0, n, C.byref(params), flags, rate,
                                             dm.ctypes.data, dn.ctypes.data, rows, mm, ck.ctypes.data,
                                             ck.shape[1] * ck.shape[2], ck.shape[1], every, dfit.ctypes.data, None,
                                             out.ctypes.data, threads,
                                             None if dmass is None else np.ascontiguousarray(dmass, np.float64).ctypes.data)
        return dfit, out, secs
