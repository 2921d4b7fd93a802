"""B200 creature-evaluation engine.

Runs the evolution simulator's per-creature position-based-dynamics trials
(the reference's shaders/creature.cu path) on sm_100a GPUs behind a C ABI
(include/creature_engine.h). This package holds the CUDA kernels and host
library sources (csrc/), their build (build.py), the ctypes binding of the C
ABI (api.py) and the seeded workloads (configs.py).
"""
from .api import (  # noqa: F401
    CE_ERR_BUSY, CE_ERR_DEVICE, CE_ERR_INVALID, CE_ERR_OOM, CE_ERR_TIMEOUT, CE_ERR_UNSUPPORTED, CE_OK,
    EXPORTED, FLAG_NAMES, METRICS_DTYPE, GenerationGraph, RESULT_DTYPE, RESULT_FIELDS, Engine, EngineError, GenSpecPy, Params,
    Population, Tape, WavePack, World, creature_substeps, evaluate, forward, gene_gradients, frame_stride, generate, lib, make_params, make_world, measure_fp32, niche,
    niche_cells, pack, pack_device, pack_plan, PackPlan, Ascent,
    DUMP_HEAD_DTYPE, DUMP_ROW_BYTES, dump_rows, dump_rows_device, height_bin_edges, metrics_device, replay_decode, settle_frames, shape_classes, to_metrics, trial_steps,
    world_flags)
