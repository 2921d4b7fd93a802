// The metrics epilogue on the device: scheduler::to_metrics
// (src/scheduler.rs:859-923) and Descriptor::niche_in with cell_index
// (src/qd.rs:762-846, 988-999) for every result of a batch, so the archive
// gets its cells without a host pass over the results (niche.cuh holds the
// arithmetic, which the creature kernel also runs at its result store).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/creature_engine.h"
#include "host_model.h"
#include "kernels.h"
#include "niche.cuh"

using cek::Behavior;
using cek::MetricsArgs;
using cek::behavior;
using cek::to_metrics;

namespace {

__global__ void metrics_kernel(const ce_result* results, const uint4* heads, const uint8_t* shape, size_t count,
                               const MetricsArgs k, ce_metrics* metrics, int64_t* cells) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < count; c += (size_t)gridDim.x * blockDim.x) {
        const ce_result r = results[c];
        const uint32_t nodes = heads[2 * c].x & 255u;
        const ce_metrics m = to_metrics(r, nodes, k);
        if (metrics) metrics[c] = m;
        cells[c] = cek::cell_of(m, nodes, shape[c], k);
    }
}

// One 64-byte generation dump row (storage/dump.rs:76-113, write_rows
// 409-455) per result: the caller's breeding fields, the behaviour cell of
// the result, its fitness and its rung trace words. Rows are written as 16
// words, so a warp stores 2 KB in one coalesced sweep.
__global__ void dump_rows_kernel(const ce_result* results, const uint4* heads, const ce_dump_head* dump,
                                 const float* archive_fitness, size_t count, const MetricsArgs k, uint4* rows) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < count; c += (size_t)gridDim.x * blockDim.x) {
        const ce_result r = results[c];
        const ce_dump_head h = dump[c];
        const ce_metrics m = to_metrics(r, heads[2 * c].x & 255u, k);
        const Behavior v = behavior(m, k);
        const uint32_t cell = ((v.gc * 8u + v.gf) * 6u + v.hb) * 5u + v.feet;
        const uint32_t flags = h.flags | (m.screened ? CE_DUMP_SCREENED : 0u);
        const uint32_t kind = (h.kind & 15u) | (((uint32_t)(h.op >> 8) & 15u) << 4);
        const float archive = archive_fitness ? archive_fitness[c] : r.fitness;
        uint4 w0, w1, w2, w3;
        w0.x = h.slot;
        w0.y = (uint32_t)h.emitter | ((uint32_t)(h.op & 0xffu) << 8) | (flags << 16) | (kind << 24);
        w0.z = (uint32_t)h.parent;
        w0.w = (uint32_t)(h.parent >> 32);
        w1.x = (uint32_t)h.parent_cell | (cell << 16);
        w1.y = (uint32_t)h.cma | ((uint32_t)h.nodes << 16) | ((uint32_t)h.muscles << 24);
        w1.z = (uint32_t)h.parent_nodes | ((uint32_t)h.parent_muscles << 8) | ((uint32_t)h.period << 16);
        w1.w = __float_as_uint(r.fitness);
        w2.x = __float_as_uint(archive);
        w2.y = __float_as_uint(r.contact_hi);
        w2.z = __float_as_uint(r.lift_hi);
        w2.w = __float_as_uint(r.ground_hi);
        w3.x = __float_as_uint(r.previous_center_y);
        w3.y = __float_as_uint(r.vertical_extremum);
        w3.z = __float_as_uint(r.vertical_trend);
        w3.w = __float_as_uint(r.gait_turns);
        rows[4 * c] = w0;
        rows[4 * c + 1] = w1;
        rows[4 * c + 2] = w2;
        rows[4 * c + 3] = w3;
    }
}

}  // namespace

namespace cek {
MetricsArgs metrics_args(const ce_world* world, int global_layout) {
    MetricsArgs k;
    k.all_steps = std::max(ce::world_steps(*world), 1u);
    k.rate = (float)ce::world_rate(*world);
    ce::height_bin_thresholds(k.height_edges);
    if (global_layout) {
        k.edges = 3;
        k.node_edges[0] = 9;
        k.node_edges[1] = 11;
        k.node_edges[2] = 14;
    } else {
        k.edges = 2;
        k.node_edges[0] = 9;
        k.node_edges[1] = 12;
        k.node_edges[2] = 0;
    }
    return k;
}
}  // namespace cek

using cek::metrics_args;

// Metrics and dense cells of `count` results on the device (device
// pointers; `metrics` may be NULL); asynchronous on `stream`.
extern "C" ce_status ce_metrics_device(const ce_result* results, const uint32_t* heads, const uint8_t* shape_classes,
                                       size_t count, const ce_world* world, int global_layout, ce_metrics* metrics,
                                       int64_t* cells, void* stream) {
    if (!results || !heads || !shape_classes || !world || !cells) {
        ce::set_error("ce_metrics_device: null argument");
        return CE_ERR_INVALID;
    }
    const MetricsArgs k = metrics_args(world, global_layout);
    if (count == 0) return CE_OK;
    const unsigned block = 256;
    const unsigned grid = (unsigned)std::min<size_t>((count + block - 1) / block, 148u * 16u);
    metrics_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        results, reinterpret_cast<const uint4*>(heads), shape_classes, count, k, metrics, cells);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ce::set_error(std::string("metrics launch: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    return CE_OK;
}

// Generation dump rows of `count` results on the device (device pointers;
// `archive_fitness` may be NULL); asynchronous on `stream`.
extern "C" ce_status ce_dump_rows_device(const ce_result* results, const uint32_t* heads, const ce_dump_head* dump,
                                         const float* archive_fitness, size_t count, const ce_world* world,
                                         uint8_t* rows, void* stream) {
    if (!results || !heads || !dump || !world || !rows) {
        ce::set_error("ce_dump_rows_device: null argument");
        return CE_ERR_INVALID;
    }
    if (reinterpret_cast<uintptr_t>(rows) % 16u != 0u) {
        ce::set_error("ce_dump_rows_device: rows must be 16-byte aligned");
        return CE_ERR_INVALID;
    }
    const MetricsArgs k = metrics_args(world, 1);
    if (count == 0) return CE_OK;
    const unsigned block = 256;
    const unsigned grid = (unsigned)std::min<size_t>((count + block - 1) / block, 148u * 16u);
    dump_rows_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        results, reinterpret_cast<const uint4*>(heads), dump, archive_fitness, count, k,
        reinterpret_cast<uint4*>(rows));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ce::set_error(std::string("dump rows launch: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    return CE_OK;
}

// The five mean heights where the niche's height bin steps up.
extern "C" void ce_height_bin_edges(float out[5]) { ce::height_bin_thresholds(out); }
