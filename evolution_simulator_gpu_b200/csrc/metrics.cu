// The metrics epilogue on the device: scheduler::to_metrics
// (src/scheduler.rs:859-923) and Descriptor::niche_in with cell_index
// (src/qd.rs:762-846, 988-999) for every result of a batch, so the archive
// gets its cells without a host pass over the results.
//
// Cells must equal the host's to the bit. The arithmetic is the host's with
// every rounding explicit (IEEE division, no fused multiply-add); the height
// axis, a logarithm on the host, becomes a comparison with the five heights
// where its bin steps up, which the host finds with its own arithmetic
// (height_bin_thresholds); a body's shape class depends on its genes alone
// and comes computed per creature (ce_shape_classes).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/creature_engine.h"
#include "host_model.h"

namespace {

struct MetricsArgs {
    uint32_t all_steps;
    float rate;
    float height_edges[5];
    uint32_t node_edges[3];
    uint32_t edges;  // 3 for the global layout, 2 for an island's
};

__device__ __forceinline__ float clamp_host(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

__device__ __forceinline__ uint32_t qd_bin(float v, float lo, float hi, uint32_t count) {
    const float f = floorf(__fmul_rn(__fdiv_rn(__fsub_rn(clamp_host(v, lo, hi), lo), __fsub_rn(hi, lo)), (float)count));
    const uint32_t b = f <= 0.0f ? 0u : (f >= 255.0f ? 255u : (uint32_t)f);
    return min(b, count - 1u);
}

// scheduler::to_metrics of one result of a body with `nodes` nodes.
__device__ __forceinline__ ce_metrics to_metrics(const ce_result& r, uint32_t nodes, const MetricsArgs& k) {
    const float ended = r.fall_time > 0.0f ? r.fall_time : r.screened;
    uint32_t steps = k.all_steps;
    if (ended > 0.0f) {
        const float x = roundf(__fmul_rn(ended, k.rate));
        const uint32_t s = x <= 0.0f ? 0u : (x >= 4294967295.0f ? 0xffffffffu : (uint32_t)x);
        steps = min(max(s, 1u), k.all_steps);
    }
    const float denom = (float)(steps * nodes);
    ce_metrics m;
    m.fitness = r.fitness;
    m.ground_contact = clamp_host(__fdiv_rn(r.ground_contact, denom), 0.0f, 1.0f);
    m.vertical_oscillation = isfinite(r.vertical_oscillation) ? fmaxf(r.vertical_oscillation, 0.0f) : 0.0f;
    m.gait_frequency = isfinite(r.gait_frequency) ? fmaxf(r.gait_frequency, 0.0f) : 0.0f;
    m.mean_height = fmaxf(__fdiv_rn(r.height_sum, (float)steps), 0.0f);
    m.feet = (float)__popc(__float_as_uint(r.lift_lo));
    m.screen_x = r.screen_x;
    m.screened = r.screened > 0.0f ? 1u : 0u;
    m.steps = steps;
    return m;
}

// The behaviour axes of a niche (Descriptor::niche_in, src/qd.rs:795-806):
// contact, cadence, height and feet (the last one less 1).
struct Behavior {
    uint32_t gc, gf, hb, feet;
};
__device__ __forceinline__ Behavior behavior(const ce_metrics& m, const MetricsArgs& k) {
    Behavior v;
    v.gc = qd_bin(clamp_host(m.ground_contact, 0.0f, 1.0f), 0.0f, 1.0f, 6u);
    v.gf = qd_bin(clamp_host(m.gait_frequency, 0.0f, 20.0f), 0.0f, 6.0f, 8u);
    const float mh = fmaxf(m.mean_height, 0.0f);
    v.hb = 0u;
    for (int b = 0; b < 5; b++) v.hb += mh >= k.height_edges[b] ? 1u : 0u;
    const float fr = roundf(fmaxf(m.feet, 0.0f));
    int fi = fr >= 2147483647.0f ? 2147483647 : (fr <= -2147483648.0f ? (-2147483647 - 1) : (int)fr);
    v.feet = (uint32_t)(min(max(fi, 1), 5) - 1);
    return v;
}

__global__ void metrics_kernel(const ce_result* results, const uint4* heads, const uint8_t* shape, size_t count,
                               const MetricsArgs k, ce_metrics* metrics, int64_t* cells) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < count; c += (size_t)gridDim.x * blockDim.x) {
        const ce_result r = results[c];
        const uint32_t nodes = heads[2 * c].x & 255u;
        const ce_metrics m = to_metrics(r, nodes, k);
        if (metrics) metrics[c] = m;
        const Behavior v = behavior(m, k);
        const uint32_t gc = v.gc, gf = v.gf, hb = v.hb;
        const int fi = (int)v.feet + 1;
        uint32_t size = 0u;
        for (uint32_t e = 0; e < k.edges; e++) size += nodes >= k.node_edges[e] ? 1u : 0u;
        const uint32_t classes = k.edges + 1u;
        const uint32_t sh = shape[c];
        int64_t index = -1;
        if (sh < classes) {
            index = ((((int64_t)gc * 8 + gf) * classes + sh) * 6 + hb) * 5 + (fi - 1);
            index = index * classes + size;
        }
        cells[c] = index;
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

}  // namespace

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
