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

__global__ void metrics_kernel(const ce_result* results, const uint4* heads, const uint8_t* shape, size_t count,
                               const MetricsArgs k, ce_metrics* metrics, int64_t* cells) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < count; c += (size_t)gridDim.x * blockDim.x) {
        const ce_result r = results[c];
        const uint32_t nodes = heads[2 * c].x & 255u;
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
        if (metrics) metrics[c] = m;
        const uint32_t gc = qd_bin(clamp_host(m.ground_contact, 0.0f, 1.0f), 0.0f, 1.0f, 6u);
        const uint32_t gf = qd_bin(clamp_host(m.gait_frequency, 0.0f, 20.0f), 0.0f, 6.0f, 8u);
        const float mh = fmaxf(m.mean_height, 0.0f);
        uint32_t hb = 0u;
        for (int b = 0; b < 5; b++) hb += mh >= k.height_edges[b] ? 1u : 0u;
        const float fr = roundf(fmaxf(m.feet, 0.0f));
        int fi = fr >= 2147483647.0f ? 2147483647 : (fr <= -2147483648.0f ? (-2147483647 - 1) : (int)fr);
        fi = min(max(fi, 1), 5);
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

// The five mean heights where the niche's height bin steps up.
extern "C" void ce_height_bin_edges(float out[5]) { ce::height_bin_thresholds(out); }
