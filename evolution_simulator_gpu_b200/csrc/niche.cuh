// The niche of a trial on the device: scheduler::to_metrics
// (src/scheduler.rs:859-923) and Descriptor::niche_in with cell_index
// (src/qd.rs:762-846, 988-999), shared by the metrics epilogue kernel and
// the creature kernel's end-of-trial store.
//
// Cells must equal the host's to the bit. The arithmetic is the host's with
// every rounding explicit (IEEE division, no fused multiply-add); the height
// axis, a logarithm on the host, becomes a comparison with the five heights
// where its bin steps up, which the host finds with its own arithmetic
// (height_bin_thresholds); a body's shape class depends on its genes alone
// and comes computed per creature (ce_shape_classes).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/creature_engine.h"

namespace cek {

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

// The dense cell of a trial's metrics for a body of `nodes` nodes and shape
// class `shape` (-1 for a shape outside the layout).
__device__ __forceinline__ int64_t cell_of(const ce_metrics& m, uint32_t nodes, uint32_t shape,
                                           const MetricsArgs& k) {
    const Behavior v = behavior(m, k);
    uint32_t size = 0u;
    for (uint32_t e = 0; e < k.edges; e++) size += nodes >= k.node_edges[e] ? 1u : 0u;
    const uint32_t classes = k.edges + 1u;
    if (shape >= classes) return -1;
    const int64_t index = ((((int64_t)v.gc * 8 + v.gf) * classes + shape) * 6 + v.hb) * 5 + v.feet;
    return index * classes + size;
}

}  // namespace cek
