// The packer on the device: kernel::fill_creature and the head words of
// kernel::pack_reusing (src/kernel.rs:336-411, 554-565) over physics2's model
// and start pose (src/physics2.rs:190-399), one creature a thread, writing
// the same records, muscle records and heads as the host's ce_pack.
//
// The arithmetic is packer.h, shared with the host. This file is built with
// IEEE division and square root and without fused multiply-adds, so each
// operation rounds as the host's (and the reference's Rust host's) does. The
// bone directions and the sines and cosines of the start pose come from the
// host (ce_pack_plan), computed with the C library's functions: they depend
// on the node genes only, so a batch whose muscles or frictions change (the
// gradient-refined search's ascent) repacks on the device with the same
// plan.
#include <cuda_runtime.h>

#include <string>

#include "../../include/creature_engine.h"
#include "host_model.h"
#include "packer.h"

namespace {

// The host's values of bone j: its gene-pose direction, and the sine and
// cosine of its start-pose angle (3 floats a bone gene).
struct PlanAngle {
    const float* t;
    __device__ float operator()(size_t j, float, float) const { return t[3 * j]; }
};
struct PlanTrig {
    const float* t;
    __device__ void operator()(size_t j, float, float& sn, float& cs) const {
        sn = t[3 * j + 1];
        cs = t[3 * j + 2];
    }
};

__global__ void __launch_bounds__(128) pack_kernel(const ce_population pop, const float* trig, const uint32_t* order,
                                                   const uint32_t* record_at, const uint32_t* muscle_at, size_t n,
                                                   const ce_world w, uint32_t* lanes, float* muscles,
                                                   uint32_t* heads) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = order[c];
        const float* t = trig + 3 * (size_t)pop.genomes[i].bone_start;
        ce::fill_creature(pop, i, w, lanes + record_at[c], muscles + muscle_at[c], heads + 8 * c, record_at[c],
                          muscle_at[c], PlanAngle{t}, PlanTrig{t});
    }
}

}  // namespace

extern "C" ce_status ce_pack_device(const ce_population* pop, const float* trig, const uint32_t* order,
                                    const uint32_t* record_at, const uint32_t* muscle_at, size_t n,
                                    const ce_world* world, uint32_t* lanes, float* muscles, uint32_t* heads,
                                    void* stream) {
    if (!pop || !trig || !order || !record_at || !muscle_at || !world || !lanes || !muscles || !heads) {
        ce::set_error("ce_pack_device: null argument");
        return CE_ERR_INVALID;
    }
    if (n == 0) return CE_OK;
    const unsigned block = 128;
    const size_t blocks = (n + block - 1) / block;
    const unsigned grid = (unsigned)(blocks < 148u * 32u ? blocks : 148u * 32u);
    pack_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(*pop, trig, order, record_at, muscle_at, n,
                                                                      *world, lanes, muscles, heads);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ce::set_error(std::string("ce_pack_device: launch: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    return CE_OK;
}

// ------------------------------------------------- the refinement's ascent
// Gene gradients on the device (the host's ce_gene_gradients, the same
// double arithmetic: packer.h), one creature a thread, from the backward
// run's record gradients of the packed batch.
namespace {

__global__ void __launch_bounds__(128) gene_grads_kernel(const ce_population pop, const float* trig,
                                                         const uint32_t* order, size_t n, const ce_world w,
                                                         const float* grads, uint32_t rows, uint32_t mm,
                                                         double* muscle_grads, double* node_grads) {
    const size_t per = (size_t)9 * mm + 4 * (size_t)rows;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = order[c];
        const float* t = trig + 3 * (size_t)pop.genomes[i].bone_start;
        ce::gene_gradients_one(pop, i, w, grads + c * per, rows, mm, muscle_grads, node_grads, PlanAngle{t},
                               PlanTrig{t});
    }
}

__device__ __forceinline__ double finite_or_zero(double g) { return isfinite(g) ? g : 0.0; }
// step x g clipped to [-unit, unit], rounded to float (g finite: a NaN or
// infinite gradient counts as 0).
__device__ __forceinline__ float clipped_move(double step, double g, double unit) {
    double v = step * g;
    v = v < -unit ? -unit : v;
    v = v > unit ? unit : v;
    return (float)v;
}
__device__ __forceinline__ float clip32(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
// x mod 1 into [0, 1), as numpy's float32 remainder rounds it.
__device__ __forceinline__ float wrap_unit(float x) {
    float m = fmodf(x, 1.0f);
    if (m != 0.0f) {
        if (m < 0.0f) m += 1.0f;
    } else {
        m = 0.0f;
    }
    return m;
}

// One clipped ascent step of every creature's differentiated genes, in
// place: per muscle short, long, strength scale, phase and duty, per node
// friction; each move is step x gradient clipped to the coordinate's unit
// (0.02 x the body's mean bone length for lengths, 0.05 for phase, duty
// and strength, 0.03 for friction), then the genes' clamps.
__global__ void __launch_bounds__(128) ascend_kernel(const ce_genome* genomes, const ce_bone_gene* bones,
                                                     ce_node_gene* nodes, ce_muscle_gene* muscles, float* strength,
                                                     const double* muscle_grads, const double* node_grads,
                                                     size_t count, double step) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const ce_genome g = genomes[i];
        double total = 0.0;
        for (uint32_t j = 0; j < g.bone_count; j++) total += (double)bones[g.bone_start + j].rest_length;
        double size = g.bone_count > 0 ? total / (double)g.bone_count : 1.0;
        size = size < 0.05 ? 0.05 : (size > 10.0 ? 10.0 : size);
        const double unit = (double)(0.02f * (float)size);
        for (uint32_t k = 0; k < g.muscle_count; k++) {
            ce_muscle_gene& m = muscles[g.muscle_start + k];
            const double* d = muscle_grads + 5 * (size_t)(g.muscle_start + k);
            const double T = (double)m.period;
            const float s = clip32(m.short_len + clipped_move(step, finite_or_zero(d[0]), unit), 0.01f, 1.6f);
            m.short_len = s;
            m.long_len = clip32(m.long_len + clipped_move(step, finite_or_zero(d[1]), unit), s, 2.0f);
            m.phase = wrap_unit(m.phase + clipped_move(step, -T * (finite_or_zero(d[3]) + finite_or_zero(d[4])), 0.05));
            m.duty = clip32(m.duty + clipped_move(step, T * finite_or_zero(d[4]), 0.05), 0.05f, 0.95f);
            if (strength) {
                float& st = strength[g.muscle_start + k];
                st = clip32(st + clipped_move(step, finite_or_zero(d[2]), 0.05), 0.5f, 1.5f);
            }
        }
        for (uint32_t r = 0; r < g.node_count; r++) {
            ce_node_gene& nd = nodes[g.node_start + r];
            nd.friction = clip32(nd.friction + clipped_move(step, finite_or_zero(node_grads[g.node_start + r]), 0.03), 0.0f, 1.0f);
        }
    }
}

}  // namespace

namespace cek {
cudaError_t launch_gene_grads(const ce_population& pop, const float* trig, const uint32_t* order, size_t n,
                              const ce_world& w, const float* grads, uint32_t rows, uint32_t mm, double* muscle_grads,
                              double* node_grads, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const size_t blocks = (n + 127) / 128;
    gene_grads_kernel<<<(unsigned)(blocks < 148u * 32u ? blocks : 148u * 32u), 128, 0, stream>>>(
        pop, trig, order, n, w, grads, rows, mm, muscle_grads, node_grads);
    return cudaGetLastError();
}
cudaError_t launch_ascend(const ce_population& pop, ce_node_gene* nodes, ce_muscle_gene* muscles, float* strength,
                          const double* muscle_grads, const double* node_grads, double step, cudaStream_t stream) {
    if (pop.count == 0) return cudaSuccess;
    const size_t blocks = (pop.count + 127) / 128;
    ascend_kernel<<<(unsigned)(blocks < 148u * 32u ? blocks : 148u * 32u), 128, 0, stream>>>(
        pop.genomes, pop.bones, nodes, muscles, strength, muscle_grads, node_grads, pop.count, step);
    return cudaGetLastError();
}
cudaError_t launch_pack(const ce_population& pop, const float* trig, const uint32_t* order, const uint32_t* record_at,
                        const uint32_t* muscle_at, size_t n, const ce_world& w, uint32_t* lanes, float* muscles,
                        uint32_t* heads, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const size_t blocks = (n + 127) / 128;
    pack_kernel<<<(unsigned)(blocks < 148u * 32u ? blocks : 148u * 32u), 128, 0, stream>>>(
        pop, trig, order, record_at, muscle_at, n, w, lanes, muscles, heads);
    return cudaGetLastError();
}
}  // namespace cek
