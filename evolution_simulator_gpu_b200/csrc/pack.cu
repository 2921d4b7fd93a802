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
