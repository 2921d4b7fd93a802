// FP32 calibration: the multiply-add rate this GPU sustains, which is the
// denominator of the creature kernel's FP32 roofline. Every thread runs eight
// independent chains of fused multiply-adds on registers; the grid fills
// every multiprocessor. Two floating-point operations per multiply-add.
#include <cuda_runtime.h>

#include "../../include/creature_engine.h"
#include "host_model.h"

namespace {

__global__ void __launch_bounds__(256) fma_chains(float* out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (float)(threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 123.456f) out[0] = s;  // keeps the chains live
}

}  // namespace

extern "C" ce_status ce_measure_fp32(int device, double* tflops, double* seconds) {
    if (!tflops) return CE_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) {
        ce::set_error("ce_measure_fp32: cudaSetDevice failed");
        return CE_ERR_DEVICE;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float* out = nullptr;
    if (cudaMalloc(&out, 4) != cudaSuccess) {
        ce::set_error("ce_measure_fp32: cudaMalloc failed");
        return CE_ERR_OOM;
    }
    const int blocks = sms * 8, threads = 256, iters = 1 << 16;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    fma_chains<<<blocks, threads>>>(out, 256, 0.999f, 0.001f);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(t0);
        fma_chains<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
        cudaEventRecord(t1);
        cudaEventSynchronize(t1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t0, t1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(out);
    if (err != cudaSuccess) {
        ce::set_error(std::string("ce_measure_fp32: ") + cudaGetErrorString(err));
        return CE_ERR_DEVICE;
    }
    const double flops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    if (seconds) *seconds = best * 1e-3;
    return CE_OK;
}
