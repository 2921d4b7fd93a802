// Test infrastructure: launches the reference kernel.
//
// This file is compiled with the reference's own shaders/creature.cu
// (REF_SOURCE) and the #define prelude its host writes in front of it
// (src/kernel.rs:268-332, generated by oracle/build_ref.py). ref_run launches
// it as the reference engine does (src/cuda_engine.rs:2106-2316): the
// preferred shared-memory carveout at 100%, waves of at most 262,144
// creatures, a grid of min(ceil(count / 128), resident blocks - 2) blocks
// (src/cuda_engine.rs:518-530), one counter per wave and up to 8 streams.
// Only the tests, the smoke check and the benchmark's reference arm use it.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include REF_SOURCE

namespace {

constexpr size_t kWave = 262144;
constexpr int kStreamLimit = 8;
constexpr int kReservedBlocks = 2;

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

int fail(cudaError_t e, const char* what, char* err, size_t errlen) {
    if (err && errlen) snprintf(err, errlen, "%s: %s", what, cudaGetErrorString(e));
    return (int)e;
}

}  // namespace

#define TRY(expr, what)                                        \
    do {                                                       \
        cudaError_t _e = (expr);                               \
        if (_e != cudaSuccess) return fail(_e, what, err, errlen); \
    } while (0)

extern "C" int ref_params_size() { return (int)sizeof(Params); }
extern "C" int ref_result_size() { return (int)sizeof(Result); }
extern "C" int ref_record() { return RECORD; }

// Runs `count` creatures of a packed batch (host memory) through the
// reference kernel on the current device. `params_host` is a Params with the
// world's fields (count and base are set per wave here). Returns 0 or the
// CUDA error; `gpu_ms` receives the time from the first launch to the end of
// the last wave.
extern "C" int ref_run(const uint32_t* lanes, size_t lanes_len, const float* muscles, size_t muscles_len,
                       const uint32_t* heads, size_t count, const void* params_host, void* results_host,
                       float* frames_host, size_t frames_floats, float* gpu_ms, char* err, size_t errlen) {
    Params base_params;
    memcpy(&base_params, params_host, sizeof(Params));
    int dev = 0;
    TRY(cudaGetDevice(&dev), "cudaGetDevice");
    int sms = 0;
    TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
    TRY(cudaFuncSetAttribute(advance, cudaFuncAttributePreferredSharedMemoryCarveout, 100), "carveout");
    int per_sm = 0;
    TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, advance, BLOCK, 0), "occupancy");
    const size_t waves = (count + kWave - 1) / kWave;
    DevBuf d_lanes, d_muscles, d_unused, d_heads, d_results, d_counters, d_frames;
    TRY(cudaMalloc(&d_lanes.p, lanes_len * 4 + 16), "cudaMalloc");
    TRY(cudaMalloc(&d_muscles.p, muscles_len * 4 + 16), "cudaMalloc");
    TRY(cudaMalloc(&d_unused.p, 16), "cudaMalloc");
    TRY(cudaMalloc(&d_heads.p, count * 32 + 32), "cudaMalloc");
    TRY(cudaMalloc(&d_results.p, count * sizeof(Result) + 16), "cudaMalloc");
    TRY(cudaMalloc(&d_counters.p, (waves + 1) * 4), "cudaMalloc");
    TRY(cudaMemcpy(d_lanes.p, lanes, lanes_len * 4, cudaMemcpyHostToDevice), "H2D");
    TRY(cudaMemcpy(d_muscles.p, muscles, muscles_len * 4, cudaMemcpyHostToDevice), "H2D");
    TRY(cudaMemcpy(d_heads.p, heads, count * 32, cudaMemcpyHostToDevice), "H2D");
    TRY(cudaMemset(d_counters.p, 0, (waves + 1) * 4), "memset");
#if RECORD
    if (!frames_host || count != 1) {
        if (err && errlen) snprintf(err, errlen, "a recording holds one creature and needs a frame buffer");
        return -1;
    }
    TRY(cudaMalloc(&d_frames.p, frames_floats * 4), "cudaMalloc");
    TRY(cudaMemset(d_frames.p, 0, frames_floats * 4), "memset");
#endif
    const int nstreams = (int)(waves < (size_t)kStreamLimit ? waves : (size_t)kStreamLimit);
    std::vector<cudaStream_t> streams(nstreams > 0 ? nstreams : 1);
    for (auto& s : streams) TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    cudaEvent_t start, stop;
    TRY(cudaEventCreate(&start), "event");
    TRY(cudaEventCreate(&stop), "event");
    TRY(cudaDeviceSynchronize(), "sync");
    TRY(cudaEventRecord(start, 0), "event");
    for (auto& s : streams) TRY(cudaStreamWaitEvent(s, start, 0), "wait");
    for (size_t w = 0; w < waves; w++) {
        const size_t first = w * kWave;
        const size_t n = count - first < kWave ? count - first : kWave;
        Params p = base_params;
        p.count = (unsigned)n;
        p.base = (unsigned)first;
        size_t blocks = (n + BLOCK - 1) / BLOCK;
        const size_t resident = (size_t)per_sm * (size_t)sms;
        const size_t cap = resident > (size_t)kReservedBlocks ? resident - kReservedBlocks : 0;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        cudaStream_t s = streams[w % streams.size()];
        advance<<<(unsigned)blocks, BLOCK, 0, s>>>(
            static_cast<const unsigned*>(d_lanes.p), static_cast<const float*>(d_muscles.p),
            static_cast<const unsigned*>(d_unused.p), static_cast<const uint4*>(d_heads.p),
            static_cast<Result*>(d_results.p), static_cast<unsigned*>(d_counters.p) + w, p
#if RECORD
            , static_cast<float2*>(d_frames.p)
#endif
        );
        TRY(cudaGetLastError(), "launch");
    }
    for (auto& s : streams) {
        cudaEvent_t j;
        TRY(cudaEventCreateWithFlags(&j, cudaEventDisableTiming), "event");
        TRY(cudaEventRecord(j, s), "event");
        TRY(cudaStreamWaitEvent(0, j, 0), "wait");
        cudaEventDestroy(j);
    }
    TRY(cudaEventRecord(stop, 0), "event");
    TRY(cudaEventSynchronize(stop), "kernel");
    float ms = 0.0f;
    TRY(cudaEventElapsedTime(&ms, start, stop), "elapsed");
    if (gpu_ms) *gpu_ms = ms;
    TRY(cudaMemcpy(results_host, d_results.p, count * sizeof(Result), cudaMemcpyDeviceToHost), "D2H");
#if RECORD
    TRY(cudaMemcpy(frames_host, d_frames.p, frames_floats * 4, cudaMemcpyDeviceToHost), "D2H");
#endif
    for (auto& s : streams) cudaStreamDestroy(s);
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    return 0;
}
