// ce_advance_device_noalloc: the device-level creature kernel for callers that
// cannot allocate GPU memory.
//
// Who needs it: code on the evolution loop's critical path that must not call
// cudaMalloc or cudaFree, because cudaFree waits for all work on the device
// (a stall the simulator's own engine measured at 0.05 to 2.2 s per growth of
// a buffer), and hosts whose device memory is owned by another allocator, so
// that the engine may not take any of its own. Such a caller passes only its
// inputs and outputs; the kernel's scratch (the claim counter and the lane
// slots) is a fixed array in the library's device memory.
//
// Limits: the array holds kNoAllocBytes (32 MiB) on every GPU that loads the
// library, until the process exits. A launch runs as many warps as the array
// has room for at the request's body size (fewer than the full GPU for large
// bodies, so this entry point can be slower than ce_advance_device); a body
// size whose single block does not fit is rejected. Every call shares the
// array: calls whose work overlaps on the GPU (two streams, or two host
// threads) race on it and must not be issued. Each call outside a stream
// capture looks the array's address up on the current device (so it stays
// right after the host recreates the device's primary context); a call
// inside a capture reuses the address of the last call outside one, so the
// first call on a device must come before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/creature_engine.h"
#include "host_model.h"
#include "kernels.h"

namespace {

constexpr size_t kNoAllocBytes = (size_t)32 << 20;
constexpr size_t kCounterBytes = 256;  // the claim counter, then the slots

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// The array's device address on the current device. Outside a stream
// capture it is looked up on every call, so a primary context that the host
// tore down and created again (cudaDeviceReset, which reloads the library's
// module at a new address) is followed; inside a capture the address that
// the last call outside a capture found is used, since a capture must not
// be broken by a lookup.
ce_status scratch_address(int device, cudaStream_t stream, void** out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (device < 0 || device >= kMaxDevices) {
        ce::set_error("ce_advance_device_noalloc: device ordinal out of range");
        return CE_ERR_INVALID;
    }
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    const cudaError_t q = cudaStreamIsCapturing(stream, &capture);
    if (q != cudaSuccess) {
        ce::set_error(std::string("ce_advance_device_noalloc: cudaStreamIsCapturing: ") + cudaGetErrorString(q));
        return CE_ERR_DEVICE;
    }
    if (capture == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            ce::set_error(std::string("ce_advance_device_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return CE_ERR_DEVICE;
        }
        g_scratch_addr[device] = p;
    } else if (!g_scratch_addr[device]) {
        ce::set_error("ce_advance_device_noalloc: the first call on a device must come before any stream capture");
        return CE_ERR_INVALID;
    }
    *out = g_scratch_addr[device];
    return CE_OK;
}

}  // namespace

extern "C" size_t ce_noalloc_scratch_bytes(void) { return kNoAllocBytes; }

extern "C" ce_status ce_advance_device_noalloc(const uint32_t* records, const float* muscles,
                                               const uint32_t* heads, ce_result* results,
                                               const ce_params* params, uint32_t world_flags, uint32_t rate,
                                               uint32_t max_nodes, uint32_t max_muscles, void* stream) {
    if (!records || !muscles || !heads || !results || !params) {
        ce::set_error("ce_advance_device_noalloc: null argument");
        return CE_ERR_INVALID;
    }
    if (max_nodes < 2 || max_nodes > CE_MAX_NODES || max_muscles > CE_MAX_MUSCLES || params->steps < 1 ||
        (rate != 60 && rate != 120)) {
        ce::set_error("ce_advance_device_noalloc: unsupported sizes");
        return CE_ERR_INVALID;
    }
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) {
        ce::set_error(std::string("ce_advance_device_noalloc: cudaGetDevice: ") + cudaGetErrorString(err));
        return CE_ERR_DEVICE;
    }
    void* base = nullptr;
    ce_status s = scratch_address(device, static_cast<cudaStream_t>(stream), &base);
    if (s != CE_OK) return s;
    // Warps whose slots fit in the array at this body size.
    const size_t warp_bytes = (size_t)cek::slot_lines(max_nodes, max_muscles, false) * 32u * 16u;
    const size_t warps_fit = (kNoAllocBytes - kCounterBytes) / warp_bytes;
    const size_t blocks_fit = warps_fit / (cek::kBlock / 32u);
    if (blocks_fit < 1) {
        ce::set_error("ce_advance_device_noalloc: the scratch of one block at " + std::to_string(max_nodes) +
                      " nodes and " + std::to_string(max_muscles) + " muscles exceeds the " +
                      std::to_string(kNoAllocBytes >> 20) + " MiB array");
        return CE_ERR_INVALID;
    }
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    err = cek::advance_occupancy(max_nodes, max_muscles, world_flags, false, (int)rate, cek::kBlock, &per_sm);
    if (err != cudaSuccess || per_sm < 1) {
        ce::set_error(std::string("ce_advance_device_noalloc: occupancy: ") + cudaGetErrorString(err));
        return CE_ERR_DEVICE;
    }
    const size_t needed = ((size_t)params->count + cek::kBlock - 1) / cek::kBlock;
    const size_t grid = std::max<size_t>(1, std::min({needed, (size_t)per_sm * (size_t)sms, blocks_fit}));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The counter must start at zero; the slots are written before they are read.
    err = cudaMemsetAsync(base, 0, kCounterBytes, st);
    if (err != cudaSuccess) {
        ce::set_error(std::string("ce_advance_device_noalloc: cudaMemsetAsync: ") + cudaGetErrorString(err));
        return CE_ERR_DEVICE;
    }
    cek::KernelArgs a{};
    a.records = records;
    a.muscles = muscles;
    a.heads = reinterpret_cast<const uint4*>(heads);
    a.results = results;
    a.counter = static_cast<uint32_t*>(base);
    a.scratch = reinterpret_cast<float4*>(static_cast<unsigned char*>(base) + kCounterBytes);
    a.frames = nullptr;
    a.order = nullptr;
    a.count = params->count;
    a.rows = max_nodes;
    a.mm = max_muscles;
    a.frames_per_creature = 0;
    a.chunk_k = 4;
    cek::LaunchSpec ls{max_nodes, max_muscles, world_flags, false, (int)rate, (unsigned)grid, cek::kBlock, st};
    err = cek::launch_advance(ls, a, *params);
    if (err != cudaSuccess) {
        ce::set_error(std::string("ce_advance_device_noalloc: launch: ") + cudaGetErrorString(err));
        return CE_ERR_DEVICE;
    }
    return CE_OK;
}
