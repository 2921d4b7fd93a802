// Bucketing of a packed batch by node count, on the device: the claim
// queues of the persistent launch (kernels.h).
//
// A counting sort in three kernels. Each block counts the node counts of
// one tile of kBucketTile creatures, one block scans the per-tile counts
// (node count major, tile minor) into start positions, and each block then
// scatters its tile. Tiles keep their order, so inside a node count the
// creatures keep the packed order up to the order within a tile (a tile
// spans about one muscle count of a batch sorted by muscle count). The
// order within a tile is not fixed from run to run; a creature's result
// does not depend on when or on which lane it runs.
#include <cuda_runtime.h>

#include "kernels.h"

namespace cek {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr unsigned kTileThreads = 256u;
constexpr unsigned kScanThreads = 1024u;

size_t align256(size_t b) { return (b + 255u) & ~(size_t)255u; }

__device__ __forceinline__ unsigned node_count(const uint4* heads, uint32_t cidx) {
    return min(heads[2ull * cidx].x & 255u, (unsigned)CE_MAX_NODES);
}

// Operations of one substep of a body, about 75 a muscle, 40 a bone, 36 a
// node and 110 a joint: the weight that splits the warps between queues.
__device__ __forceinline__ unsigned long long body_work(unsigned n, unsigned m) {
    const unsigned bones = n > 0u ? n - 1u : 0u, joints = n > 1u ? n - 2u : 0u;
    return 75ull * m + 40ull * bones + 36ull * n + 110ull * joints;
}

__global__ void __launch_bounds__(kTileThreads) bucket_count(const uint4* heads, uint32_t base, uint32_t count,
                                                             uint32_t tiles, uint32_t* hist,
                                                             unsigned long long* bins) {
    __shared__ uint32_t h[kQueues];
    __shared__ unsigned long long wk[kQueues];
    for (unsigned q = threadIdx.x; q < kQueues; q += blockDim.x) {
        h[q] = 0u;
        wk[q] = 0ull;
    }
    __syncthreads();
    const uint32_t lo = blockIdx.x * kBucketTile, hi = min(count, lo + kBucketTile);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint4 h0 = heads[2ull * (base + i)];
        const unsigned n = min(h0.x & 255u, (unsigned)CE_MAX_NODES);
        atomicAdd(&h[n], 1u);
        atomicAdd(&wk[n], body_work(n, h0.y));
    }
    __syncthreads();
    for (unsigned q = threadIdx.x; q < kQueues; q += blockDim.x) {
        hist[q * tiles + blockIdx.x] = h[q];
        if (wk[q] != 0ull) {
            atomicAdd(&bins[q], wk[q]);
        }
    }
}

// One block: exclusive scan of the kQueues x tiles counts in place, then the
// queue bounds, the work prefix and zeroed counters.
__global__ void __launch_bounds__(kScanThreads) bucket_scan(uint32_t* hist, uint32_t tiles, uint32_t count,
                                                            uint32_t* bounds, unsigned long long* work,
                                                            const unsigned long long* bins, uint32_t* counters) {
    __shared__ uint32_t warp_sums[kScanThreads / 32u];
    const uint32_t entries = kQueues * tiles;
    const uint32_t per = (entries + blockDim.x - 1u) / blockDim.x;
    const uint32_t lo = min(entries, threadIdx.x * per), hi = min(entries, lo + per);
    uint32_t sum = 0u;
    for (uint32_t i = lo; i < hi; i++) {
        sum += hist[i];
    }
    const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5u;
    uint32_t x = sum;
    for (unsigned o = 1u; o < 32u; o <<= 1u) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31u) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0u) {
        uint32_t v = lane < (blockDim.x >> 5u) ? warp_sums[lane] : 0u;
        for (unsigned o = 1u; o < 32u; o <<= 1u) {
            const uint32_t y = __shfl_up_sync(kFull, v, o);
            if (lane >= o) v += y;
        }
        warp_sums[lane] = v;
    }
    __syncthreads();
    uint32_t run = x - sum + (wid > 0u ? warp_sums[wid - 1u] : 0u);
    for (uint32_t i = lo; i < hi; i++) {
        const uint32_t v = hist[i];
        hist[i] = run;
        run += v;
    }
    __syncthreads();
    if (threadIdx.x < kQueues) {
        bounds[threadIdx.x] = hist[threadIdx.x * tiles];
        counters[threadIdx.x] = 0u;
    }
    if (threadIdx.x == 0u) {
        bounds[kQueues] = count;
        unsigned long long acc = 0ull;
        for (unsigned q = 0u; q < kQueues; q++) {
            work[q] = acc;
            acc += bins[q];
        }
        work[kQueues] = acc;
    }
}

__global__ void __launch_bounds__(kTileThreads) bucket_scatter(const uint4* heads, uint32_t base, uint32_t count,
                                                               uint32_t tiles, const uint32_t* hist,
                                                               uint32_t* order) {
    __shared__ uint32_t off[kQueues];
    for (unsigned q = threadIdx.x; q < kQueues; q += blockDim.x) {
        off[q] = hist[q * tiles + blockIdx.x];
    }
    __syncthreads();
    const uint32_t lo = blockIdx.x * kBucketTile, hi = min(count, lo + kBucketTile);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t at = atomicAdd(&off[node_count(heads, base + i)], 1u);
        order[at] = base + i;
    }
}

}  // namespace

size_t bucket_bytes(size_t count) {
    const size_t tiles = (count + kBucketTile - 1u) / kBucketTile;
    return align256(kQueues * 4u) + align256((kQueues + 1u) * 4u) + align256((kQueues + 1u) * 8u) +
           align256(kQueues * 8u) + align256(kQueues * tiles * 4u) + align256(count * 4u);
}

Buckets bucket_layout(void* area, size_t count) {
    Buckets b;
    const size_t tiles = (count + kBucketTile - 1u) / kBucketTile;
    char* p = static_cast<char*>(area);
    b.counters = reinterpret_cast<uint32_t*>(p);
    p += align256(kQueues * 4u);
    b.bounds = reinterpret_cast<uint32_t*>(p);
    p += align256((kQueues + 1u) * 4u);
    b.work = reinterpret_cast<unsigned long long*>(p);
    p += align256((kQueues + 1u) * 8u);
    b.bins = reinterpret_cast<unsigned long long*>(p);
    p += align256(kQueues * 8u);
    b.hist = reinterpret_cast<uint32_t*>(p);
    p += align256(kQueues * tiles * 4u);
    b.order = reinterpret_cast<uint32_t*>(p);
    b.tiles = (uint32_t)tiles;
    return b;
}

cudaError_t launch_bucket(const uint4* heads, uint32_t base, uint32_t count, const Buckets& b,
                          cudaStream_t stream) {
    cudaError_t e;
    if (count == 0u) {
        // Every queue empty.
        if ((e = cudaMemsetAsync(b.counters, 0, kQueues * 4u, stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b.bounds, 0, (kQueues + 1u) * 4u, stream)) != cudaSuccess) return e;
        return cudaMemsetAsync(b.work, 0, (kQueues + 1u) * 8u, stream);
    }
    if ((e = cudaMemsetAsync(b.bins, 0, kQueues * 8u, stream)) != cudaSuccess) return e;
    bucket_count<<<b.tiles, kTileThreads, 0, stream>>>(heads, base, count, b.tiles, b.hist, b.bins);
    bucket_scan<<<1, kScanThreads, 0, stream>>>(b.hist, b.tiles, count, b.bounds, b.work, b.bins, b.counters);
    bucket_scatter<<<b.tiles, kTileThreads, 0, stream>>>(heads, base, count, b.tiles, b.hist, b.order);
    return cudaGetLastError();
}

}  // namespace cek
