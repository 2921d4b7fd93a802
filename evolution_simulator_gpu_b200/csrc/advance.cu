// The creature kernel family's launchers: persistent warps, one creature
// per lane, compiled ahead of time for sm_100a per world, node-row class,
// recording switch and step rate.
#include <cuda_runtime.h>

#include <cstdio>
#include <type_traits>

#include "trial.cuh"

namespace cek {

// Shared memory carveout (percent of the largest) that fits `blocks`
// blocks of `smem` bytes each, leaving the rest of the multiprocessor's
// memory to the L1 cache that holds the creatures' constant lines.
static int carveout_for(size_t smem, int blocks) {
    const size_t need = (smem + 1024u) * (size_t)blocks;
    const size_t full = 228u * 1024u;
    int pct = (int)((need * 100u + full - 1u) / full);
    return pct < 1 ? 1 : (pct > 100 ? 100 : pct);
}

// The kernel of a world, recording switch and step rate.
template <class W, bool RECORD, int RATE>
constexpr auto kernel_of() {
    return advance_kernel<W, RECORD, RATE>;
}

template <class W, bool RECORD, int RATE>
static cudaError_t occupancy_one(unsigned rows, unsigned mm, unsigned block, int* blocks) {
    auto kern = kernel_of<W, RECORD, RATE>();
    const size_t smem = smem_bytes(rows, mm, block);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, kern, (int)block, smem);
}

template <class W, bool RECORD, int RATE>
static cudaError_t launch_one(const LaunchSpec& s, const KernelArgs& a, const ce_params& p, const W& w) {
    auto kern = kernel_of<W, RECORD, RATE>();
    const size_t smem = smem_bytes(s.rows, s.mm, s.block);
    int blocks = 0;
    cudaError_t e = occupancy_one<W, RECORD, RATE>(s.rows, s.mm, s.block, &blocks);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             carveout_for(smem, blocks > 0 ? blocks : 1));
    if (e != cudaSuccess) return e;
    kern<<<s.grid, s.block, smem, s.stream>>>(a, p, w);
    return cudaGetLastError();
}

// The compiled worlds. Any other world runs on the run-time-world kernel.
template <bool RECORD, int RATE, class F>
static cudaError_t by_world(uint32_t flags, F&& f) {
    switch (flags) {
        case kWorldCalm: return f(StaticWorld<kWorldCalm>{});
        case kWorldEffects: return f(StaticWorld<kWorldEffects>{});
        case kWorldEffectsQuake: return f(StaticWorld<kWorldEffectsQuake>{});
        case kWorldAll: return f(StaticWorld<kWorldAll>{});
        default: return f(RuntimeWorld{flags});
    }
}

template <bool RECORD, int RATE>
static cudaError_t dispatch(const LaunchSpec& s, const KernelArgs& a, const ce_params& p) {
    return by_world<RECORD, RATE>(s.flags, [&](auto w) { return launch_one<decltype(w), RECORD, RATE>(s, a, p, w); });
}

cudaError_t launch_advance(const LaunchSpec& s, const KernelArgs& a, const ce_params& p) {
    if (s.rows < 2 || s.rows > CE_MAX_NODES || s.mm > CE_MAX_MUSCLES || a.rows != s.rows || a.mm != s.mm) {
        return cudaErrorInvalidValue;
    }
    if (s.rate == 60) {
        return s.record ? dispatch<true, 60>(s, a, p) : dispatch<false, 60>(s, a, p);
    }
    if (s.rate == 120) {
        return s.record ? dispatch<true, 120>(s, a, p) : dispatch<false, 120>(s, a, p);
    }
    return cudaErrorInvalidValue;
}

cudaError_t advance_reserve_smem(unsigned rows, unsigned mm, uint32_t flags, bool record, int rate, unsigned block) {
    const int smem = (int)smem_bytes(rows, mm, block);
    auto go = [&](auto rec_tag, auto rate_tag) -> cudaError_t {
        constexpr bool R = decltype(rec_tag)::value;
        constexpr int RT = decltype(rate_tag)::value;
        return by_world<R, RT>(flags, [&](auto w) {
            return cudaFuncSetAttribute(kernel_of<decltype(w), R, RT>(),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        });
    };
    using Tt = std::true_type;
    using Ft = std::false_type;
    using R60 = std::integral_constant<int, 60>;
    using R120 = std::integral_constant<int, 120>;
    if (rate == 60) return record ? go(Tt{}, R60{}) : go(Ft{}, R60{});
    if (rate == 120) return record ? go(Tt{}, R120{}) : go(Ft{}, R120{});
    return cudaErrorInvalidValue;
}

cudaError_t advance_occupancy(unsigned rows, unsigned mm, uint32_t flags, bool record, int rate, unsigned block,
                              int* blocks) {
    auto go = [&](auto rec_tag, auto rate_tag) -> cudaError_t {
        constexpr bool R = decltype(rec_tag)::value;
        constexpr int RT = decltype(rate_tag)::value;
        return by_world<R, RT>(flags, [&](auto w) { return occupancy_one<decltype(w), R, RT>(rows, mm, block, blocks); });
    };
    using Tt = std::true_type;
    using Ft = std::false_type;
    using R60 = std::integral_constant<int, 60>;
    using R120 = std::integral_constant<int, 120>;
    if (rate == 60) return record ? go(Tt{}, R60{}) : go(Ft{}, R60{});
    if (rate == 120) return record ? go(Tt{}, R120{}) : go(Ft{}, R120{});
    return cudaErrorInvalidValue;
}

}  // namespace cek

namespace cek {
unsigned slot_lines(unsigned rows, unsigned mm, bool record) { return SlotLayout::make(rows, mm, record).lines; }

// Transpose of a rows x creatures matrix of float2 into creatures x rows,
// 32 x 32 tiles through shared memory (the extra column keeps the tile's
// column reads free of bank conflicts), both sides read and written as
// coalesced rows. Tiles are taken by a grid-stride loop.
__global__ void __launch_bounds__(256) frames_transpose(const float2* __restrict__ src, float2* __restrict__ dst,
                                                        size_t rows, uint32_t creatures) {
    __shared__ float2 tile[32][33];
    const size_t tiles_r = (rows + 31u) / 32u, tiles_c = (creatures + 31u) / 32u;
    for (size_t tile_i = blockIdx.x; tile_i < tiles_r * tiles_c; tile_i += gridDim.x) {
        const size_t r0 = (tile_i / tiles_c) * 32u, c0 = (tile_i % tiles_c) * 32u;
        for (unsigned y = threadIdx.y; y < 32u; y += 8u) {
            const size_t r = r0 + y, c = c0 + threadIdx.x;
            if (r < rows && c < creatures) tile[y][threadIdx.x] = src[r * creatures + c];
        }
        __syncthreads();
        for (unsigned y = threadIdx.y; y < 32u; y += 8u) {
            const size_t c = c0 + y, r = r0 + threadIdx.x;
            if (r < rows && c < creatures) dst[c * rows + r] = tile[threadIdx.x][y];
        }
        __syncthreads();
    }
}

cudaError_t launch_frames_to_creature_major(const float2* src, float2* dst, size_t rows, uint32_t creatures,
                                            cudaStream_t stream) {
    const size_t tiles = ((rows + 31u) / 32u) * ((creatures + 31u) / 32u);
    const unsigned grid = (unsigned)(tiles < 148u * 16u ? tiles : 148u * 16u);
    if (grid == 0u) return cudaSuccess;
    frames_transpose<<<grid, dim3(32, 8), 0, stream>>>(src, dst, rows, creatures);
    return cudaGetLastError();
}
}  // namespace cek
