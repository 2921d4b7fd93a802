// The rung audit of one batch on the device, from its resident results:
// Audit::note over every trial (src/rungs.rs:510-525) and GenAudit::of over
// the audit rows (src/rungs.rs:319-345), the rows that record_rungs files
// (src/storage.rs:672-708): trials of creatures flagged AUDIT whose trace is
// not empty, in batch order. Each rung's class A (reached the 5 s bar) and
// class B get Sums::add's float64 sums (src/rungs.rs:286-299) of the six
// features (src/rungs.rs:224-235), and class A's feature words are listed.
//
// The sums are order dependent in float64, so they are added in row order,
// one thread a sum: the rows are first compacted in order (a count, a scan of
// the tiles' counts and an ordered write), then a block walks them in chunks,
// the chunk's features staged in shared memory, and each of its 172 threads
// (2 rungs x 2 classes x (count, 6 sums, 36 products)) adds its own column.
// Built with no fused multiply-adds, so every sum equals the reference's to
// the bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/creature_engine.h"
#include "host_model.h"

namespace {

constexpr uint32_t kAudit = 1u, kExempt = 2u;  // rungs::AUDIT, rungs::EXEMPT (src/rungs.rs:18-22)
constexpr unsigned kFeatures = 6u;
constexpr unsigned kTile = 256u;                 // threads of the count and write kernels
constexpr unsigned kColumns = 1u + kFeatures + kFeatures * kFeatures;  // count, sums, products: 43
constexpr unsigned kGroup = 64u;                 // threads a (rung, class) group of the sum kernel
constexpr unsigned kChunk = 4u * kGroup;         // rows staged at a time: one a thread

__device__ __forceinline__ uint32_t bits(float f) { return __float_as_uint(f); }

// The seven trace words of a result (RungTrace, src/creature_kernel.rs:
// 120-218).
struct Trace {
    uint32_t w[7];
    __device__ explicit Trace(const ce_result& r)
        : w{bits(r.contact_hi), bits(r.lift_hi), bits(r.ground_hi), bits(r.previous_center_y),
            bits(r.vertical_extremum), bits(r.vertical_trend), bits(r.gait_turns)} {}
    __device__ uint32_t steps() const { return w[2] >> 16; }
    __device__ uint32_t stopped_by() const { return (w[2] >> 6) & 3u; }
};

// IEEE half to single precision (exact).
__device__ float half_to_float(uint32_t h) {
    const uint32_t sign = (h >> 15) << 31, exponent = (h >> 10) & 0x1fu, mantissa = h & 0x3ffu;
    uint32_t out;
    if (exponent == 0u && mantissa == 0u) {
        out = sign;
    } else if (exponent == 0u) {
        const uint32_t shift = (uint32_t)__clz(mantissa) - 21u;
        out = sign | ((113u - shift) << 23) | (((mantissa << shift) & 0x3ffu) << 13);
    } else if (exponent == 31u) {
        out = sign | 0x7f800000u | (mantissa ? (0x00400000u | (mantissa << 13)) : 0u);
    } else {
        out = sign | ((exponent + 112u) << 23) | (mantissa << 13);
    }
    return __uint_as_float(out);
}

// Single to half precision, rounding to nearest even (the kernel's
// conversion, src/creature_kernel.rs:220-260).
__device__ uint32_t float_to_half(float v) {
    const uint32_t b = __float_as_uint(v);
    const uint32_t sign = (b >> 16) & 0x8000u, mantissa = b & 0x7fffffu;
    const int exponent = (int)((b >> 23) & 0xffu);
    if (exponent == 0xff) return sign | 0x7c00u | (mantissa ? 0x200u : 0u);
    const int e = exponent - 127 + 15;
    if (e >= 31) return sign | 0x7c00u;
    if (e <= 0) {
        if (e < -10) return sign;
        const uint32_t m = mantissa | 0x800000u, shift = (uint32_t)(14 - e);
        const uint32_t half = 1u << (shift - 1u), rest = m & ((1u << shift) - 1u);
        uint32_t out = m >> shift;
        if (rest > half || (rest == half && (out & 1u))) out += 1u;
        return sign | out;
    }
    const uint32_t rest = mantissa & 0x1fffu;
    uint32_t out = ((uint32_t)e << 10) | (mantissa >> 13);
    if (rest > 0x1000u || (rest == 0x1000u && (out & 1u))) out += 1u;
    return sign | out;
}

__device__ __forceinline__ float half_of(uint32_t w, bool high) { return half_to_float(high ? w >> 16 : w & 0xffffu); }

struct Inputs {
    const ce_result* results;
    const ce_genome* genomes;
    const ce_muscle_gene* muscles;
    const float* bars;
    size_t count;
    size_t tile;  // creatures a block of the count and write kernels
};

__device__ __forceinline__ bool is_row(const Inputs& in, size_t i, const Trace& t) {
    return (in.genomes[i].flags & kAudit) != 0u && t.steps() != 0u;
}

// Audit::note's tallies and the audit rows of each block's tile.
__global__ void __launch_bounds__(kTile) audit_count_kernel(const Inputs in, uint32_t* tile_rows, ce_audit* out) {
    __shared__ unsigned long long s_steps, s_stops[3];
    __shared__ unsigned s_rows;
    if (threadIdx.x == 0u) {
        s_steps = 0ull;
        s_stops[0] = s_stops[1] = s_stops[2] = 0ull;
        s_rows = 0u;
    }
    __syncthreads();
    const size_t lo = (size_t)blockIdx.x * in.tile, hi = min(lo + in.tile, in.count);
    unsigned long long steps = 0ull, stops[3] = {0ull, 0ull, 0ull};
    unsigned rows = 0u;
    for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const ce_result& r = in.results[i];
        const Trace t(r);
        steps += t.steps();
        if (r.screened > 0.0f) {
            const uint32_t k = t.stopped_by();
            stops[k == 1u ? 0 : (k == 2u ? 1 : 2)] += 1ull;
        }
        rows += is_row(in, i, t) ? 1u : 0u;
    }
    atomicAdd(&s_steps, steps);
    for (int k = 0; k < 3; k++) atomicAdd(&s_stops[k], stops[k]);
    atomicAdd(&s_rows, rows);
    __syncthreads();
    if (threadIdx.x == 0u) {
        tile_rows[blockIdx.x] = s_rows;
        atomicAdd(reinterpret_cast<unsigned long long*>(&out->steps), s_steps);
        for (int k = 0; k < 3; k++) atomicAdd(reinterpret_cast<unsigned long long*>(&out->stops[k]), s_stops[k]);
    }
}

// Exclusive offsets of the tiles' rows and the batch's totals: one block of
// 1024 threads, two tiles a thread (at most 2048 tiles).
constexpr unsigned kMaxTiles = 2048u;
__global__ void __launch_bounds__(1024) audit_scan_kernel(uint32_t* tile_rows, unsigned tiles, size_t count,
                                                           ce_audit* out) {
    __shared__ uint32_t warp_sum[32];
    const unsigned t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const uint32_t x0 = 2u * t < tiles ? tile_rows[2u * t] : 0u, x1 = 2u * t + 1u < tiles ? tile_rows[2u * t + 1u] : 0u;
    const uint32_t mine = x0 + x1;
    uint32_t incl = mine;
    for (unsigned d = 1u; d < 32u; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31u) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0u) {
        uint32_t w = warp_sum[lane], wi = w;
        for (unsigned d = 1u; d < 32u; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += y;
        }
        warp_sum[lane] = wi - w;  // exclusive
        if (lane == 31u) {
            out->rows = wi;
            out->creatures = count;
        }
    }
    __syncthreads();
    const uint32_t before = warp_sum[warp] + incl - mine;
    if (2u * t < tiles) tile_rows[2u * t] = before;
    if (2u * t + 1u < tiles) tile_rows[2u * t + 1u] = before + x0;
}

// Each tile writes its rows' indices in order: a block-wide ordered
// compaction, 256 creatures at a time.
__global__ void __launch_bounds__(kTile) audit_write_kernel(const Inputs in, const uint32_t* tile_rows,
                                                            uint32_t* row_index) {
    __shared__ unsigned warp_rows[kTile / 32u];
    __shared__ unsigned base;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0u) base = tile_rows[blockIdx.x];
    const size_t lo = (size_t)blockIdx.x * in.tile, hi = min(lo + in.tile, in.count);
    for (size_t start = lo; start < hi; start += blockDim.x) {
        const size_t i = start + threadIdx.x;
        const bool row = i < hi && is_row(in, i, Trace(in.results[i]));
        const unsigned ballot = __ballot_sync(0xffffffffu, row);
        __syncthreads();  // `base` and `warp_rows` of the last round are read
        if (lane == 0u) warp_rows[warp] = __popc(ballot);
        __syncthreads();
        unsigned before = base;
        for (unsigned k = 0u; k < warp; k++) before += warp_rows[k];
        if (row) row_index[before + __popc(ballot & ((1u << lane) - 1u))] = (uint32_t)i;
        __syncthreads();
        if (threadIdx.x == 0u) {
            unsigned all = 0u;
            for (unsigned k = 0u; k < blockDim.x / 32u; k++) all += warp_rows[k];
            base += all;
        }
    }
}

// GenAudit::of over the compacted rows, in order. Four groups of 64
// threads, one a (rung, class): per chunk of 256 rows each row's features
// are staged once as float64 (with a constant 1 in slot 6), each group gets
// the chunk's rows of its class in row order, and thread c < 43 of a group
// adds its column over them: c = 0 the count, 1-6 feature c - 1 times the
// constant 1 (an exact product, so the sum is Sums::add's), 7-42 the product
// of features (c - 7) / 6 and (c - 7) % 6. Every column is one row-ordered
// chain of float64 multiply and add, with no branch on the row.
__global__ void __launch_bounds__(kChunk) audit_sum_kernel(const Inputs in, const uint32_t* row_index, ce_audit* out,
                                                           uint16_t* a_words, size_t a_cap) {
    __shared__ double feat[kChunk][2][kFeatures + 1u];
    __shared__ uint16_t list[4][kChunk];
    __shared__ unsigned warp_count[4][kChunk / 32u], list_len[4];
    const unsigned t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const unsigned group = t / kGroup, col = t % kGroup, r = group >> 1, k = group & 1u;
    const unsigned fa = col == 0u ? kFeatures : (col <= kFeatures ? col - 1u : (col - 1u - kFeatures) / kFeatures);
    const unsigned fb = col <= kFeatures ? kFeatures : (col - 1u - kFeatures) % kFeatures;
    const uint32_t rows = out->rows;
    double acc = 0.0;
    unsigned long long n = 0ull;
    for (uint32_t start = 0u; start < rows; start += kChunk) {
        const uint32_t len = min(kChunk, rows - start);
        __syncthreads();  // the last chunk's lists and features are read
        unsigned cls[2] = {2u, 2u};  // per rung: 0 class A, 1 class B, 2 neither
        if (t < len) {
            const uint32_t i = row_index[start + t];
            const ce_result& res = in.results[i];
            const Trace tr(res);
            const ce_genome& g = in.genomes[i];
            const float bar = in.bars[i];
            const bool counted = (g.flags & kExempt) == 0u && isfinite(bar);
            const bool pass3 = res.screen_x >= bar;
            const float period = g.muscle_count > 0u ? in.muscles[g.muscle_start].period : 0.0f;
            const float ph = half_to_float(float_to_half(period));
            for (unsigned rr = 0u; rr < 2u; rr++) {
                const float f[kFeatures] = {half_of(tr.w[rr / 2u], rr % 2u == 1u), half_of(tr.w[3], rr == 1u),
                                            half_of(tr.w[4u + rr], false), half_of(tr.w[6], rr == 1u),
                                            half_of(tr.w[4u + rr], true), ph};
                bool finite = true;
#pragma unroll
                for (unsigned x = 0u; x < kFeatures; x++) {
                    feat[t][rr][x] = (double)f[x];
                    finite = finite && isfinite(f[x]);
                }
                feat[t][rr][kFeatures] = 1.0;
                // rungs::RUNG_STEPS: R1 at step 60, R2 at 150.
                cls[rr] = (counted && tr.steps() > (rr == 0u ? 60u : 150u) && finite) ? (pass3 ? 0u : 1u) : 2u;
            }
        }
        // Each group's rows in row order: a ballot a warp, then the warps'
        // counts before this one.
        unsigned ballot[4];
#pragma unroll
        for (unsigned q = 0u; q < 4u; q++) {
            ballot[q] = __ballot_sync(0xffffffffu, cls[q >> 1] == (q & 1u));
            if (lane == 0u) warp_count[q][warp] = __popc(ballot[q]);
        }
        __syncthreads();
#pragma unroll
        for (unsigned q = 0u; q < 4u; q++) {
            if ((ballot[q] >> lane) & 1u) {
                unsigned before = 0u;
                for (unsigned v = 0u; v < warp; v++) before += warp_count[q][v];
                list[q][before + __popc(ballot[q] & ((1u << lane) - 1u))] = (uint16_t)t;
            }
        }
        if (t < 4u) {
            unsigned all = 0u;
            for (unsigned v = 0u; v < kChunk / 32u; v++) all += warp_count[t][v];
            list_len[t] = all;
        }
        __syncthreads();
        const unsigned L = list_len[group];
        if (col < kColumns) {
            if (col > 0u) {
#pragma unroll 4
                for (unsigned j = 0u; j < L; j++) {
                    const unsigned q = list[group][j];
                    acc += feat[q][r][fa] * feat[q][r][fb];
                }
            }
            if (k == 0u && a_words) {
                // Class A's feature words, the group's threads sharing the rows.
                for (unsigned j = col; j < L; j += kColumns) {
                    if (n + j >= a_cap) break;
                    const unsigned q = list[group][j];
                    uint16_t* w = a_words + ((size_t)r * a_cap + n + j) * kFeatures;
                    for (unsigned x = 0u; x < kFeatures; x++) w[x] = (uint16_t)float_to_half((float)feat[q][r][x]);
                }
            }
        }
        n += L;
    }
    if (col < kColumns) {
        ce_audit_sums& s = k == 0u ? out->a[r] : out->b[r];
        if (col == 0u) s.n = n;
        else if (col <= kFeatures) s.sum[col - 1u] = acc;
        else s.xx[(col - 1u - kFeatures) / kFeatures][(col - 1u - kFeatures) % kFeatures] = acc;
    }
}

}  // namespace

extern "C" size_t ce_audit_scratch_bytes(size_t count) {
    return 4096ull * sizeof(uint32_t) + count * sizeof(uint32_t);
}

extern "C" ce_status ce_audit_device(const ce_result* results, const ce_genome* genomes, const ce_muscle_gene* muscles,
                                     const float* bars, size_t count, void* scratch, size_t scratch_bytes,
                                     ce_audit* out, uint16_t* a_words, size_t a_cap, void* stream) {
    if (!out || (count && (!results || !genomes || !muscles || !bars || !scratch))) {
        ce::set_error("ce_audit_device: null argument");
        return CE_ERR_INVALID;
    }
    if (count > 0xffffffffull) {
        ce::set_error("ce_audit_device: at most 2^32 - 1 trials a call");
        return CE_ERR_INVALID;
    }
    if (scratch_bytes < ce_audit_scratch_bytes(count)) {
        ce::set_error("ce_audit_device: scratch smaller than ce_audit_scratch_bytes");
        return CE_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(ce_audit), st);
    if (e != cudaSuccess) {
        ce::set_error(std::string("ce_audit_device: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    if (count == 0) return CE_OK;  // every tally and sum is zero
    uint32_t* tile_rows = static_cast<uint32_t*>(scratch);
    uint32_t* row_index = tile_rows + 4096;
    const unsigned tiles = (unsigned)std::min<size_t>(148u * 8u, std::max<size_t>(1u, (count + kTile - 1u) / kTile));
    Inputs in{results, genomes, muscles, bars, count, (count + tiles - 1u) / tiles};
    if (in.tile == 0u) in.tile = 1u;
    audit_count_kernel<<<tiles, kTile, 0, st>>>(in, tile_rows, out);
    audit_scan_kernel<<<1, 1024, 0, st>>>(tile_rows, tiles, count, out);
    audit_write_kernel<<<tiles, kTile, 0, st>>>(in, tile_rows, row_index);
    audit_sum_kernel<<<1, kChunk, 0, st>>>(in, row_index, out, a_words, a_cap);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        ce::set_error(std::string("ce_audit_device: launch: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    return CE_OK;
}
