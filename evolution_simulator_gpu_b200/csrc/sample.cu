// Gaussian samples of parent genomes on the device: the ask step of the
// gradient-refined search, on the optimizer's parameter vector of a body
// (src/qd.rs:2700-2770: per node x, y, diameter, friction; per bone rest
// length, joint range, organ mass and place; one log period; per muscle the
// anchors, short and long length, phase, duty, log stiffness and reset
// phase), back to genes with apply_parameters' clamps (src/qd.rs:2773-2811)
// and the workload's diameter and friction ranges, as repair holds them
// (src/evolution.rs:1230-1234).
//
// Sample g (a global index) is a child of parent g mod P. The parents'
// genes are packed in order from row 0, so the children [first, first +
// count) tile them: child row R is parent row R mod T (T the parents' rows
// of that kind), and nothing but the parents and a few totals is needed to
// place a row. Every move is a normal deviate drawn from a counter-based
// hash of (seed, g, gene kind, row of the creature, field): a sample does not
// depend on which range of samples a call draws.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/creature_engine.h"
#include "host_model.h"

namespace {

constexpr float kMaxBone = 2.0f, kMaxStroke = 2.0f, kMinPeriod = 0.2f;  // physics::Limits::DEFAULT
constexpr float kJointLimit = 2.0943951f;                             // 120 degrees (src/evolution.rs:92)
constexpr float kDiameterLo = 0.06f, kDiameterHi = 0.12f, kFrictionLo = 0.0f, kFrictionHi = 1.0f;

// SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// A standard normal deviate for (seed, sample, kind, row, field), by the
// Box-Muller transform of two 24-bit uniforms of one hash.
__device__ __forceinline__ float normal(uint64_t seed, uint64_t g, uint32_t kind, uint32_t row, uint32_t field) {
    const uint64_t h = mix64(mix64(seed * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull) ^
                             (g * 0xd1342543de82ef95ull + ((uint64_t)kind << 48) + ((uint64_t)row << 8) + field));
    const float u1 = (float)((h >> 40) + 1u) * (1.0f / 16777216.0f);  // (0, 1]
    const float u2 = (float)(h & 0xffffffu) * (1.0f / 16777216.0f);   // [0, 1)
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float wrap01(float x) {
    const float r = x - floorf(x);
    return r >= 1.0f ? 0.0f : r;
}

struct SampleArgs {
    const ce_node_gene* nodes;
    const ce_bone_gene* bones;
    const ce_muscle_gene* muscles;
    const ce_genome* genomes;  // the parents'
    const float* strength;     // the parents' (may be NULL)
    uint32_t parents;
    uint64_t first, seed, first_id;
    uint64_t tn, tb, tm;        // the parents' rows
    uint64_t base_n, base_b, base_m;  // global row of the first child's first row
    float sigma;
};

// The parent whose rows of a kind hold row `local` (starts ascending).
template <int KIND>
__device__ __forceinline__ uint32_t owner(const ce_genome* gs, uint32_t parents, uint64_t local) {
    uint32_t lo = 0, hi = parents;  // start(lo) <= local < start(hi)
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) / 2u;
        const uint32_t s = KIND == 0 ? gs[mid].node_start : (KIND == 1 ? gs[mid].bone_start : gs[mid].muscle_start);
        if (s <= local) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    // Skip parents with no rows of this kind that share the start.
    for (;;) {
        const uint32_t n = KIND == 0 ? gs[lo].node_count : (KIND == 1 ? gs[lo].bone_count : gs[lo].muscle_count);
        const uint32_t s = KIND == 0 ? gs[lo].node_start : (KIND == 1 ? gs[lo].bone_start : gs[lo].muscle_start);
        if (local < (uint64_t)s + n || lo + 1u >= parents) return lo;
        lo++;
    }
}

__global__ void sample_genomes(const SampleArgs a, size_t count, ce_genome* out) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < count; c += (size_t)gridDim.x * blockDim.x) {
        const uint64_t g = a.first + c, k = g / a.parents;
        const ce_genome pg = a.genomes[g % a.parents];
        ce_genome o = pg;
        o.node_start = (uint32_t)(k * a.tn + pg.node_start - a.base_n);
        o.bone_start = (uint32_t)(k * a.tb + pg.bone_start - a.base_b);
        o.muscle_start = (uint32_t)(k * a.tm + pg.muscle_start - a.base_m);
        o.id = a.first_id + g;
        out[c] = o;
    }
}

__global__ void sample_nodes(const SampleArgs a, size_t rows, ce_node_gene* out) {
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < rows; r += (size_t)gridDim.x * blockDim.x) {
        const uint64_t R = a.base_n + r, k = R / a.tn, local = R - k * a.tn;
        const uint32_t p = owner<0>(a.genomes, a.parents, local);
        const uint64_t g = k * a.parents + p;
        const uint32_t row = (uint32_t)(local - a.genomes[p].node_start);
        ce_node_gene n = a.nodes[local];
        n.x += a.sigma * normal(a.seed, g, 0u, row, 0u);
        n.y = fmaxf(n.y + a.sigma * normal(a.seed, g, 0u, row, 1u), 0.0f);
        n.diameter = clampf(n.diameter + a.sigma * normal(a.seed, g, 0u, row, 2u), kDiameterLo, kDiameterHi);
        n.friction = clampf(n.friction + a.sigma * normal(a.seed, g, 0u, row, 3u), kFrictionLo, kFrictionHi);
        out[r] = n;
    }
}

__global__ void sample_bones(const SampleArgs a, size_t rows, ce_bone_gene* out) {
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < rows; r += (size_t)gridDim.x * blockDim.x) {
        const uint64_t R = a.base_b + r, k = R / a.tb, local = R - k * a.tb;
        const uint32_t p = owner<1>(a.genomes, a.parents, local);
        const uint64_t g = k * a.parents + p;
        const uint32_t row = (uint32_t)(local - a.genomes[p].bone_start);
        ce_bone_gene b = a.bones[local];
        b.rest_length = clampf(b.rest_length + a.sigma * normal(a.seed, g, 1u, row, 0u), 0.03f, kMaxBone);
        b.min_angle = clampf(b.min_angle + a.sigma * normal(a.seed, g, 1u, row, 1u), -kJointLimit, 0.0f);
        b.max_angle = clampf(b.max_angle + a.sigma * normal(a.seed, g, 1u, row, 2u), 0.0f, kJointLimit);
        b.organ_mass = fmaxf(b.organ_mass + a.sigma * normal(a.seed, g, 1u, row, 3u), 0.0f);
        b.organ_at = clampf(b.organ_at + a.sigma * normal(a.seed, g, 1u, row, 4u), 0.0f, 1.0f);
        out[r] = b;
    }
}

__global__ void sample_muscles(const SampleArgs a, size_t rows, ce_muscle_gene* out, float* strength) {
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < rows; r += (size_t)gridDim.x * blockDim.x) {
        const uint64_t R = a.base_m + r, k = R / a.tm, local = R - k * a.tm;
        const uint32_t p = owner<2>(a.genomes, a.parents, local);
        const uint64_t g = k * a.parents + p;
        const ce_genome& pg = a.genomes[p];
        const uint32_t row = (uint32_t)(local - pg.muscle_start);
        ce_muscle_gene m = a.muscles[local];
        // One log period a body: every muscle's period moves by one factor.
        const float base = fmaxf(a.muscles[pg.muscle_start].period, 1e-3f);
        const float scale = clampf(expf(logf(base) + a.sigma * normal(a.seed, g, 3u, 0u, 0u)), kMinPeriod, 10.0f) / base;
        m.anchor_a = clampf(m.anchor_a + a.sigma * normal(a.seed, g, 2u, row, 0u), 0.0f, 1.0f);
        m.anchor_b = clampf(m.anchor_b + a.sigma * normal(a.seed, g, 2u, row, 1u), 0.0f, 1.0f);
        m.short_len = clampf(m.short_len + a.sigma * normal(a.seed, g, 2u, row, 2u), 0.01f, 0.8f * kMaxStroke);
        m.long_len = clampf(m.long_len + a.sigma * normal(a.seed, g, 2u, row, 3u), m.short_len, kMaxStroke);
        m.period = clampf(m.period * scale, kMinPeriod, 10.0f);
        m.phase = wrap01(m.phase + a.sigma * normal(a.seed, g, 2u, row, 4u));
        m.duty = clampf(m.duty + a.sigma * normal(a.seed, g, 2u, row, 5u), 0.05f, 0.95f);
        m.stiffness =
            clampf(expf(logf(fmaxf(m.stiffness, 1e-3f)) + a.sigma * normal(a.seed, g, 2u, row, 6u)), 1.0f, 120.0f);
        m.reset = wrap01(m.reset + a.sigma * normal(a.seed, g, 2u, row, 7u));
        out[r] = m;
        if (strength) strength[r] = a.strength ? a.strength[local] : 1.0f;
    }
}

unsigned grid_of(size_t n) { return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148u * 16u)); }

}  // namespace

// Rows of each kind of samples [first, first + count) of `parents` parents
// with the given (host) genomes.
extern "C" ce_status ce_sample_rows(const ce_genome* parent_genomes, size_t parents, uint64_t first, size_t count,
                                   size_t* nodes, size_t* bones, size_t* muscles) {
    if (!parent_genomes || !parents || !nodes || !bones || !muscles) {
        ce::set_error("ce_sample_rows: null argument or no parents");
        return CE_ERR_INVALID;
    }
    uint64_t t[3] = {0, 0, 0};
    std::vector<uint64_t> pre(3 * (parents + 1), 0);
    for (size_t p = 0; p < parents; p++) {
        const ce_genome& g = parent_genomes[p];
        pre[3 * (p + 1)] = pre[3 * p] + g.node_count;
        pre[3 * (p + 1) + 1] = pre[3 * p + 1] + g.bone_count;
        pre[3 * (p + 1) + 2] = pre[3 * p + 2] + g.muscle_count;
    }
    for (int k = 0; k < 3; k++) t[k] = pre[3 * parents + k];
    auto offset = [&](uint64_t g, int k) { return (g / parents) * t[k] + pre[3 * (g % parents) + k]; };
    *nodes = (size_t)(offset(first + count, 0) - offset(first, 0));
    *bones = (size_t)(offset(first + count, 1) - offset(first, 1));
    *muscles = (size_t)(offset(first + count, 2) - offset(first, 2));
    // A sample's gene starts are 32-bit, counted from the call's first row.
    if (*nodes > 0xffffffffull || *bones > 0xffffffffull || *muscles > 0xffffffffull || count > 0xffffffffull) {
        ce::set_error("ce_sample_rows: more than 2^32 - 1 gene rows of a kind in one call; draw fewer samples a call");
        return CE_ERR_INVALID;
    }
    return CE_OK;
}

// Samples [first, first + count) of the parents on the device (all gene
// pointers device pointers; `parents->genomes` packed in order from row 0;
// the outputs sized by ce_sample_rows); asynchronous on `stream` after a
// small synchronous read of the parents' genomes.
extern "C" ce_status ce_sample_device(const ce_population* parents, uint64_t first, size_t count, float sigma,
                                     uint64_t seed, uint64_t first_id, ce_node_gene* nodes, ce_bone_gene* bones,
                                     ce_muscle_gene* muscles, float* strength, ce_genome* genomes, void* stream) {
    if (!parents || !parents->count || !parents->genomes || !parents->nodes || !parents->bones ||
        !parents->muscles || !genomes || (count && (!nodes || !muscles))) {
        ce::set_error("ce_sample_device: null argument or no parents");
        return CE_ERR_INVALID;
    }
    const size_t P = parents->count;
    std::vector<ce_genome> hg(P);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(hg.data(), parents->genomes, P * sizeof(ce_genome), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ce::set_error(std::string("ce_sample_device: reading the parents: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    uint64_t at[3] = {0, 0, 0};
    for (size_t p = 0; p < P; p++) {
        const ce_genome& g = hg[p];
        if (g.node_start != at[0] || g.bone_start != at[1] || g.muscle_start != at[2]) {
            ce::set_error("ce_sample_device: the parents' genes must be packed in order from row 0");
            return CE_ERR_INVALID;
        }
        at[0] += g.node_count;
        at[1] += g.bone_count;
        at[2] += g.muscle_count;
    }
    if (!at[0] || !at[1] || !at[2]) {
        ce::set_error("ce_sample_device: the parents have no nodes, bones or muscles");
        return CE_ERR_INVALID;
    }
    SampleArgs a;
    a.nodes = parents->nodes;
    a.bones = parents->bones;
    a.muscles = parents->muscles;
    a.genomes = parents->genomes;
    a.strength = parents->strength_scale;
    a.parents = (uint32_t)P;
    a.first = first;
    a.seed = seed;
    a.first_id = first_id;
    a.tn = at[0];
    a.tb = at[1];
    a.tm = at[2];
    a.sigma = sigma;
    const ce_genome& f = hg[first % P];
    a.base_n = (first / P) * a.tn + f.node_start;
    a.base_b = (first / P) * a.tb + f.bone_start;
    a.base_m = (first / P) * a.tm + f.muscle_start;
    size_t rn = 0, rb = 0, rm = 0;
    ce_status s = ce_sample_rows(hg.data(), P, first, count, &rn, &rb, &rm);
    if (s != CE_OK) return s;
    if (count == 0) return CE_OK;
    sample_genomes<<<grid_of(count), 256, 0, st>>>(a, count, genomes);
    if (rn) sample_nodes<<<grid_of(rn), 256, 0, st>>>(a, rn, nodes);
    if (rb) sample_bones<<<grid_of(rb), 256, 0, st>>>(a, rb, bones);
    if (rm) sample_muscles<<<grid_of(rm), 256, 0, st>>>(a, rm, muscles, strength);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        ce::set_error(std::string("ce_sample_device: launch: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    return CE_OK;
}
