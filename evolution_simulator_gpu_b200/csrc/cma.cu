// CMA-ES emitters on the device: the reference's CmaEmitter (src/qd.rs:
// 2130-2474) in both of its modes, one emitter per template body, ask and
// tell as kernels. An optimizer (CmaEmitter::optimizer) searches the
// parameter vector of write_parameters (src/qd.rs:2734-2770) in the physical
// units that Layout scales (src/qd.rs:2607-2699); a CMA-ME emitter
// (CmaEmitter::new) searches exploring_parameters (src/qd.rs:2504-2538),
// each coordinate normalised to about 0-1, with a rank-one step along its
// evolution path. A sample goes back to genes with apply_parameters or
// apply_exploring_parameters and the diameter and friction ranges that repair
// holds (src/evolution.rs:1230-1234).
//
// Ask: sample g (a global index, the ring slot of the reference's breeding
// stream) belongs to emitter g mod E; one thread draws its coordinates from
// Rng::stream(seed, generation, round, g) exactly as the reference's
// sample_into does (the generator is counter-based and integer, restated
// below), and writes its genes. The samples [first, first + count) tile the
// templates as the parents of ce_sample_device tile theirs, so
// ce_sample_rows sizes them.
// Tell: one block per emitter takes that emitter's samples among [first,
// first + count), keeps the finite ones above the failure score whose body
// plan is the template's, the best 1024 sorted best first (ties by sample
// index: the reference's unstable sort leaves their order open), and applies
// the mode's CMA-ES update.
//
// This file is built with IEEE division and square root and no fused
// multiply-adds, so each operation rounds as the reference's Rust f32 code
// does; its exp and ln are the device's (within a few units in the last
// place of the host C library's).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/creature_engine.h"
#include "host_model.h"

namespace {

constexpr float kMaxBone = 2.0f, kMaxStroke = 2.0f, kMinPeriod = 0.2f;  // physics::Limits::DEFAULT
constexpr float kJointLimit = 2.0943951f;                             // 120 degrees (src/evolution.rs:92)
constexpr float kFailed = -1.0e20f;          // evolution::FAILED (src/evolution.rs:18)
constexpr unsigned kMaxUpdate = 1024u;       // tell's MAX_UPDATE_SAMPLES (src/qd.rs:2233)
constexpr unsigned kTellBlock = 256u;
constexpr float kPathWeight = 0.3f;          // PATH_WEIGHT (src/qd.rs:2494)

// Layout's unit steps (src/qd.rs:2621-2636).
__constant__ float kNodeScales[4] = {0.02f, 0.02f, 0.005f, 0.03f};
__constant__ float kBoneScales[5] = {0.02f, 0.1f, 0.1f, 0.02f, 0.05f};
__constant__ float kMuscleScales[8] = {0.05f, 0.05f, 0.02f, 0.02f, 0.05f, 0.05f, 0.1f, 0.05f};
constexpr float kPeriodScale = 0.05f;

// ---- the reference's breeding streams (src/evolution.rs:455-600) ----
// SplitMix64's finaliser; a stream's key absorbs its coordinates one at a
// time; value (gene, draw) of a stream is the finaliser at key + counter x
// the golden ratio, counter = gene << 32 | draw; the cursor is gene 2^32 - 1.
__device__ __forceinline__ uint64_t finalize(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t keyed(uint64_t key, uint32_t gene, uint32_t draw) {
    const uint64_t counter = ((uint64_t)gene << 32) | draw;
    return finalize(key + counter * 0x9e3779b97f4a7c15ull);
}
__device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t generation, uint64_t round, uint64_t slot) {
    uint64_t key = finalize(seed + 0x632be59bd9b4e019ull);
    key = finalize(key ^ (generation * 0xd1342543de82ef95ull));
    key = finalize(key ^ (round * 0xd1342543de82ef95ull));
    return finalize(key ^ (slot * 0xd1342543de82ef95ull));
}
constexpr uint32_t kCursor = 0xffffffffu;
// Twelve 16-bit uniforms of three draws, summed as integers and centred:
// mean 0, variance 1 (+3e-5), cut at 6.
__device__ __forceinline__ float twelve_uniforms(uint64_t a, uint64_t b, uint64_t c) {
    int64_t sum = 0;
    for (const uint64_t w : {a, b, c})
        sum += (int64_t)(w & 0xffffu) + (int64_t)((w >> 16) & 0xffffu) + (int64_t)((w >> 32) & 0xffffu) +
               (int64_t)(w >> 48);
    return (float)(sum - 6 * 65535) * (1.0f / 65535.0f);
}
// Genes::gaussian: the gaussian of gene d in the sub-stream `genes`.
__device__ __forceinline__ float gene_gaussian(uint64_t genes, uint32_t d) {
    return twelve_uniforms(keyed(genes, d, 0u), keyed(genes, d, 1u), keyed(genes, d, 2u));
}

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// f32::rem_euclid(x, 1.0): the remainder of x / 1 made non-negative (it can
// round to 1.0 for a tiny negative x, as Rust's does).
__device__ __forceinline__ float rem_euclid1(float x) {
    const float r = fmodf(x, 1.0f);
    return r < 0.0f ? r + 1.0f : r;
}
// wrap_phase (src/qd.rs:2484-2486): a phase difference in [-0.5, 0.5).
__device__ __forceinline__ float wrap_phase(float delta) { return rem_euclid1(delta + 0.5f) - 0.5f; }

// The counts of a body plan, its typical bone length (Layout::of,
// src/qd.rs:2640-2651) and the coordinate maps of both modes.
struct Layout {
    unsigned nodes, bones, muscles;
    float size;
    bool exploring;
    __device__ static Layout of(const ce_genome& g, const ce_bone_gene* bones, bool exploring) {
        Layout l{g.node_count, g.bone_count, g.muscle_count, 1.0f, exploring};
        if (g.bone_count > 0u) {
            float sum = 0.0f;
            for (unsigned j = 0u; j < g.bone_count; j++) sum += bones[g.bone_start + j].rest_length;
            l.size = clampf(sum / (float)g.bone_count, 0.05f, 10.0f);
        }
        return l;
    }
    __device__ unsigned node_end() const { return nodes * 4u; }
    // Optimizer: 5 a bone, one shared period, 8 a muscle. CMA-ME: the rest
    // length of a bone, 8 a muscle.
    __device__ unsigned bone_end() const { return nodes * 4u + bones * (exploring ? 1u : 5u); }
    __device__ unsigned muscle_start() const { return bone_end() + (exploring ? 0u : 1u); }
    __device__ unsigned dims() const { return muscle_start() + muscles * 8u; }
    // Layout::scale (src/qd.rs:2658-2680), optimizers only.
    __device__ float scale(unsigned d) const {
        if (d < node_end()) return kNodeScales[d % 4u] * (d % 4u < 2u ? size : 1.0f);
        if (d < bone_end()) {
            const unsigned f = (d - node_end()) % 5u;
            return kBoneScales[f] * (f == 0u ? size : 1.0f);
        }
        if (d == bone_end()) return kPeriodScale;
        const unsigned f = (d - bone_end() - 1u) % 8u;
        return kMuscleScales[f] * (f == 2u || f == 3u ? size : 1.0f);
    }
    // The phase coordinates, which wrap: Layout::wraps (src/qd.rs:2681-2686;
    // muscle fields 4 and 7) and is_phase_dimension (src/qd.rs:2480-2482;
    // muscle field 5).
    __device__ bool wraps(unsigned d) const {
        if (d < muscle_start()) return false;
        const unsigned f = (d - muscle_start()) % 8u;
        return exploring ? f == 5u : (f == 4u || f == 7u);
    }
    // Layout::delta and moved (src/qd.rs:2687-2698).
    __device__ float delta(unsigned d, float value, float mean) const {
        return wraps(d) ? rem_euclid1(value - mean + 0.5f) - 0.5f : value - mean;
    }
    __device__ float moved(unsigned d, float mean, float step) const {
        return wraps(d) ? rem_euclid1(mean + step) : mean + step;
    }
};

// Coordinate d of write_parameters (src/qd.rs:2734-2770) for the genes of
// one body.
__device__ float opt_parameter(const Layout& l, const ce_node_gene* n, const ce_bone_gene* b,
                               const ce_muscle_gene* m, unsigned d) {
    if (d < l.node_end()) {
        const ce_node_gene& x = n[d / 4u];
        switch (d % 4u) {
            case 0u: return x.x;
            case 1u: return x.y;
            case 2u: return x.diameter;
            default: return x.friction;
        }
    }
    if (d < l.bone_end()) {
        const unsigned k = d - l.node_end();
        const ce_bone_gene& x = b[k / 5u];
        switch (k % 5u) {
            case 0u: return x.rest_length;
            case 1u: return x.min_angle;
            case 2u: return x.max_angle;
            case 3u: return x.organ_mass;
            default: return x.organ_at;
        }
    }
    if (d == l.bone_end()) return logf(fmaxf(l.muscles > 0u ? m[0].period : 1.0f, 1e-3f));
    const unsigned k = d - l.muscle_start();
    const ce_muscle_gene& x = m[k / 8u];
    switch (k % 8u) {
        case 0u: return x.anchor_a;
        case 1u: return x.anchor_b;
        case 2u: return x.short_len;
        case 3u: return x.long_len;
        case 4u: return x.phase;
        case 5u: return x.duty;
        case 6u: return logf(fmaxf(x.stiffness, 1e-3f));
        default: return x.reset;
    }
}

// Coordinate d of exploring_parameters (src/qd.rs:2504-2538).
__device__ float explore_parameter(const Layout& l, const ce_node_gene* n, const ce_bone_gene* b,
                                   const ce_muscle_gene* m, unsigned d) {
    if (d < l.node_end()) {
        const ce_node_gene& x = n[d / 4u];
        switch (d % 4u) {
            case 0u: return (x.x + 4.0f) / 8.0f;
            case 1u: return fmaxf(x.y / 4.0f, 0.0f);
            case 2u: return clampf((x.diameter - 0.01f) / 0.99f, 0.0f, 1.0f);
            default: return clampf(x.friction, 0.0f, 1.0f);
        }
    }
    if (d < l.bone_end()) return clampf((b[d - l.node_end()].rest_length - 0.03f) / (kMaxBone - 0.03f), 0.0f, 1.0f);
    const unsigned k = d - l.muscle_start();
    const ce_muscle_gene& x = m[k / 8u];
    switch (k % 8u) {
        case 0u: return clampf(x.anchor_a, 0.0f, 1.0f);
        case 1u: return clampf(x.anchor_b, 0.0f, 1.0f);
        case 2u: return fmaxf((x.short_len - 0.01f) / 0.79f, 0.0f);
        case 3u: return fmaxf((x.long_len - 0.01f) / 0.99f, 0.0f);
        case 4u: return clampf((x.period - kMinPeriod) / (10.0f - kMinPeriod), 0.0f, 1.0f);
        case 5u: return clampf(x.phase, 0.0f, 1.0f);
        case 6u: return clampf((x.duty - 0.05f) / 0.90f, 0.0f, 1.0f);
        default: return clampf((x.stiffness - 1.0f) / 119.0f, 0.0f, 1.0f);
    }
}

__device__ __forceinline__ float parameter(const Layout& l, const ce_node_gene* n, const ce_bone_gene* b,
                                           const ce_muscle_gene* m, unsigned d) {
    return l.exploring ? explore_parameter(l, n, b, m, d) : opt_parameter(l, n, b, m, d);
}

// What the kernels share: the emitters (device pointers of a ce_cma).
struct Emitters {
    ce_population t;  // the templates, genes packed from row 0
    const uint8_t* exploring;
    const uint64_t* offsets;
    float *mean, *covariance, *path_c, *path_sigma, *sigma;
    __device__ bool explores(uint64_t e) const { return exploring && exploring[e]; }
};

// CmaEmitter::optimizer and CmaEmitter::new (src/qd.rs:2130-2165): the mean
// at the template's coordinates, unit covariance, zero paths, step size 0.5
// or 0.12. One thread an emitter.
__global__ void cma_init_kernel(const Emitters em) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < em.t.count;
         e += (size_t)gridDim.x * blockDim.x) {
        const ce_genome g = em.t.genomes[e];
        const Layout l = Layout::of(g, em.t.bones, em.explores(e));
        const uint64_t off = em.offsets[e];
        for (unsigned d = 0u; d < l.dims(); d++) {
            em.mean[off + d] = parameter(l, em.t.nodes + g.node_start, em.t.bones + g.bone_start,
                                         em.t.muscles + g.muscle_start, d);
            em.covariance[off + d] = 1.0f;
            em.path_c[off + d] = 0.0f;
            em.path_sigma[off + d] = 0.0f;
        }
        em.sigma[e] = l.exploring ? 0.12f : 0.5f;
    }
}

struct AskArgs {
    ce_cma_draw draw;
    uint64_t first;
    ce_node_gene* nodes;
    ce_bone_gene* bones;
    ce_muscle_gene* muscles;
    float* strength_out;  // may be NULL
    ce_genome* genomes;
    float* values;        // may be NULL: the drawn coordinates, `stride` a sample
    size_t stride;
};

// sample_optimizing and apply_parameters (src/qd.rs:2381-2402, 2773-2811),
// sample_exploring and apply_exploring_parameters (src/qd.rs:2244-2289,
// 2579-2606), with repair's clamps of single genes (src/evolution.rs:
// 1230-1234, 1278-1330). One thread a sample.
__global__ void cma_ask_kernel(const Emitters em, const AskArgs a, size_t count) {
    const uint64_t E = em.t.count;
    const ce_cma_draw& w = a.draw;
    // The templates' rows (packed from row 0, so the last one ends them) and
    // the global row of the call's first sample, which starts its outputs.
    const ce_genome last = em.t.genomes[E - 1u], f = em.t.genomes[a.first % E];
    const uint64_t tn = last.node_start + last.node_count, tb = last.bone_start + last.bone_count,
                   tm = last.muscle_start + last.muscle_count;
    const uint64_t base_n = (a.first / E) * tn + f.node_start, base_b = (a.first / E) * tb + f.bone_start,
                   base_m = (a.first / E) * tm + f.muscle_start;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < count; c += (size_t)gridDim.x * blockDim.x) {
        const uint64_t g = a.first + c, e = g % E, k = g / E;
        const ce_genome tg = em.t.genomes[e];
        ce_genome o = tg;
        o.node_start = (uint32_t)(k * tn + tg.node_start - base_n);
        o.bone_start = (uint32_t)(k * tb + tg.bone_start - base_b);
        o.muscle_start = (uint32_t)(k * tm + tg.muscle_start - base_m);
        o.id = w.first_id + g;
        a.genomes[c] = o;
        const Layout l = Layout::of(tg, em.t.bones, em.explores(e));
        const uint64_t off = em.offsets[e];
        const float sig = em.sigma[e];
        // The child's stream; sample_into is its first use of the cursor.
        const uint64_t key = stream_key(w.seed, w.generation, w.round, g);
        uint32_t cursor = 0u;
        float path_scale = 0.0f;
        if (l.exploring) {
            // A rank-one term along the evolution path (src/qd.rs:2247-2254).
            float norm = 0.0f;
            for (unsigned d = 0u; d < l.dims(); d++) norm += em.path_c[off + d] * em.path_c[off + d];
            norm = sqrtf(norm);
            if (norm > 1e-6f) {
                const float z = twelve_uniforms(keyed(key, kCursor, 0u), keyed(key, kCursor, 1u),
                                                keyed(key, kCursor, 2u));
                path_scale = sqrtf(kPathWeight) * z / norm * sqrtf((float)l.dims());
                cursor = 3u;
            }
        }
        const uint64_t genes = keyed(key, kCursor, cursor);  // Rng::genes
        auto v = [&](unsigned d) {
            const float mean = em.mean[off + d], var = em.covariance[off + d];
            float x;
            if (!l.exploring) {
                x = mean + sig * w.strength * l.scale(d) * sqrtf(var) * gene_gaussian(genes, d);
            } else {
                const float step = sqrtf(var) * gene_gaussian(genes, d) + em.path_c[off + d] * path_scale;
                const float value = mean + sig * step * w.strength;
                const bool node = d < l.node_end();
                const unsigned f = d >= l.muscle_start() ? (d - l.muscle_start()) % 8u : 8u;
                if (l.wraps(d)) x = rem_euclid1(value);
                else if (node && d % 4u == 0u) x = value;
                else if ((node && d % 4u == 1u) || f == 2u || f == 3u) x = fmaxf(value, 0.0f);
                else x = clampf(value, 0.0f, 1.0f);
            }
            if (a.values && d < a.stride) a.values[c * a.stride + d] = x;
            return x;
        };
        const ce_muscle_gene* tm = em.t.muscles + tg.muscle_start;
        if (!l.exploring) {
            for (unsigned i = 0u; i < l.nodes; i++) {
                ce_node_gene n = em.t.nodes[tg.node_start + i];
                n.x = v(4u * i);
                n.y = fmaxf(v(4u * i + 1u), 0.0f);
                n.diameter = clampf(v(4u * i + 2u), w.min_size, w.max_size);
                n.friction = clampf(v(4u * i + 3u), w.min_friction, w.max_friction);
                a.nodes[o.node_start + i] = n;
            }
            for (unsigned j = 0u; j < l.bones; j++) {
                ce_bone_gene b = em.t.bones[tg.bone_start + j];
                const unsigned d = l.node_end() + 5u * j;
                b.rest_length = clampf(v(d), 0.03f, kMaxBone);
                // Bone::clamp_range (src/evolution.rs:114-117).
                b.min_angle = clampf(v(d + 1u), -kJointLimit, 0.0f);
                b.max_angle = clampf(v(d + 2u), 0.0f, kJointLimit);
                b.organ_mass = fmaxf(v(d + 3u), 0.0f);
                b.organ_at = clampf(v(d + 4u), 0.0f, 1.0f);
                a.bones[o.bone_start + j] = b;
            }
            // One log period scales the whole body clock.
            const float base = fmaxf(l.muscles > 0u ? tm[0].period : 1.0f, 1e-3f);
            const float pscale = clampf(expf(v(l.bone_end())), kMinPeriod, 10.0f) / base;
            for (unsigned q = 0u; q < l.muscles; q++) {
                ce_muscle_gene m = tm[q];
                const unsigned d = l.muscle_start() + 8u * q;
                m.anchor_a = clampf(v(d), 0.0f, 1.0f);
                m.anchor_b = clampf(v(d + 1u), 0.0f, 1.0f);
                m.short_len = clampf(v(d + 2u), 0.01f, 0.8f * kMaxStroke);
                m.long_len = clampf(v(d + 3u), m.short_len, kMaxStroke);
                m.period = clampf(m.period * pscale, kMinPeriod, 10.0f);
                m.phase = rem_euclid1(v(d + 4u));
                m.duty = clampf(v(d + 5u), 0.05f, 0.95f);
                m.stiffness = clampf(expf(v(d + 6u)), 1.0f, 120.0f);
                m.reset = rem_euclid1(v(d + 7u));
                a.muscles[o.muscle_start + q] = m;
            }
        } else {
            for (unsigned i = 0u; i < l.nodes; i++) {
                ce_node_gene n = em.t.nodes[tg.node_start + i];
                n.x = v(4u * i) * 8.0f - 4.0f;
                n.y = v(4u * i + 1u) * 4.0f;
                n.diameter = clampf(0.01f + v(4u * i + 2u) * 0.99f, w.min_size, w.max_size);
                n.friction = clampf(v(4u * i + 3u), w.min_friction, w.max_friction);
                a.nodes[o.node_start + i] = n;
            }
            for (unsigned j = 0u; j < l.bones; j++) {
                ce_bone_gene b = em.t.bones[tg.bone_start + j];
                b.rest_length = 0.03f + v(l.node_end() + j) * (kMaxBone - 0.03f);
                a.bones[o.bone_start + j] = b;
            }
            for (unsigned q = 0u; q < l.muscles; q++) {
                ce_muscle_gene m = tm[q];
                const unsigned d = l.muscle_start() + 8u * q;
                m.anchor_a = clampf(v(d), 0.0f, 1.0f);
                m.anchor_b = clampf(v(d + 1u), 0.0f, 1.0f);
                const float short_len = 0.01f + v(d + 2u) * 0.79f;
                const float long_len = fmaxf(0.01f + v(d + 3u) * 0.99f, short_len);
                m.short_len = clampf(short_len, 0.01f, 0.8f * kMaxStroke);
                m.long_len = clampf(long_len, m.short_len, kMaxStroke);
                m.period = clampf(kMinPeriod + v(d + 4u) * (10.0f - kMinPeriod), kMinPeriod, 10.0f);
                const float phase = v(d + 5u);
                m.phase = rem_euclid1(phase - truncf(phase));  // f32::fract
                m.duty = clampf(0.05f + v(d + 6u) * 0.90f, 0.05f, 0.95f);
                m.stiffness = clampf(1.0f + v(d + 7u) * 119.0f, 1.0f, 120.0f);
                a.muscles[o.muscle_start + q] = m;
            }
        }
        if (a.strength_out) {
            for (unsigned q = 0u; q < l.muscles; q++)
                a.strength_out[o.muscle_start + q] =
                    em.t.strength_scale ? em.t.strength_scale[tg.muscle_start + q] : 1.0f;
        }
    }
}

constexpr unsigned kTellMax = 4096u;   // samples an emitter a tell (the block's sort)
constexpr unsigned kMaxDims = 4u * CE_MAX_NODES + 5u * (CE_MAX_NODES - 1u) + 1u + 8u * CE_MAX_MUSCLES;

// The body plan check of tell's filter (src/qd.rs:2217-2228): the counts and
// the bone and muscle connections of sample `sg` are the template's. Edges
// are compared gene by gene as unordered pairs, which is the reference's
// sorted-edge comparison for samples whose genes keep the template's order
// (every ce_cma_ask sample does).
__device__ bool same_plan(const ce_population& t, const ce_genome& tg, const ce_population& s, const ce_genome& sg) {
    if (sg.node_count != tg.node_count || sg.bone_count != tg.bone_count || sg.muscle_count != tg.muscle_count)
        return false;
    for (unsigned j = 0u; j < tg.bone_count; j++) {
        const ce_bone_gene &x = t.bones[tg.bone_start + j], &y = s.bones[sg.bone_start + j];
        if (min(x.a, x.b) != min(y.a, y.b) || max(x.a, x.b) != max(y.a, y.b)) return false;
    }
    for (unsigned q = 0u; q < tg.muscle_count; q++) {
        const ce_muscle_gene &x = t.muscles[tg.muscle_start + q], &y = s.muscles[sg.muscle_start + q];
        if (min(x.bone_a, x.bone_b) != min(y.bone_a, y.bone_b) || max(x.bone_a, x.bone_b) != max(y.bone_a, y.bone_b))
            return false;
    }
    return true;
}

// CmaEmitter::tell, tell_exploring and tell_optimizing (src/qd.rs:
// 2213-2243, 2290-2376, 2405-2474), one block an emitter.
__global__ void __launch_bounds__(kTellBlock) cma_tell_kernel(const Emitters em, const ce_population s,
                                                             const float* keys, uint64_t first, size_t count) {
    __shared__ float key[kTellMax];
    __shared__ uint32_t idx[kTellMax];
    // Optimizer: the weighted step and squared steps in units of sigma.
    // CMA-ME: the mean's step in units of sigma, the squared steps and the
    // new mean.
    __shared__ float step[kMaxDims], rank_mu[kMaxDims], new_mean[kMaxDims], wts[kMaxUpdate / 2u];
    __shared__ unsigned valid;
    __shared__ float mu_eff, c_sigma_s, d_sigma_s, c_c_s, c1_s, c_mu_s, norm_s, chi_s;
    __shared__ bool hsig_s;
    const uint64_t E = em.t.count, e = blockIdx.x;
    const unsigned tid = threadIdx.x;
    const ce_genome tg = em.t.genomes[e];
    // This emitter's samples among [first, first + count): c0 + q E.
    const uint64_t c0 = (e + E - first % E) % E;
    const unsigned n = count > c0 ? (unsigned)((count - c0 + E - 1u) / E) : 0u;
    unsigned P = 1u;
    while (P < n) P <<= 1u;
    if (tid == 0u) valid = 0u;
    __syncthreads();
    for (unsigned q = tid; q < P; q += blockDim.x) {
        float f = -INFINITY;
        uint32_t c = 0xffffffffu;
        if (q < n) {
            c = (uint32_t)(c0 + (uint64_t)q * E);
            const float x = keys[c];
            if (isfinite(x) && x > kFailed && same_plan(em.t, tg, s, s.genomes[c])) {
                f = x;
                atomicAdd(&valid, 1u);
            }
        }
        key[q] = f;
        idx[q] = c;
    }
    __syncthreads();
    // Bitonic sort, best first (ties by sample index).
    for (unsigned size = 2u; size <= P; size <<= 1u) {
        for (unsigned stride = size >> 1u; stride > 0u; stride >>= 1u) {
            for (unsigned q = tid; q < P; q += blockDim.x) {
                const unsigned r = q ^ stride;
                if (r > q) {
                    const bool up = (q & size) == 0u;
                    const bool before = key[r] > key[q] || (key[r] == key[q] && idx[r] < idx[q]);
                    if (before == up) {
                        const float tk = key[q];
                        key[q] = key[r];
                        key[r] = tk;
                        const uint32_t ti = idx[q];
                        idx[q] = idx[r];
                        idx[r] = ti;
                    }
                }
            }
            __syncthreads();
        }
    }
    const unsigned len = min(valid, kMaxUpdate);
    if (len < 2u) return;
    const unsigned mu = (len + 1u) / 2u;
    const Layout l = Layout::of(tg, em.t.bones, em.explores(e));
    const unsigned D = l.dims();
    const uint64_t off = em.offsets[e];
    const float sigma = fmaxf(em.sigma[e], 1e-6f);
    if (tid == 0u) {
        float sum = 0.0f;
        for (unsigned i = 0u; i < mu; i++) {
            wts[i] = logf((float)mu + 0.5f) - logf((float)(i + 1u));
            sum += wts[i];
        }
        sum = fmaxf(sum, 1.17549435e-38f);
        float sq = 0.0f;
        for (unsigned i = 0u; i < mu; i++) {
            wts[i] /= sum;
            sq += wts[i] * wts[i];
        }
        mu_eff = 1.0f / fmaxf(sq, 1e-6f);
    }
    __syncthreads();
    // One pass over the mu best samples a coordinate, in rank order.
    for (unsigned d = tid; d < D; d += blockDim.x) {
        const float mean = em.mean[off + d];
        float st = 0.0f, rm = 0.0f;
        if (!l.exploring) {
            const float unit = sigma * l.scale(d);
            for (unsigned rank = 0u; rank < mu; rank++) {
                const ce_genome sg = s.genomes[idx[rank]];
                const float value = opt_parameter(l, s.nodes + sg.node_start, s.bones + sg.bone_start,
                                                  s.muscles + sg.muscle_start, d);
                const float y = l.delta(d, value, mean) / unit;
                st += wts[rank] * y;
                rm += wts[rank] * y * y;
            }
            step[d] = st;
        } else {
            const bool phase = l.wraps(d);
            for (unsigned rank = 0u; rank < mu; rank++) {
                const ce_genome sg = s.genomes[idx[rank]];
                const float value = explore_parameter(l, s.nodes + sg.node_start, s.bones + sg.bone_start,
                                                      s.muscles + sg.muscle_start, d);
                st += wts[rank] * (phase ? wrap_phase(value - mean) : value);
                const float delta = (phase ? wrap_phase(value - mean) : value - mean) / sigma;
                rm += wts[rank] * delta * delta;
            }
            const float nm = phase ? rem_euclid1(mean + st) : st;
            new_mean[d] = nm;
            step[d] = (phase ? wrap_phase(nm - mean) : nm - mean) / sigma;
        }
        rank_mu[d] = rm;
    }
    if (tid == 0u) {
        const float nn = (float)D;
        c_sigma_s = (mu_eff + 2.0f) / (nn + mu_eff + 5.0f);
        d_sigma_s = 1.0f + 2.0f * fmaxf(sqrtf(fmaxf(mu_eff - 1.0f, 0.0f) / (nn + 1.0f)) - 1.0f, 0.0f) + c_sigma_s;
        c_c_s = (4.0f + mu_eff / nn) / (nn + 4.0f + 2.0f * mu_eff / nn);
        if (!l.exploring) {
            // A diagonal covariance learns (n + 2) / 3 times faster than a full one.
            const float separable = (nn + 2.0f) / 3.0f;
            c1_s = fminf(2.0f / ((nn + 1.3f) * (nn + 1.3f) + mu_eff) * separable, 0.5f);
            c_mu_s = fminf(2.0f * fmaxf(mu_eff - 2.0f + 1.0f / mu_eff, 0.0f) / ((nn + 2.0f) * (nn + 2.0f) + mu_eff) *
                               separable,
                           1.0f - c1_s);
        } else {
            c1_s = 2.0f / ((nn + 1.3f) * (nn + 1.3f) + mu_eff);
            c_mu_s = fminf(2.0f * fmaxf(mu_eff - 2.0f + 1.0f / mu_eff, 0.0f) / ((nn + 2.0f) * (nn + 2.0f) + mu_eff),
                           1.0f - c1_s);
        }
        chi_s = sqrtf(nn) * (1.0f - 1.0f / (4.0f * nn) + 1.0f / (21.0f * nn * nn));
    }
    __syncthreads();
    // The step-size path (its norm: one thread, in coordinate order).
    for (unsigned d = tid; d < D; d += blockDim.x) {
        const float k = sqrtf(c_sigma_s * (2.0f - c_sigma_s) * mu_eff);
        const float sd = fmaxf(sqrtf(em.covariance[off + d]), 1e-6f);
        float p = em.path_sigma[off + d];
        p = l.exploring ? (1.0f - c_sigma_s) * p + k * (step[d] / sd) : (1.0f - c_sigma_s) * p + k * step[d] / sd;
        em.path_sigma[off + d] = p;
    }
    __syncthreads();
    if (tid == 0u) {
        float norm = 0.0f;
        for (unsigned d = 0u; d < D; d++) {
            const float p = em.path_sigma[off + d];
            norm += p * p;
        }
        norm_s = sqrtf(norm);
        hsig_s = norm_s / fmaxf(chi_s, 1e-6f) < 1.4f + 2.0f / ((float)D + 1.0f);
    }
    __syncthreads();
    const float correction = hsig_s ? 0.0f : c_c_s * (2.0f - c_c_s);
    const float lo = l.exploring ? 0.0025f : 1e-4f, hi = l.exploring ? 4.0f : 1e4f;
    for (unsigned d = tid; d < D; d += blockDim.x) {
        const float pc = (1.0f - c_c_s) * em.path_c[off + d] +
                         (hsig_s ? sqrtf(c_c_s * (2.0f - c_c_s) * mu_eff) * step[d] : 0.0f);
        em.path_c[off + d] = pc;
        em.covariance[off + d] = clampf((1.0f - c1_s - c_mu_s + c1_s * correction) * em.covariance[off + d] +
                                            c1_s * pc * pc + c_mu_s * rank_mu[d],
                                        lo, hi);
        em.mean[off + d] = l.exploring ? new_mean[d] : l.moved(d, em.mean[off + d], sigma * l.scale(d) * step[d]);
    }
    if (tid == 0u) {
        const float grow = expf((c_sigma_s / d_sigma_s) * (norm_s / fmaxf(chi_s, 1e-6f) - 1.0f));
        if (l.exploring) {
            em.sigma[e] = clampf(em.sigma[e] * grow, 0.005f, 0.35f);
        } else {
            float sg = clampf(em.sigma[e] * grow, 0.01f, 30.0f);
            // Fast gaits are fragile: when most samples fail outright, shrink
            // the steps instead of letting step-length control grow them.
            if (key[len / 2u] < 0.25f * key[0]) sg = fmaxf(sg * 0.6f, 0.01f);
            em.sigma[e] = sg;
        }
    }
}

// CmaEmitter::recentered (src/qd.rs:2166-2177), one thread a pair:
// emitter which[i] restarts from body i of `b`. Counts that differ from the
// template's leave the emitter as it was (rejected[i] = 1). Otherwise the
// plan test runs on the old template, the body's genes replace the
// template's, the mean moves to the body's coordinates and the covariance,
// paths and step size stay when the plan is the template's, else restart as
// the mode's constructor sets them.
__global__ void cma_recenter_kernel(const Emitters em, const ce_population b, const uint32_t* which, size_t n,
                                    uint32_t* rejected) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t e = which[i];
        if (e >= em.t.count) {  // no such emitter
            if (rejected) rejected[i] = 1u;
            continue;
        }
        const ce_genome tg = em.t.genomes[e], bg = b.genomes[i];
        const bool fits = bg.node_count == tg.node_count && bg.bone_count == tg.bone_count &&
                          bg.muscle_count == tg.muscle_count;
        if (rejected) rejected[i] = fits ? 0u : 1u;
        if (!fits) continue;
        const bool keep = same_plan(em.t, tg, b, bg);
        ce_node_gene* tn = const_cast<ce_node_gene*>(em.t.nodes) + tg.node_start;
        ce_bone_gene* tb = const_cast<ce_bone_gene*>(em.t.bones) + tg.bone_start;
        ce_muscle_gene* tm = const_cast<ce_muscle_gene*>(em.t.muscles) + tg.muscle_start;
        for (unsigned k = 0u; k < tg.node_count; k++) tn[k] = b.nodes[bg.node_start + k];
        for (unsigned k = 0u; k < tg.bone_count; k++) tb[k] = b.bones[bg.bone_start + k];
        for (unsigned k = 0u; k < tg.muscle_count; k++) tm[k] = b.muscles[bg.muscle_start + k];
        if (em.t.strength_scale && b.strength_scale) {
            float* ts = const_cast<float*>(em.t.strength_scale) + tg.muscle_start;
            for (unsigned k = 0u; k < tg.muscle_count; k++) ts[k] = b.strength_scale[bg.muscle_start + k];
        }
        const Layout l = Layout::of(tg, em.t.bones, em.explores(e));
        const uint64_t off = em.offsets[e];
        for (unsigned d = 0u; d < l.dims(); d++) {
            em.mean[off + d] = parameter(l, tn, tb, tm, d);
            if (!keep) {
                em.covariance[off + d] = 1.0f;
                em.path_c[off + d] = 0.0f;
                em.path_sigma[off + d] = 0.0f;
            }
        }
        if (!keep) em.sigma[e] = l.exploring ? 0.12f : 0.5f;
    }
}

}  // namespace

namespace {

unsigned grid_for(size_t n) {
    const size_t b = (n + 255u) / 256u;
    return (unsigned)(b < 148u * 16u ? (b > 0 ? b : 1) : 148u * 16u);
}

ce_status launched(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ce::set_error(std::string(what) + ": launch: " + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    return CE_OK;
}

bool usable(const ce_cma* c) {
    return c && c->templates.count && c->templates.genomes && c->templates.nodes && c->templates.bones &&
           c->templates.muscles && c->offsets && c->mean && c->covariance && c->path_c && c->path_sigma &&
           c->sigma;
}

Emitters emitters_of(const ce_cma* c) {
    return Emitters{c->templates, c->exploring, c->offsets, c->mean, c->covariance, c->path_c, c->path_sigma,
                    c->sigma};
}

uint64_t dims_of(const ce_genome& g, bool exploring) {
    return exploring ? 4ull * g.node_count + g.bone_count + 8ull * g.muscle_count
                     : 4ull * g.node_count + 5ull * g.bone_count + 1ull + 8ull * g.muscle_count;
}

}  // namespace

extern "C" ce_status ce_cma_offsets(const ce_genome* templates, const uint8_t* exploring, size_t emitters,
                                    uint64_t* offsets) {
    if (!templates || !offsets) {
        ce::set_error("ce_cma_offsets: null argument");
        return CE_ERR_INVALID;
    }
    uint64_t at = 0;
    for (size_t e = 0; e < emitters; e++) {
        const ce_genome& g = templates[e];
        if (g.node_count < 2 || g.node_count > CE_MAX_NODES || g.bone_count + 1 != g.node_count ||
            g.muscle_count > CE_MAX_MUSCLES) {
            ce::set_error("ce_cma_offsets: template " + std::to_string(e) + " is not a body the engine runs");
            return CE_ERR_INVALID;
        }
        offsets[e] = at;
        at += dims_of(g, exploring && exploring[e]);
    }
    offsets[emitters] = at;
    return CE_OK;
}

extern "C" ce_status ce_cma_init(const ce_cma* cma, void* stream) {
    if (!usable(cma)) {
        ce::set_error("ce_cma_init: null argument or no emitters");
        return CE_ERR_INVALID;
    }
    // The templates' genes must be packed in order from row 0: ask derives
    // every sample's rows from that (checked here, once).
    const size_t E = cma->templates.count;
    std::vector<ce_genome> hg(E);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(hg.data(), cma->templates.genomes, E * sizeof(ce_genome), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ce::set_error(std::string("ce_cma_init: reading the templates: ") + cudaGetErrorString(e));
        return CE_ERR_DEVICE;
    }
    uint64_t at[3] = {0, 0, 0};
    for (size_t q = 0; q < E; q++) {
        const ce_genome& g = hg[q];
        if (g.node_start != at[0] || g.bone_start != at[1] || g.muscle_start != at[2]) {
            ce::set_error("ce_cma_init: the templates' genes must be packed in order from row 0");
            return CE_ERR_INVALID;
        }
        at[0] += g.node_count;
        at[1] += g.bone_count;
        at[2] += g.muscle_count;
    }
    cma_init_kernel<<<grid_for(E), 256, 0, st>>>(emitters_of(cma));
    return launched("ce_cma_init");
}

extern "C" ce_status ce_cma_ask(const ce_cma* cma, const ce_cma_draw* draw, uint64_t first, size_t count,
                                ce_node_gene* nodes, ce_bone_gene* bones, ce_muscle_gene* muscles,
                                float* strength_out, ce_genome* genomes, float* values, size_t stride,
                                void* stream) {
    if (!usable(cma) || !draw || !genomes || (count && (!nodes || !bones || !muscles)) || (values && stride == 0)) {
        ce::set_error("ce_cma_ask: null argument or no emitters");
        return CE_ERR_INVALID;
    }
    if (!(draw->min_size <= draw->max_size) || !(draw->min_friction <= draw->max_friction)) {
        ce::set_error("ce_cma_ask: an empty diameter or friction range");
        return CE_ERR_INVALID;
    }
    if (count == 0) return CE_OK;
    AskArgs a;
    a.draw = *draw;
    a.first = first;
    a.nodes = nodes;
    a.bones = bones;
    a.muscles = muscles;
    a.strength_out = strength_out;
    a.genomes = genomes;
    a.values = values;
    a.stride = stride;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cma_ask_kernel<<<grid_for(count), 256, 0, st>>>(emitters_of(cma), a, count);
    return launched("ce_cma_ask");
}

extern "C" ce_status ce_cma_tell(const ce_cma* cma, const ce_population* samples, const float* keys,
                                 uint64_t first, size_t count, void* stream) {
    if (!usable(cma) || !samples || !samples->genomes || !samples->nodes || !samples->bones || !samples->muscles ||
        !keys) {
        ce::set_error("ce_cma_tell: null argument or no emitters");
        return CE_ERR_INVALID;
    }
    const size_t E = cma->templates.count;
    if ((count + E - 1) / E > kTellMax) {
        ce::set_error("ce_cma_tell: at most " + std::to_string(kTellMax) + " samples an emitter in one tell");
        return CE_ERR_INVALID;
    }
    if (count > 0xffffffffull) {
        ce::set_error("ce_cma_tell: too many samples");
        return CE_ERR_INVALID;
    }
    if (count == 0) return CE_OK;
    cma_tell_kernel<<<(unsigned)E, kTellBlock, 0, static_cast<cudaStream_t>(stream)>>>(emitters_of(cma), *samples,
                                                                                         keys, first, count);
    return launched("ce_cma_tell");
}

extern "C" ce_status ce_cma_recenter(const ce_cma* cma, const ce_population* bodies, const uint32_t* which, size_t n,
                                     uint32_t* rejected, void* stream) {
    if (!usable(cma) || !bodies || (n && (!which || !bodies->genomes || !bodies->nodes || !bodies->bones ||
                                          !bodies->muscles))) {
        ce::set_error("ce_cma_recenter: null argument or no emitters");
        return CE_ERR_INVALID;
    }
    if (n == 0) return CE_OK;
    cma_recenter_kernel<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(emitters_of(cma), *bodies, which,
                                                                                     n, rejected);
    return launched("ce_cma_recenter");
}
