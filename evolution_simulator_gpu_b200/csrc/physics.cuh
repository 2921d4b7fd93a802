// Device physics of one creature: the substep passes and the ground, written
// for one creature per GPU lane.
//
// The arithmetic of every pass follows the reference kernel operation for
// operation (shaders/creature.cu:130-742), because scoring must agree with
// the reference bit for bit: the same products, sums and their order give the
// same rounding and the same fused multiply-adds under nvcc's
// -fmad=true -prec-div=false -prec-sqrt=false. The data layout is this
// engine's own:
//   * node state sits in shared-memory tables, one column per lane and
//     8 bytes an entry: positions, velocities, and the force / previous
//     position pair, so every access of a warp to one table is free of bank
//     conflicts;
//   * a creature's constants sit in 16-byte "lines" of a per-lane slot in
//     global memory, laid out lane-major (line L of lane l at
//     slot + (L * 32 + l) * 16), so the 32 lanes of a warp read a line as one
//     512-byte coalesced request; `Lines` hides where a line lives.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/creature_engine.h"

namespace cek {

// ------------------------------------------------------------- constants
// The reference's #define block (src/kernel.rs:268-317) with the same float
// values.
constexpr float kMuscleRecovery = 0.5f;
constexpr float kInvJointDamping = 10.0f;
constexpr float kJointBreak = 0.5f;
constexpr float kMudNormal = 2.0f;
constexpr float kMudGrip = 2.0f;
constexpr float kMudDrag = 2.0f;
constexpr float kMudFullDepth = 0.1f;
constexpr float kBrambleReach = 0.01f;
constexpr float kAirDrag = 0.6f;
constexpr float kWaterDrag = 100.0f;
constexpr float kWaterAlong = 0.25f;
constexpr float kWaterBuoyancy = 0.7f;
constexpr float kIceInv = 0.16666667f;
constexpr float kHeadShakeLimit = 78.4f;
constexpr float kHeadShakeWindow = 0.1f;
constexpr float kContactSlack = 0.002f;
constexpr float kLiftClearance = 0.01f;
constexpr float kGapDepth = 2.0f;
constexpr float kGapRun = 0.15f;
constexpr float kHurdleSpacing = 3.0f;
constexpr float kHurdleTop = 1.2f;
constexpr float kHurdleRun = 0.2f;
constexpr float kPiF = 3.14159265359f;
constexpr float kTauF = 6.28318530718f;
constexpr uint32_t kNone = 0xffffffffu;

// Step clock of a fidelity: RATE steps per second, 16 substeps per step.
template <int RATE>
struct Clock {
    static constexpr float rate = (float)RATE;
    static constexpr float dt = 1.0f / rate;
    static constexpr float h = 1.0f / (rate * 16u);
    static constexpr float inv_h = rate * 16u;
    static constexpr uint32_t settle = (200u * RATE + 119u) / 120u;
    static constexpr uint32_t sample = RATE / 30 > 1 ? RATE / 30 : 1;
    static constexpr uint32_t head_sample = (uint32_t)(rate / 60.0f + 0.5f);
};

// The world's effect switches, fixed at compile time (F) or read at run
// time (RuntimeWorld). `has` of a compile-time world folds to a constant.
template <uint32_t F>
struct StaticWorld {
    __device__ __forceinline__ static constexpr bool has(uint32_t bit) { return (F & bit) != 0u; }
};
struct RuntimeWorld {
    uint32_t f;
    __device__ __forceinline__ bool has(uint32_t bit) const { return (f & bit) != 0u; }
};

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float wrapf(float a) { return a - kTauF * floorf((a + kPiF) * (1.0f / kTauF)); }
__device__ __forceinline__ float fracf(float x) { return x - floorf(x); }
__device__ __forceinline__ unsigned f2h(float v) { return (unsigned)__half_as_ushort(__float2half_rn(v)); }
__device__ __forceinline__ float h2f(unsigned h) { return __half2float(__ushort_as_half((unsigned short)h)); }

// Half-cosine rhythm (shaders/creature.cu:153-159).
__device__ __forceinline__ float rhythm(float t, float inv_period, float phase, float offset, float duty,
                                        float inv_duty, float inv_complement) {
    const float ph = fracf(t * inv_period + phase + offset);
    if (ph < duty) {
        return 0.5f - 0.5f * __cosf(kPiF * ph * inv_duty);
    }
    return 0.5f + 0.5f * __cosf(kPiF * (ph - duty) * inv_complement);
}

// Ground height and slope under x (shaders/creature.cu:166-226).
template <class W>
__device__ __forceinline__ float2 ground(const W& w, float x, float amp, float qphase, const ce_params& p) {
    float height = 0.0f, slope = 0.0f;
    if (w.has(CE_FLAG_TERRAIN)) {
        const float t0 = x * (1.0f / 1.1f) + qphase;
        const float u0 = fracf(t0);
        const float w0 = u0 * (1.0f - u0);
        const float t1 = x * (1.0f / 0.43f) + 0.3f + qphase;
        const float u1 = fracf(t1);
        const float w1 = u1 * (1.0f - u1);
        height = amp * (0.65f * 16.0f * w0 * w0 + 0.35f * 16.0f * w1 * w1);
        slope = amp * (0.65f * 32.0f * w0 * (1.0f - 2.0f * u0) * (1.0f / 1.1f) +
                       0.35f * 32.0f * w1 * (1.0f - 2.0f * u1) * (1.0f / 0.43f));
    }
    if (w.has(CE_FLAG_SLOPE)) {
        height += p.slope * x;
        slope += p.slope;
    }
    if (w.has(CE_FLAG_GAPS)) {
        const float spacing = 2.0f + 4.0f * p.gaps;
        const float center = spacing * 0.5f;
        const float r = x - floorf(x / spacing) * spacing;
        const float distance = fabsf(r - center);
        const float half_w = 0.5f * p.gaps;
        const float run = fmaxf(fminf(kGapRun, half_w), 1e-6f);
        float factor = clampf((half_w - distance) / run, 0.0f, 1.0f);
        if (distance <= half_w - run) {
            factor = 1.0f;
        } else if (distance >= half_w) {
            factor = 0.0f;
        }
        height -= kGapDepth * factor;
        if (distance > half_w - run && distance < half_w) {
            slope -= kGapDepth * ((r < center ? 1.0f : -1.0f) / run);
        }
    }
    if (w.has(CE_FLAG_HURDLES)) {
        const float spacing = kHurdleSpacing;
        const float center = spacing * 0.5f;
        const float r = x - floorf(x / spacing) * spacing;
        const float distance = fabsf(r - center);
        const float half_w = 0.5f * kHurdleTop;
        const float run = kHurdleRun;
        float factor = clampf((half_w + run - distance) / run, 0.0f, 1.0f);
        if (distance <= half_w) {
            factor = 1.0f;
        } else if (distance >= half_w + run) {
            factor = 0.0f;
        }
        height += p.hurdles * factor;
        if (distance > half_w && distance < half_w + run) {
            slope += p.hurdles * ((r < center ? 1.0f : -1.0f) / run);
        }
    }
    return make_float2(height, slope);
}


// The ground and floor height of the step's contact tallies with every
// rounding pinned (fused multiply-adds where the reference kernel's compiled
// tallies fuse them, measured on the GPU), so no other code change can move
// the contact tests at their edges.
template <class W>
__device__ __forceinline__ float2 ground_tally(const W& w, float x, float amp, float qphase, const ce_params& p) {
    float height = 0.0f, slope = 0.0f;
    if (w.has(CE_FLAG_TERRAIN)) {
        const float t0 = __fmaf_rn(x, (1.0f / 1.1f), qphase);
        const float u0 = __fsub_rn(t0, floorf(t0));
        const float w0 = __fmul_rn(u0, __fsub_rn(1.0f, u0));
        const float t1 = __fadd_rn(__fmaf_rn(x, (1.0f / 0.43f), 0.3f), qphase);
        const float u1 = __fsub_rn(t1, floorf(t1));
        const float w1 = __fmul_rn(u1, __fsub_rn(1.0f, u1));
        height = __fmul_rn(amp, __fmaf_rn(__fmul_rn(0.65f * 16.0f, w0), w0, __fmul_rn(__fmul_rn(0.35f * 16.0f, w1), w1)));
        const float a2 = __fmul_rn(__fmul_rn(0.65f * 32.0f, w0), __fsub_rn(1.0f, __fmul_rn(2.0f, u0)));
        const float b2 = __fmul_rn(__fmul_rn(0.35f * 32.0f, w1), __fsub_rn(1.0f, __fmul_rn(2.0f, u1)));
        slope = __fmaf_rn(a2, (1.0f / 1.1f), __fmul_rn(b2, (1.0f / 0.43f)));
        if (w.has(CE_FLAG_SLOPE)) {
            height = __fmaf_rn(p.slope, x, height);
            slope = __fmaf_rn(amp, slope, p.slope);
        } else {
            slope = __fmul_rn(amp, slope);
        }
    } else if (w.has(CE_FLAG_SLOPE)) {
        height = __fmul_rn(p.slope, x);
        slope = p.slope;
    }
    if (w.has(CE_FLAG_GAPS)) {
        const float spacing = __fmaf_rn(4.0f, p.gaps, 2.0f);
        const float center = __fmul_rn(spacing, 0.5f);
        const float r = __fmaf_rn(-floorf(x / spacing), spacing, x);
        const float distance = fabsf(__fsub_rn(r, center));
        const float half_w = __fmul_rn(0.5f, p.gaps);
        const float run = fmaxf(fminf(kGapRun, half_w), 1e-6f);
        float factor = clampf(__fsub_rn(half_w, distance) / run, 0.0f, 1.0f);
        if (distance <= __fsub_rn(half_w, run)) {
            factor = 1.0f;
        } else if (distance >= half_w) {
            factor = 0.0f;
        }
        height = __fmaf_rn(-kGapDepth, factor, height);
        if (distance > __fsub_rn(half_w, run) && distance < half_w) {
            slope = __fmaf_rn(-kGapDepth, (r < center ? 1.0f : -1.0f) / run, slope);
        }
    }
    if (w.has(CE_FLAG_HURDLES)) {
        const float spacing = kHurdleSpacing;
        const float center = spacing * 0.5f;
        const float r = __fmaf_rn(-floorf(x / spacing), spacing, x);
        const float distance = fabsf(__fsub_rn(r, center));
        const float half_w = 0.5f * kHurdleTop;
        const float run = kHurdleRun;
        float factor = clampf((half_w + run - distance) / run, 0.0f, 1.0f);
        if (distance <= half_w) {
            factor = 1.0f;
        } else if (distance >= half_w + run) {
            factor = 0.0f;
        }
        height = __fmaf_rn(p.hurdles, factor, height);
        if (distance > half_w && distance < half_w + run) {
            slope = __fmaf_rn(p.hurdles, (r < center ? 1.0f : -1.0f) / run, slope);
        }
    }
    return make_float2(height, slope);
}

// Ice at x (shaders/creature.cu:230-235).
__device__ __forceinline__ float ice_at(float x) {
    const float w = fracf(x * kIceInv);
    const float t = fabsf(w - 0.5f) * 2.0f;
    const float s = clampf((0.7f - t) * 2.5f, 0.0f, 1.0f);
    return s * s * (3.0f - 2.0f * s);
}

// ------------------------------------------------------------ the tables
// Node state of the lanes of a block in shared memory. Row i of a table
// holds node i of every lane, so a warp reads a row without bank conflicts
// whatever node each lane asks for.
// Position and velocity have tables of their own: a lane's 8-byte entries
// then lie 8 bytes apart across the lanes, so a warp reading positions only
// (or velocities only) meets no bank twice.
struct NodeTables {
    float2* p;   // (x, y)
    float2* v;   // (vx, vy)
    float2* fp;  // muscle force, then the position at the start of the substep
    float2* ms;  // per muscle: (energy store, demand of the step)
    // Entries between rows: the threads of a block (kBlock), a constant so
    // that a row's address is one shift and add.
    static constexpr unsigned stride = 128u;
    __device__ __forceinline__ float4 at(unsigned i) const {
        const float2 q = p[i * stride], u = v[i * stride];
        return make_float4(q.x, q.y, u.x, u.y);
    }
    __device__ __forceinline__ void set_at(unsigned i, const float4& s) const {
        p[i * stride] = make_float2(s.x, s.y);
        v[i * stride] = make_float2(s.z, s.w);
    }
    __device__ __forceinline__ float2& f(unsigned i) const { return fp[i * stride]; }
    __device__ __forceinline__ float2& pos(unsigned i) const { return p[i * stride]; }
    __device__ __forceinline__ float2& vel(unsigned i) const { return v[i * stride]; }
    __device__ __forceinline__ float2& muscle(unsigned k) const { return ms[k * stride]; }
};

// The constant lines of a lane's creature: 16-byte lines, and regions of
// 8-byte half lines and of single words (entry k of a half-line region that
// starts at line R is float2 R * 64 + k * 32 + lane of the warp's slot, of a
// word region float R * 128 + k * 32 + lane), so that a warp reads a half
// line as one 256-byte request and a word as one 128-byte request when a
// pass needs only part of an item.
struct Lines {
    float4* base;  // line 0 of this lane
    float2* half;  // float2 0 of the warp's slot, plus this lane
    float* words;  // float 0 of the warp's slot, plus this lane
    __device__ __forceinline__ static Lines make(float4* warp_slot, unsigned lane) {
        return Lines{warp_slot + lane, reinterpret_cast<float2*>(warp_slot) + lane,
                     reinterpret_cast<float*>(warp_slot) + lane};
    }
    __device__ __forceinline__ float4 get(unsigned L) const { return base[L * 32u]; }
    __device__ __forceinline__ float2 get2(unsigned R, unsigned k) const { return half[R * 64u + k * 32u]; }
    __device__ __forceinline__ void put2(unsigned R, unsigned k, float2 v) const { half[R * 64u + k * 32u] = v; }
    __device__ __forceinline__ float get1(unsigned R, unsigned k) const { return words[R * 128u + k * 32u]; }
    __device__ __forceinline__ void put1(unsigned R, unsigned k, float v) const { words[R * 128u + k * 32u] = v; }
    __device__ __forceinline__ void put(unsigned L, float4 v) const { base[L * 32u] = v; }
    __device__ __forceinline__ float& word(unsigned L, unsigned k) const {
        return reinterpret_cast<float*>(&base[L * 32u])[k];
    }
    // Lines touched once a step (muscle rhythm and state, the lane lines) go
    // through the evict-first cache operator (ld/st.global.cs), so the lines
    // that every substep reads keep their place in L2: the slots of all
    // resident lanes together are about as large as L2.
    __device__ __forceinline__ float4 get_cold(unsigned L) const { return __ldcs(&base[L * 32u]); }
    __device__ __forceinline__ void put_cold(unsigned L, float4 v) const { __stcs(&base[L * 32u], v); }
    __device__ __forceinline__ float word_cold(unsigned L, unsigned k) const {
        return __ldcs(reinterpret_cast<const float*>(&base[L * 32u]) + k);
    }
    __device__ __forceinline__ void set_cold(unsigned L, unsigned k, float v) const {
        __stcs(reinterpret_cast<float*>(&base[L * 32u]) + k, v);
    }
};

// Where each kind of line starts in a slot of a class with NS node rows and
// MM muscles at most. A recording slot also has a line per node for its
// contact forces (`rec_force`), the kept result (`rec_kept`, 5 lines) and
// the muscles' pulls, four to a line (`rec_pull`).
//
// The half-line and word regions repeat words of the lines for the passes
// that need only some of them, so those passes move fewer bytes from L2: a
// node's (mass, 1/mass) for the force pass (`mass`) and (radius, friction)
// for the ground pass (`ground`), a muscle's (force cap, 1/capacity)
// (`cap`) and (tendon stiffness, slack length) (`tendon`, read only for a
// creature with a tendon), a bone's pivot node for the air drag (`pivot`)
// and a joint's topology word for the damping (`topo`).
//
// The node, bone and joint passes load the line of the next item while they
// work on the current one, so each loads one item past its last. The
// regions follow each other (nodes, bones, joints, muscles, then the nine
// lane lines), so that extra load always lands inside the lane's own slot;
// a layout that ends with one of those regions needs padding after it, and
// each half-line region holds one entry more than it has items.
struct SlotLayout {
    unsigned node, bone, joint, muscle, lane, rec_force, rec_kept, rec_pull, mass, ground, cap, tendon, pivot, topo,
        lines;
    __host__ __device__ static SlotLayout make(unsigned ns, unsigned mm, bool record) {
        SlotLayout s;
        s.node = 0;
        s.bone = ns;
        s.joint = s.bone + 2u * (ns - 1u);
        s.muscle = s.joint + 2u * (ns - 1u);
        s.lane = s.muscle + 5u * mm;
        s.rec_force = s.lane + 9u;
        s.rec_kept = s.rec_force + ns;
        s.rec_pull = s.rec_kept + 5u;
        s.mass = record ? s.rec_pull + (mm + 3u) / 4u : s.rec_force;
        s.ground = s.mass + (ns + 2u) / 2u;
        s.cap = s.ground + (ns + 2u) / 2u;
        s.tendon = s.cap + (mm + 2u) / 2u;
        s.pivot = s.tendon + (mm + 2u) / 2u;
        s.topo = s.pivot + (ns + 3u) / 4u;
        s.lines = s.topo + (ns + 3u) / 4u;
        return s;
    }
};
// Words of the lane lines: the result (0-18), then the tallies.
constexpr unsigned kWContact = 19, kWLift = 20, kWGround = 21, kWHeadShake = 22, kWHeadAt = 23,
                   kWHeadVel = 25, kWRungX = 27, kWRungSpeed = 28, kWRungEarly = 29, kWRungLate = 30,
                   kWRungBits = 31;
// Lines of muscle k: pull 0 and 1, rhythm 0 and 1, and its state line
// (unused, unused, touchdown offset, sensor); the energy store and the
// step's demand live in shared memory (NodeTables::muscle).
constexpr unsigned kPull0 = 0, kPull1 = 1, kRhythm0 = 2, kRhythm1 = 3, kMState = 4;

}  // namespace cek
