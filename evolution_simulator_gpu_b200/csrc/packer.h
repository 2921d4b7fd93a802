// The packer's arithmetic, shared by the host (host_model.cpp, built by the
// C++ compiler without contraction) and the device (pack.cu, built with IEEE
// division and square root and no contraction): a body's model, start pose
// and kernel records, restating the reference's host model so that a body
// packs into the same words the reference would upload:
//   physics::node_mass / body / add_muscle_masses  src/physics.rs:182-296
//   physics2::Model::new / start / kinematics      src/physics2.rs:186-428
//   kernel::fill_creature / pack_reusing           src/kernel.rs:336-593
//   physics ground, quake hash                     src/physics.rs:523-714
//   f32 -> f16                                      src/creature_kernel.rs:242-274
// The reference host is Rust, whose f32 arithmetic is IEEE single with no
// contraction of multiply-adds; both builds of this file round as it does.
// The one thing the two sides cannot share is the C library's
// single-precision arctangent, sine and cosine (what Rust's f32 methods call
// on Linux), which are not correctly rounded and so have no device
// equivalent: the model takes them through two policies, `Angle` (a bone's
// gene-pose direction, atan2) and `Trig` (the sine and cosine of a bone's
// start-pose angle). The host computes them; the device reads the host's
// values (ce_pack_plan), once per body, since they depend only on the
// node positions of the genes.
#pragma once
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "../../include/creature_engine.h"

#if defined(__CUDACC__)
#define CE_HD __host__ __device__ inline
#else
#define CE_HD inline
#endif

namespace ce {

namespace lim {  // physics::Limits::DEFAULT, src/physics.rs:142-153
constexpr float muscle_speed = 24.0f;
constexpr float muscle_force = 200.0f;
constexpr float muscle_energy = 120.0f;
constexpr float max_bone = 2.0f;
constexpr float bone_density = 4.0f;
}  // namespace lim
constexpr float kPi = 3.14159265358979323846f;   // std::f32::consts::PI
constexpr float kTau = 6.28318530717958647692f;  // std::f32::consts::TAU
constexpr float kDrivenAcceleration = 200.0f;   // src/physics2.rs:34
constexpr float kHillSpeed = 8.0f;              // src/physics2.rs:24-26
constexpr float kTendonStretch = 0.25f;         // src/evolution.rs:245
constexpr float kMuscleMassBase = 0.05f;        // src/physics.rs:244
constexpr float kMuscleMassPerM = 1.0f;         // src/physics.rs:246
// (a function, so device code reads no host array)
CE_HD float terrain_level(uint32_t i) {
    return i == 0u ? 0.0f : i == 1u ? 0.03f : i == 2u ? 0.08f : i == 3u ? 0.15f : 0.25f;
}
constexpr float kGapDepth = 2.0f, kGapRun = 0.15f;
constexpr float kHurdleSpacing = 3.0f, kHurdleTop = 1.2f, kHurdleRun = 0.2f;

CE_HD float terrain_amplitude(uint32_t level) { return terrain_level(level < 4u ? level : 4u); }

CE_HD uint32_t quake_hash(uint64_t id) {
    uint32_t x = (uint32_t)id;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
CE_HD float quake_phase(uint32_t h) { return (float)(h & 0xffffu) * (1.0f / 65536.0f); }
CE_HD float quake_scale(uint32_t h) { return 0.6f + (float)((h >> 16) & 0xffffu) * (0.8f / 65536.0f); }


CE_HD uint16_t f32_to_f16(float v) {
    uint32_t bits;
    memcpy(&bits, &v, 4);
    const uint16_t sign = (uint16_t)((bits >> 16) & 0x8000u);
    const int32_t exponent = (int32_t)((bits >> 23) & 0xffu);
    const uint32_t mantissa = bits & 0x7fffffu;
    if (exponent == 0xff) return (uint16_t)(sign | 0x7c00u | (mantissa != 0 ? 0x200u : 0u));
    const int32_t e = exponent - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return sign;
        const uint32_t m = mantissa | 0x800000u;
        const uint32_t shift = (uint32_t)(14 - e);
        const uint32_t half = 1u << (shift - 1);
        const uint32_t rest = m & ((1u << shift) - 1u);
        uint32_t out = m >> shift;
        if (rest > half || (rest == half && (out & 1u))) out += 1;
        return (uint16_t)(sign | out);
    }
    const uint32_t rest = mantissa & 0x1fffu;
    uint32_t out = ((uint32_t)e << 10) | (mantissa >> 13);
    if (rest > 0x1000u || (rest == 0x1000u && (out & 1u))) out += 1;
    return (uint16_t)(sign | out);
}


CE_HD uint32_t fbits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
CE_HD float ubits(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
// Rust's f32::min / f32::max / clamp for numbers that are not NaN.
CE_HD float fmin_(float a, float b) { return fminf(a, b); }
CE_HD float fmax_(float a, float b) { return fmaxf(a, b); }
CE_HD float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }


// ------------------------------------------------------------------ ground
// physics::terrain_phase, gaps, hurdles and ground (src/physics.rs:541-683).
CE_HD void terrain_phase(float x, float amp, float phase, float& h, float& s) {
    const float waves[2][3] = {{1.1f, 0.65f, 0.0f}, {0.43f, 0.35f, 0.3f}};
    float height = 0.0f, slope = 0.0f;
    for (int k = 0; k < 2; k++) {
        const float* w = waves[k];
        const float t = x / w[0] + w[2] + phase;
        const float u = t - floorf(t);
        const float q = u * (1.0f - u);
        height += w[1] * 16.0f * q * q;
        slope += w[1] * 32.0f * q * (1.0f - 2.0f * u) / w[0];
    }
    h = amp * height;
    s = amp * slope;
}
CE_HD void gaps(float x, float width, float& h, float& s) {
    h = 0.0f;
    s = 0.0f;
    if (width <= 0.0f) return;
    const float spacing = 2.0f + 4.0f * width;
    const float r = x - floorf(x / spacing) * spacing;
    const float center = 0.5f * spacing;
    const float distance = fabsf(r - center);
    const float half = 0.5f * width;
    const float run = fmin_(kGapRun, half);
    float factor, fs;
    if (distance >= half) factor = 0.0f;
    else if (distance <= half - run) factor = 1.0f;
    else factor = (half - distance) / run;
    if (distance > half - run && distance < half) fs = r < center ? 1.0f / run : -1.0f / run;
    else fs = 0.0f;
    h = -kGapDepth * factor;
    s = -kGapDepth * fs;
}
CE_HD void hurdles(float x, float height, float& h, float& s) {
    h = 0.0f;
    s = 0.0f;
    if (height <= 0.0f) return;
    const float spacing = kHurdleSpacing;
    const float r = x - floorf(x / spacing) * spacing;
    const float center = 0.5f * spacing;
    const float distance = fabsf(r - center);
    const float half = 0.5f * kHurdleTop;
    const float run = kHurdleRun;
    float factor, fs;
    if (distance <= half) factor = 1.0f;
    else if (distance >= half + run) factor = 0.0f;
    else factor = (half + run - distance) / run;
    if (distance > half && distance < half + run) fs = r < center ? 1.0f / run : -1.0f / run;
    else fs = 0.0f;
    h = height * factor;
    s = height * fs;
}
CE_HD void ground(float x, float amplitude, float tilt, float width, float hurdle, float phase, float& h,
            float& s) {
    float bh, bs;
    terrain_phase(x, amplitude, phase, bh, bs);
    float height = bh + tilt * x, slope = bs + tilt;
    float ph, ps;
    gaps(x, width, ph, ps);
    height += ph;
    slope += ps;
    float hh, hs;
    hurdles(x, hurdle, hh, hs);
    h = height + hh;
    s = slope + hs;
}


// A vector of at most N elements stored inline: the packer's per-creature
// model holds a few dozen small arrays, and heap allocations for them cost
// more than the arithmetic. The interface is the part of std::vector used.
template <class T, size_t N>
struct Inline {
    T v[N];
    size_t n = 0;
    CE_HD Inline() {}
    CE_HD explicit Inline(size_t k, const T& x = T()) { assign(k, x); }
    CE_HD void assign(size_t k, const T& x) {
        n = k;
        for (size_t i = 0; i < k; i++) v[i] = x;
    }
    CE_HD void resize(size_t k) {
        for (size_t i = n; i < k; i++) v[i] = T();
        n = k;
    }
    CE_HD void reserve(size_t) {}
    CE_HD void push_back(const T& x) { v[n++] = x; }
    CE_HD size_t size() const { return n; }
    CE_HD T& operator[](size_t i) { return v[i]; }
    CE_HD const T& operator[](size_t i) const { return v[i]; }
    CE_HD T* data() { return v; }
    CE_HD const T* data() const { return v; }
};
constexpr size_t kNodesMax = CE_MAX_NODES, kBonesMax = CE_MAX_NODES - 1, kMusclesMax = CE_MAX_MUSCLES;

struct PNode {  // physics::Node, the fields the model reads
    float px, py, radius, friction, mass;
};

CE_HD float node_mass(float diameter) {
    const float q = diameter / 0.08f;
    return clampf(0.1f * (q * q), 0.02f, 10.0f);
}

CE_HD float muscle_span(const ce_bone_gene* bones, size_t nb, const PNode* nodes, size_t nn,
                         const ce_muscle_gene& m) {
    auto point = [&](uint32_t bone, float t, float out[2]) -> bool {
        if (bone >= nb) return false;
        const ce_bone_gene& b = bones[bone];
        if (b.a >= nn || b.b >= nn) return false;
        const PNode& a = nodes[b.a];
        const PNode& c = nodes[b.b];
        out[0] = a.px + (c.px - a.px) * t;
        out[1] = a.py + (c.py - a.py) * t;
        return true;
    };
    float p[2], q[2];
    if (!point(m.bone_a, m.anchor_a, p) || !point(m.bone_b, m.anchor_b, q)) return 0.0f;
    const float dx = p[0] - q[0], dy = p[1] - q[1];
    return sqrtf(dx * dx + dy * dy);
}
CE_HD float slack_length(const ce_bone_gene* bones, size_t nb, const PNode* nodes, size_t nn,
                          const ce_muscle_gene& m) {
    return fmax_(m.long_len, muscle_span(bones, nb, nodes, nn, m));
}

// physics::nodes: node masses with bones, organs and muscles.
CE_HD Inline<PNode, kNodesMax> body_nodes(const ce_node_gene* g, size_t n, const ce_bone_gene* bones,
                                           size_t nb, const ce_muscle_gene* muscles, size_t nm) {
    Inline<PNode, kNodesMax> nodes(n);
    for (size_t i = 0; i < n; i++) {
        nodes[i] = PNode{g[i].x, g[i].y, g[i].diameter * 0.5f, g[i].friction, node_mass(g[i].diameter)};
    }
    for (size_t j = 0; j < nb; j++) {
        const ce_bone_gene& b = bones[j];
        if (b.a >= n || b.b >= n) continue;
        const float half = 0.5f * lim::bone_density * b.rest_length * b.rest_length;
        nodes[b.a].mass += half;
        nodes[b.b].mass += half;
        if (b.organ_mass > 0.0f) {
            nodes[b.a].mass += b.organ_mass * (1.0f - b.organ_at);
            nodes[b.b].mass += b.organ_mass * b.organ_at;
        }
    }
    for (size_t k = 0; k < nm; k++) {
        const ce_muscle_gene& m = muscles[k];
        const float half =
            0.5f * (kMuscleMassBase + kMuscleMassPerM * slack_length(bones, nb, nodes.data(), n, m));
        const uint32_t bb[2] = {m.bone_a, m.bone_b};
        const float tt[2] = {m.anchor_a, m.anchor_b};
        for (int s = 0; s < 2; s++) {
            if (bb[s] >= nb) continue;
            const ce_bone_gene& b = bones[bb[s]];
            if (b.a >= n || b.b >= n) continue;
            const float t = clampf(tt[s], 0.0f, 1.0f);
            nodes[b.a].mass += half * (1.0f - t);
            nodes[b.b].mass += half * t;
        }
    }
    return nodes;
}

CE_HD float wrap(float a) { return a - kTau * floorf((a + kPi) / kTau); }

struct MuscleModel {
    uint32_t bone_a, bone_b;
    float anchor_a, anchor_b, hill, long_, tendon_k, amplitude, inv_period, phase, duty, inv_duty,
        inv_complement, stiffness, strength, reset;
    uint32_t sensor;  // CE_NONE when absent
};

struct Model {
    Inline<float, kNodesMax> mass, radius, friction;
    float total_mass = 0, inv_mass = 0;
    Inline<uint32_t, kBonesMax> pivot;
    Inline<int32_t, kBonesMax> parent;  // -1 = none
    Inline<float, kBonesMax> length, lo, hi, rest;
    Inline<MuscleModel, kMusclesMax> muscles;
    float quake_phase_ = 0, amplitude = 0;
    Inline<float, kNodesMax> sx, sy;  // gene positions in model order
};

// physics2::Model::new (src/physics2.rs:190-350). `angle_of(j, dy, dx)` gives
// bone j's direction in the gene pose, atan2(dy, dx).
template <class Angle>
CE_HD Model make_model(const ce_node_gene* g, size_t n, const ce_bone_gene* bones, size_t nb,
                       const ce_muscle_gene* mg, size_t nm, uint64_t id, const ce_world& w, Angle angle_of) {
    const Inline<PNode, kNodesMax> nodes = body_nodes(g, n, bones, nb, mg, nm);
    Inline<uint32_t, kNodesMax> order(n);
    order[0] = 0;
    for (size_t j = 0; j < nb; j++) order[j + 1] = bones[j].b;
    Inline<uint32_t, kNodesMax> record(n, 0);
    for (size_t r = 0; r < n; r++) record[order[r]] = (uint32_t)r;
    Inline<int32_t, kNodesMax> parent_of_node(n, -1);
    for (size_t j = 0; j < nb; j++) parent_of_node[bones[j].b] = (int32_t)j;
    // Each bone's direction in the gene pose, once a bone.
    Inline<float, kBonesMax> angles(nb);
    for (size_t j = 0; j < nb; j++) {
        const ce_node_gene& p = g[bones[j].a];
        const ce_node_gene& q = g[bones[j].b];
        angles[j] = angle_of(j, q.y - p.y, q.x - p.x);
    }
    auto angle = [&](size_t j) { return angles[j]; };
    Model M;
    M.rest.reserve(nb);
    for (size_t j = 0; j < nb; j++) {
        int32_t up = parent_of_node[bones[j].a];
        if (up < 0 && j > 0) up = 0;
        M.parent.push_back(up);
        const float relative = up >= 0 ? wrap(angle(j) - angle((size_t)up)) : angle(j);
        M.rest.push_back(relative);
        M.lo.push_back(relative + bones[j].min_angle);
        M.hi.push_back(relative + bones[j].max_angle);
    }
    M.muscles.resize(nm);
    for (size_t k = 0; k < nm; k++) {
        const ce_muscle_gene& m = mg[k];
        const ce_bone_gene& ba = bones[m.bone_a];
        const ce_bone_gene& bb = bones[m.bone_b];
        const uint32_t ends[4] = {ba.a, ba.b, bb.a, bb.b};
        MuscleModel& u = M.muscles[k];
        u.bone_a = m.bone_a;
        u.bone_b = m.bone_b;
        u.anchor_a = m.anchor_a;
        u.anchor_b = m.anchor_b;
        u.hill = 1.0f / (kHillSpeed * fmax_(m.long_len, 0.05f));
        u.long_ = slack_length(bones, nb, nodes.data(), n, m);
        u.tendon_k = 0.0f;
        u.amplitude = fmin_(m.long_len - m.short_len,
                            2.0f * lim::muscle_speed * m.period * fmin_(m.duty, 1.0f - m.duty) / kPi);
        u.inv_period = 1.0f / m.period;
        u.phase = m.phase;
        u.duty = m.duty;
        u.inv_duty = 1.0f / m.duty;
        u.inv_complement = 1.0f / (1.0f - m.duty);
        u.stiffness = m.stiffness;
        u.strength = 1.0f;
        u.sensor = m.sensor != CE_NO_SENSOR ? record[ends[m.sensor]] : CE_NONE;
        u.reset = m.reset;
    }
    // Strength from the lighter driven subtree, shared by same-side copies.
    Inline<float, kBonesMax> subtree(nb);
    for (size_t j = 0; j < nb; j++) {
        subtree[j] = nodes[order[j + 1]].mass + (j == 0 ? nodes[order[0]].mass : 0.0f);
    }
    for (size_t j = nb; j-- > 1;) {
        if (M.parent[j] >= 0) subtree[(size_t)M.parent[j]] += subtree[j];
    }
    struct Key {
        uint32_t lo, hi;
        bool side;
        CE_HD bool operator==(const Key& o) const { return lo == o.lo && hi == o.hi && side == o.side; }
    };
    auto bone_point = [&](const ce_bone_gene& b, float t, float out[2]) {
        const ce_node_gene& a = g[b.a];
        const ce_node_gene& c = g[b.b];
        out[0] = a.x + (c.x - a.x) * t;
        out[1] = a.y + (c.y - a.y) * t;
    };
    auto group = [&](const ce_muscle_gene& m) {
        const ce_bone_gene& ba = bones[m.bone_a];
        const ce_bone_gene& bb = bones[m.bone_b];
        float pa[2], pb[2], j[2];
        bone_point(ba, m.anchor_a, pa);
        bone_point(bb, m.anchor_b, pb);
        int64_t shared = -1;
        for (uint32_t nd : {ba.a, ba.b}) {
            if (nd == bb.a || nd == bb.b) {
                shared = nd;
                break;
            }
        }
        if (shared >= 0) {
            j[0] = g[shared].x;
            j[1] = g[shared].y;
        } else {
            j[0] = 0.5f * (pa[0] + pb[0]);
            j[1] = 0.5f * (pa[1] + pb[1]) - 1.0f;
        }
        const float cross = (pa[0] - j[0]) * (pb[1] - j[1]) - (pa[1] - j[1]) * (pb[0] - j[0]);
        return Key{m.bone_a < m.bone_b ? m.bone_a : m.bone_b, m.bone_a < m.bone_b ? m.bone_b : m.bone_a, cross >= 0.0f};
    };
    Inline<Key, kMusclesMax> groups(nm);
    for (size_t k = 0; k < nm; k++) groups[k] = group(mg[k]);
    for (size_t k = 0; k < nm; k++) {
        MuscleModel& u = M.muscles[k];
        const float driven = fmin_(subtree[u.bone_a], subtree[u.bone_b]);
        size_t sharing = 0;
        for (size_t q = 0; q < nm; q++) sharing += groups[q] == groups[k] ? 1 : 0;
        const float share = (float)(sharing > 1 ? sharing : 1);
        u.strength = fmin_(kDrivenAcceleration * driven / lim::muscle_force, 1.0f) / share;
        u.tendon_k = mg[k].tendon * lim::muscle_force * u.strength / (kTendonStretch * fmax_(u.long_, 0.05f));
    }
    const uint32_t qh = quake_hash(id);
    const bool still = w.quake <= 0.0f || !w.ground;
    M.mass.resize(n);
    M.radius.resize(n);
    M.friction.resize(n);
    M.sx.resize(n);
    M.sy.resize(n);
    float total = 0.0f;
    for (size_t r = 0; r < n; r++) {
        M.mass[r] = nodes[order[r]].mass;
        M.radius[r] = nodes[order[r]].radius;
        M.friction[r] = nodes[order[r]].friction;
        M.sx[r] = g[order[r]].x;
        M.sy[r] = g[order[r]].y;
        total += nodes[order[r]].mass;
    }
    M.total_mass = total;
    M.inv_mass = 1.0f / total;
    M.pivot.resize(nb);
    M.length.resize(nb);
    for (size_t j = 0; j < nb; j++) {
        M.pivot[j] = record[bones[j].a];
        M.length[j] = bones[j].rest_length;
    }
    M.quake_phase_ = still ? 0.0f : quake_phase(qh);
    M.amplitude = terrain_amplitude(w.terrain) + (still ? 0.0f : w.quake * quake_scale(qh));
    return M;
}

struct State {
    float x0[2], v0[2], th0, w0;
    Inline<float, kBonesMax> q, qd, th, om;
    Inline<float, kNodesMax> px, py, vx, vy;
};

// physics2::Model::kinematics (src/physics2.rs:402-418). `trig(j, th, sn, cs)`
// gives the sine and cosine of bone j's world angle th.
template <class Trig>
CE_HD void kinematics(const Model& M, State& s, Trig trig) {
    s.px[0] = s.x0[0];
    s.py[0] = s.x0[1];
    s.vx[0] = s.v0[0];
    s.vy[0] = s.v0[1];
    for (size_t j = 0; j < M.pivot.size(); j++) {
        float th, om;
        if (M.parent[j] >= 0) {
            const size_t p = (size_t)M.parent[j];
            th = s.th[p] + s.q[j];
            om = s.om[p] + s.qd[j];
        } else {
            th = s.th0;
            om = s.w0;
        }
        s.th[j] = th;
        s.om[j] = om;
        float sn, cs;
        trig(j, th, sn, cs);
        const size_t p = M.pivot[j], c = j + 1;
        const float l = M.length[j];
        s.px[c] = s.px[p] + l * cs;
        s.py[c] = s.py[p] + l * sn;
        s.vx[c] = s.vx[p] - l * om * sn;
        s.vy[c] = s.vy[p] + l * om * cs;
    }
}

// physics2::Model::start (src/physics2.rs:371-399).
template <class Trig>
CE_HD State start_state(const Model& M, const ce_world& w, Trig trig) {
    const size_t b = M.pivot.size(), n = M.mass.size();
    State s;
    s.x0[0] = M.sx[0];
    s.x0[1] = M.sy[0];
    s.v0[0] = s.v0[1] = 0.0f;
    s.th0 = b > 0 ? M.rest[0] : 0.0f;
    s.w0 = 0.0f;
    s.q = M.rest;
    s.qd.assign(b, 0.0f);
    s.th.assign(b, 0.0f);
    s.om.assign(b, 0.0f);
    s.px.assign(n, 0.0f);
    s.py.assign(n, 0.0f);
    s.vx.assign(n, 0.0f);
    s.vy.assign(n, 0.0f);
    kinematics(M, s, trig);
    float cx = 0.0f, cy = 0.0f;
    for (size_t i = 0; i < n; i++) {
        cx += s.px[i] * M.mass[i];
        cy += s.py[i] * M.mass[i];
    }
    cx = cx * M.inv_mass;
    cy = cy * M.inv_mass;
    (void)cy;
    float low = INFINITY;
    for (size_t i = 0; i < n; i++) {
        float h, sl;
        if (w.ground) {
            ground(s.px[i] - cx, M.amplitude, w.slope, w.gaps, w.hurdles, M.quake_phase_, h, sl);
        } else {
            h = -INFINITY;
        }
        low = fmin_(low, s.py[i] - M.radius[i] - fmax_(h, -1e6f));
    }
    if (!w.ground) low = 0.0f;
    s.x0[0] -= cx;
    s.x0[1] -= low;
    kinematics(M, s, trig);
    return s;
}


// kernel::fill_creature (src/kernel.rs:336-411) plus the head words of
// kernel::pack_reusing (src/kernel.rs:554-565).
// `angle_of` and `trig` as for make_model and kinematics.
template <class Angle, class Trig>
CE_HD void fill_creature(const ce_population& pop, size_t i, const ce_world& w, uint32_t* record, float* muscles,
                         uint32_t* head, uint32_t record_at, uint32_t muscle_at, Angle angle_of, Trig trig) {
    const ce_genome& gm = pop.genomes[i];
    const size_t n = gm.node_count, nb = gm.bone_count, nm = gm.muscle_count;
    const ce_node_gene* g = pop.nodes + gm.node_start;
    const ce_bone_gene* bones = pop.bones + gm.bone_start;
    const ce_muscle_gene* mg = pop.muscles + gm.muscle_start;
    const Model M = make_model(g, n, bones, nb, mg, nm, gm.id, w, angle_of);
    const State s = start_state(M, w, trig);
    uint32_t children[CE_MAX_NODES] = {0};
    for (size_t j = 1; j < nb; j++) {
        if (M.parent[j] >= 0) children[M.parent[j]] += 1;
    }
    for (size_t r = 0; r <= nb; r++) {
        bool foot = false;
        if (r > 0) {
            const size_t j = r - 1;
            const int32_t p = M.parent[j];
            foot = children[j] == 0 && p >= 0 && j > 0 && p > 0 && children[p] == 1;
        }
        uint32_t* rr = record + r * CE_NODE_WORDS;
        rr[0] = fbits(M.mass[r]);
        rr[1] = fbits(M.radius[r]);
        rr[2] = fbits(M.friction[r]);
        rr[3] = fbits(s.px[r]);
        rr[4] = fbits(s.py[r]);
        rr[5] = foot ? 1u : 0u;
    }
    const size_t bone_at = (nb + 1) * CE_NODE_WORDS;
    for (size_t j = 0; j < nb; j++) {
        uint32_t* rr = record + bone_at + j * CE_BONE_WORDS;
        rr[0] = M.pivot[j];
        rr[1] = fbits(M.length[j]);
        rr[2] = (j > 0 && M.parent[j] >= 0) ? (uint32_t)M.parent[j] : CE_NONE;
        rr[3] = fbits(M.lo[j]);
        rr[4] = fbits(M.hi[j]);
        rr[5] = 0;
    }
    const float* scale = pop.strength_scale ? pop.strength_scale + gm.muscle_start : nullptr;
    for (size_t k = 0; k < nm; k++) {
        const MuscleModel& u = M.muscles[k];
        const float strength = u.strength * (scale ? scale[k] : 1.0f);
        const uint32_t a0 = M.pivot[u.bone_a], b0 = M.pivot[u.bone_b];
        const uint32_t nodes = a0 | (u.bone_a + 1) << 8 | b0 << 16 | (u.bone_b + 1) << 24;
        float* v = muscles + k * CE_MUSCLE_FIELDS;
        v[0] = ubits(nodes);
        v[1] = u.anchor_a;
        v[2] = u.anchor_b;
        v[3] = u.hill;
        v[4] = lim::muscle_force * strength;
        v[5] = 1.0f / (lim::muscle_energy * strength);
        v[6] = u.tendon_k;
        v[7] = u.long_;
        v[8] = u.amplitude;
        v[9] = u.inv_period;
        v[10] = u.phase;
        v[11] = u.duty;
        v[12] = u.inv_duty;
        v[13] = u.inv_complement;
        v[14] = u.stiffness;
        v[15] = u.reset;
        v[16] = ubits(u.sensor);
        v[17] = v[18] = v[19] = 0.0f;
    }
    const float period = nm > 0 ? mg[0].period : 0.0f;
    head[0] = (uint32_t)n;
    head[1] = (uint32_t)nm;
    head[2] = quake_hash(gm.id);
    head[3] = record_at;
    head[4] = muscle_at;
    head[5] = fbits(M.total_mass);
    head[6] = fbits(M.inv_mass);
    head[7] = (uint32_t)f32_to_f16(period) | (gm.flags << 16);
}


// Gene gradients of one creature from its record-field gradient `rec`
// (ce_backward's row of `rows` node rows and `mm` muscle slots), by the
// chain rule through the packing arithmetic of make_model and
// fill_creature: per muscle d/d(short, long, strength scale, on time, off
// time) into muscle_grads (5 a muscle gene, at its muscle_start), per node
// d/d friction into node_grads (at its node_start). `angle_of` and `trig`
// as for make_model and kinematics.
template <class Angle, class Trig>
CE_HD void gene_gradients_one(const ce_population& pop, uint32_t i, const ce_world& world, const float* rec,
                              uint32_t rows, uint32_t mm, double* muscle_grads, double* node_grads, Angle angle_of,
                              Trig trig) {
    const ce_genome& gm = pop.genomes[i];
    const ce_node_gene* ng = pop.nodes + gm.node_start;
    const ce_bone_gene* bg = pop.bones + gm.bone_start;
    const ce_muscle_gene* mg = pop.muscles + gm.muscle_start;
    const Model M = make_model(ng, gm.node_count, bg, gm.bone_count, mg, gm.muscle_count, gm.id, world, angle_of);
    const size_t n = gm.node_count, nb = gm.bone_count, nm = gm.muscle_count;
    // d J / d (gene node mass): the kernel's rows, then the strengths.
    const Inline<PNode, kNodesMax> body = body_nodes(ng, n, bg, nb, mg, nm);
    uint32_t row_of[CE_MAX_NODES] = {0};
    row_of[0] = 0;
    for (size_t j = 0; j < nb; j++) row_of[bg[j].b] = (uint32_t)(j + 1);
    double dmass[CE_MAX_NODES] = {0.0};
    for (size_t node = 0; node < n; node++) dmass[node] = rec[9 * mm + rows + row_of[node]];
    // The start pose is moved by minus the centre of mass's x
    // (start_state), so a mass moves every start x by -x_start / total;
    // on uneven ground it is also lowered onto the ground under its
    // lowest node, whose height moves with the shift by the ground's
    // slope there.
    {
        const State st = start_state(M, world, trig);
        double shift = 0.0, lift = 0.0;
        for (size_t r = 0; r < n; r++) {
            shift += rec[9 * mm + 2 * rows + 2 * r];
            lift += rec[9 * mm + 2 * rows + 2 * r + 1];
        }
        if (world.ground) {
            float lowest = INFINITY, slope = 0.0f;
            for (size_t r = 0; r < n; r++) {
                float h, sl;
                ground(st.px[r], M.amplitude, world.slope, world.gaps, world.hurdles, M.quake_phase_, h, sl);
                const float low = st.py[r] - M.radius[r] - fmax_(h, -1e6f);
                if (low < lowest) {
                    lowest = low;
                    slope = sl;
                }
            }
            shift += lift * (double)slope;
        }
        for (size_t node = 0; node < n; node++) {
            dmass[node] -= shift * (double)st.px[row_of[node]] * (double)M.inv_mass;
        }
    }
    double subtree[CE_MAX_NODES] = {0.0};
    for (size_t j = 0; j < nb; j++) subtree[j] = body[bg[j].b].mass + (j == 0 ? body[0].mass : 0.0f);
    for (size_t j = nb; j-- > 1;) {
        if (M.parent[j] >= 0) subtree[(size_t)M.parent[j]] += subtree[j];
    }
    auto within = [&](size_t bone, size_t top) {  // bone in the subtree of bone `top`
        for (int64_t at = (int64_t)bone; at >= 0; at = M.parent[(size_t)at]) {
            if ((size_t)at == top) return true;
            if (at == 0) break;
        }
        return false;
    };
    for (size_t q = 0; q < nm; q++) {
        const double sa = subtree[mg[q].bone_a], sb = subtree[mg[q].bone_b];
        const double driven = sb < sa ? sb : sa;
        const size_t top = subtree[mg[q].bone_a] <= subtree[mg[q].bone_b] ? mg[q].bone_a : mg[q].bone_b;
        if (!(kDrivenAcceleration * driven / lim::muscle_force < 1.0) || driven <= 0.0) continue;
        const double strength = M.muscles[q].strength;
        const double scale = pop.strength_scale ? pop.strength_scale[gm.muscle_start + q] : 1.0;
        const double d_strength = (double)rec[9 * q + 2] * lim::muscle_force * scale -
                                  (double)rec[9 * q + 3] / (lim::muscle_energy * strength * strength * scale);
        const double per_mass = d_strength * strength / driven;
        if (top == 0) dmass[0] += per_mass;
        for (size_t i = 0; i < nb; i++) {
            if (within(i, top)) dmass[bg[i].b] += per_mass;
        }
    }
    for (size_t k = 0; k < gm.muscle_count; k++) {
        const ce_muscle_gene& m = mg[k];
        const double g_amp = rec[9 * k + 0], g_hill = rec[9 * k + 1], g_cap = rec[9 * k + 2];
        const double g_icap = rec[9 * k + 3], g_phase = rec[9 * k + 4], g_duty = rec[9 * k + 5];
        const double g_iduty = rec[9 * k + 6], g_icomp = rec[9 * k + 7];
        const float stroke = 2.0f * lim::muscle_speed * m.period * fmin_(m.duty, 1.0f - m.duty) / kPi;
        const bool by_lengths = (m.long_len - m.short_len) <= stroke;
        const double T = m.period, duty = m.duty;
        double d_duty = g_duty - g_iduty / (duty * duty) + g_icomp / ((1.0 - duty) * (1.0 - duty));
        if (!by_lengths) {
            d_duty += g_amp * 2.0 * lim::muscle_speed * T / kPi * (m.duty < 1.0f - m.duty ? 1.0 : -1.0);
        }
        const bool free_duty = m.duty > 0.05f && m.duty < 0.95f;
        const double strength = M.muscles[k].strength;
        const double scale = pop.strength_scale ? pop.strength_scale[gm.muscle_start + k] : 1.0;
        double* out = muscle_grads + 5 * (gm.muscle_start + k);
        out[0] = by_lengths ? -g_amp : 0.0;
        out[1] = (by_lengths ? g_amp : 0.0) +
                 (m.long_len > 0.05f ? -g_hill / (kHillSpeed * (double)m.long_len * m.long_len) : 0.0);
        if (m.long_len >= muscle_span(bg, nb, body.data(), n, m)) {
            const uint32_t bb[2] = {m.bone_a, m.bone_b};
            const float tt[2] = {m.anchor_a, m.anchor_b};
            for (int side = 0; side < 2; side++) {
                if (bb[side] >= nb || bg[bb[side]].a >= n || bg[bb[side]].b >= n) continue;
                const double t = clampf(tt[side], 0.0f, 1.0f);
                out[1] += 0.5 * kMuscleMassPerM * ((1.0 - t) * dmass[bg[bb[side]].a] + t * dmass[bg[bb[side]].b]);
            }
        }
        out[2] = g_cap * lim::muscle_force * strength -
                 g_icap / (lim::muscle_energy * strength * scale * scale);
        out[3] = -g_phase / T - (free_duty ? d_duty / T : 0.0);
        out[4] = free_duty ? d_duty / T : 0.0;
    }
    for (size_t r = 0; r < gm.node_count; r++) {
        const size_t gene_node = r == 0 ? 0 : bg[r - 1].b;
        node_grads[gm.node_start + gene_node] = rec[9 * mm + r];
    }
}

}  // namespace ce
