// The creature kernel: whole trials, one creature per lane, in a persistent
// launch.
//
// Work: the launch runs `count` creatures, creature i being `order[i]` of the
// packed batch (or base + i without an order list). Warps claim runs of
// creatures from a counter and free lanes take the next creature of the run
// after every step, so a lane whose creature fell early is refilled at once.
// Creatures of one launch share a size class: NS node rows per lane in the
// shared-memory tables and at most MM muscles in a lane's slot (the host
// splits a batch by node count, and the batch is sorted by muscle count, so
// the lanes of a warp hold bodies of about the same size).
//
// Per creature the kernel does what the reference's advance does
// (shaders/creature.cu:845-1248): begin (start pose, derived constants), then
// per step the muscle demands, 16 substeps and the step's tallies (centre of
// mass, contacts, touchdowns, head shake, broken joints, fall, gait turns,
// rungs, screen, end), storing the 76-byte result when the trial ends.
#pragma once
#include "kernels.h"
#include "physics.cuh"

namespace cek {

constexpr uint32_t kChunk = 32;

// Per-lane values kept in registers across a step.
struct LaneRegs {
    uint32_t nodes, muscles, feet, cidx, step, flags, rec_slot;
    float amp, qphase, inv_mass, period_f;
    bool limp, scoring;
    bool tendon;  // a muscle of the creature has a tendon
};

// The arithmetic of each item of a pass sits in its own function (the
// *_item functions), which the pass loops call.
template <class W, int RATE, bool RECORD>
struct Creature {
    using C = Clock<RATE>;
    const W& w;
    const ce_params& p;
    const NodeTables& t;
    const Lines& L;
    const SlotLayout& S;
    LaneRegs& r;

    // Joint j from its two lines (shaders/creature.cu:322-356).
    struct Joint {
        unsigned tip, far, hub;
        float2 g_tip, g_far, g_hub;
        float angle, lo, hi, w_tip, w_far, w_hub;
    };
    __device__ __forceinline__ Joint joint(unsigned j, const float4& ra, const float4& rb,
                                           bool with_angle) const {
        Joint k;
        const unsigned topo = __float_as_uint(ra.x);
        k.tip = j + 1u;
        k.hub = topo & 31u;
        const unsigned parent_tip = (topo >> 5u) & 31u, parent_pivot = (topo >> 10u) & 31u;
        k.far = (topo >> 15u) & 31u;
        const bool at_head = ((topo >> 20u) & 1u) != 0u;
        k.lo = ra.y;
        k.hi = ra.z;
        k.w_tip = rb.x;
        k.w_far = rb.y;
        k.w_hub = rb.z;
        const float2 pt = t.pos(parent_tip), pp = t.pos(parent_pivot);
        const float2 ct = t.pos(k.tip), ch = t.pos(k.hub);
        const float2 u = make_float2(pt.x - pp.x, pt.y - pp.y);
        const float2 v = make_float2(ct.x - ch.x, ct.y - ch.y);
        const float uu = fmaxf(u.x * u.x + u.y * u.y, 1e-12f), vv = fmaxf(v.x * v.x + v.y * v.y, 1e-12f);
        k.angle = 0.0f;
        if (with_angle) {
            const float turn = atan2f(u.x * v.y - u.y * v.x, u.x * v.x + u.y * v.y);
            const float mid = ra.w;
            k.angle = mid + wrapf(turn - mid);
        }
        k.g_tip = make_float2(-v.y / vv, v.x / vv);
        const float2 g_u = make_float2(-u.y / uu, u.x / uu);
        k.g_far = at_head ? make_float2(-g_u.x, -g_u.y) : g_u;
        k.g_hub = make_float2(-(k.g_tip.x + k.g_far.x), -(k.g_tip.y + k.g_far.y));
        return k;
    }
    __device__ __forceinline__ static float joint_weight(const Joint& k) {
        return k.w_tip * (k.g_tip.x * k.g_tip.x + k.g_tip.y * k.g_tip.y) +
               k.w_far * (k.g_far.x * k.g_far.x + k.g_far.y * k.g_far.y) +
               k.w_hub * (k.g_hub.x * k.g_hub.x + k.g_hub.y * k.g_hub.y);
    }
    // Each node as one 8-byte load and store: tip, far, then hub.
    template <bool VEL>
    __device__ __forceinline__ void joint_push(const Joint& k, float lambda) const {
        float2& tip = VEL ? t.vel(k.tip) : t.pos(k.tip);
        float2 e = tip;
        e.x += k.w_tip * lambda * k.g_tip.x;
        e.y += k.w_tip * lambda * k.g_tip.y;
        tip = e;
        float2& far = VEL ? t.vel(k.far) : t.pos(k.far);
        e = far;
        e.x += k.w_far * lambda * k.g_far.x;
        e.y += k.w_far * lambda * k.g_far.y;
        far = e;
        float2& hub = VEL ? t.vel(k.hub) : t.pos(k.hub);
        e = hub;
        e.x += k.w_hub * lambda * k.g_hub.x;
        e.y += k.w_hub * lambda * k.g_hub.y;
        hub = e;
    }

    // Each muscle's demand for the step that starts at t_now
    // (shaders/creature.cu:442-451).
    __device__ __forceinline__ void muscle_demands(float t_now) const {
        for (unsigned k = 0u; k < r.muscles; k++) {
            const unsigned m0 = S.muscle + 5u * k;
            const float4 r0 = L.get_cold(m0 + kRhythm0), r1 = L.get_cold(m0 + kRhythm1);
            float& demand = t.muscle(k).y;
            const float offset = L.word_cold(m0 + kMState, 2);
            const float before = rhythm(t_now, r0.y, r0.z, offset, r0.w, r1.x, r1.y);
            const float after = rhythm(t_now + C::dt, r0.y, r0.z, offset, r0.w, r1.x, r1.y);
            const float shortening = r0.x * (after - before) * C::rate;
            demand = r.limp ? 0.0f : fmaxf(shortening * r1.z * 0.25f, 0.0f);
        }
    }

    // Muscle pulls into the force table and the energy stores
    // (shaders/creature.cu:455-508).
    __device__ __forceinline__ void muscle_forces() const {
        for (unsigned i = 0u; i < r.nodes; i++) {
            t.f(i) = make_float2(0.0f, 0.0f);
        }
        // The next muscle's lines load while the current one is worked on
        // (3.5% faster on the game workload than leaving the overlap to an
        // unrolled loop); the load one past the last stays inside the slot:
        // the lane lines follow the muscle lines and each half-line region
        // holds an entry more than it has items.
        float4 n0 = L.get(S.muscle + kPull0);
        float2 nc = L.get2(S.cap, 0u);
        float2 nt = r.tendon ? L.get2(S.tendon, 0u) : make_float2(0.0f, 0.0f);
#pragma unroll 1
        for (unsigned k = 0u; k < r.muscles; k++) {
            // The pull lines: (nodes, anchors, hill), then the force cap and
            // 1/capacity, and the tendon's stiffness and slack only for a
            // creature that has a tendon (0 and 0 otherwise, which give the
            // same zero tendon force).
            const float4 q0 = n0;
            const float2 qc = nc;
            const float2 qt = nt;
            n0 = L.get(S.muscle + 5u * (k + 1u) + kPull0);
            nc = L.get2(S.cap, k + 1u);
            if (r.tendon) {
                nt = L.get2(S.tendon, k + 1u);
            }
            const float4 q1 = make_float4(qc.x, qc.y, qt.x, qt.y);
            const float2 ms = t.muscle(k);
            const unsigned nodes = __float_as_uint(q0.x);
            const unsigned a0 = nodes & 255u, a1 = (nodes >> 8u) & 255u, b0 = (nodes >> 16u) & 255u,
                           b1 = nodes >> 24u;
            const float anchor_a = q0.y, anchor_b = q0.z, hill = q0.w;
            const float cap = q1.x, inv_capacity = q1.y, tendon_k = q1.z, slack = q1.w;
            const float4 A0 = t.at(a0), A1 = t.at(a1), B0 = t.at(b0), B1 = t.at(b1);
            const float ax = A0.x + (A1.x - A0.x) * anchor_a;
            const float ay = A0.y + (A1.y - A0.y) * anchor_a;
            const float avx = A0.z + (A1.z - A0.z) * anchor_a;
            const float avy = A0.w + (A1.w - A0.w) * anchor_a;
            const float bx = B0.x + (B1.x - B0.x) * anchor_b;
            const float by = B0.y + (B1.y - B0.y) * anchor_b;
            const float bvx = B0.z + (B1.z - B0.z) * anchor_b;
            const float bvy = B0.w + (B1.w - B0.w) * anchor_b;
            const float dx = bx - ax, dy = by - ay;
            const float len = fmaxf(sqrtf(dx * dx + dy * dy), 1e-6f);
            const float ex = dx / len, ey = dy / len;
            const float lengthening = (bvx - avx) * ex + (bvy - avy) * ey;
            float drive = ms.y * ms.x;
            if (hill > 0.0f) {
                drive *= clampf(1.0f + lengthening * hill, 0.0f, 1.0f);
            }
            const float active = clampf(drive + lengthening * 0.15f, -cap, cap);
            const float work = fminf(drive, cap) * fmaxf(-lengthening, 0.0f) * C::h;
            t.muscle(k).x = clampf(ms.x - work * inv_capacity * p.inv_muscle_energy +
                                                 kMuscleRecovery * p.muscle_recovery * C::h * (1.0f - ms.x),
                                             0.0f, 1.0f);
            const float tendon = tendon_k * fmaxf(len - slack, 0.0f);
            const float pull = active + tendon;
            if (RECORD) {
                L.word(S.rec_pull + k / 4u, k % 4u) = pull;
            }
            const float fx = ex * pull, fy = ey * pull;
            // One 8-byte load and store per node, in the order a0, a1, b0,
            // b1 (two of them may be the same node).
            float2 g = t.f(a0);
            g.x += fx * (1.0f - anchor_a);
            g.y += fy * (1.0f - anchor_a);
            t.f(a0) = g;
            g = t.f(a1);
            g.x += fx * anchor_a;
            g.y += fy * anchor_a;
            t.f(a1) = g;
            g = t.f(b0);
            g.x -= fx * (1.0f - anchor_b);
            g.y -= fy * (1.0f - anchor_b);
            t.f(b0) = g;
            g = t.f(b1);
            g.x -= fx * anchor_b;
            g.y -= fy * anchor_b;
            t.f(b1) = g;
        }
    }

    // The world's force on node i (shaders/creature.cu:511-546).
    __device__ __forceinline__ float2 node_force(unsigned i, const float4& nr) const {
        const float m = nr.x;
        float fx = 0.0f, fy = -p.gravity * m;
        if (w.has(CE_FLAG_WIND)) {
            fx += p.wind * m;
        }
        float dry = 0.0f;
        if (w.has(CE_FLAG_MUD) || w.has(CE_FLAG_BRAMBLES)) {
            const float2 g = ground(w, t.pos(i).x, r.amp, r.qphase, p);
            dry = (t.pos(i).y - g.x) / sqrtf(1.0f + g.y * g.y) - nr.z;
        }
        if (w.has(CE_FLAG_MUD)) {
            fx -= m * kMudDrag * (clampf(-dry, 0.0f, p.mud) * (1.0f / kMudFullDepth)) * t.vel(i).x;
        }
        if (w.has(CE_FLAG_BRAMBLES)) {
            if (((r.feet >> i) & 1u) == 0u && dry < kBrambleReach) {
                fx -= m * p.brambles * t.vel(i).x;
            }
        }
        if (w.has(CE_FLAG_WATER)) {
            const float wet = clampf((p.water - (t.pos(i).y - nr.z)) / (2.0f * nr.z), 0.0f, 1.0f);
            fy += kWaterBuoyancy * m * p.gravity * wet;
        }
        return make_float2(fx, fy);
    }

    // Air and water drag on bone j (shaders/creature.cu:553-593), from its
    // lines `ba` (pivot, length, 1/m pivot, 1/m child) and `bb` (air drag
    // factor, drag limit, the two velocity scales); r0, r1 are the radii of
    // its two nodes (read only in a world with water).
    __device__ __forceinline__ void drag_item(unsigned j, const float4& ba, const float4& bb, float r0,
                                              float r1) const {
        const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
        const float2 v0 = t.vel(i0), v1 = t.vel(i1);
        const float wx = 0.5f * (v0.x + v1.x), wy = 0.5f * (v0.y + v1.y);
        const float speed = sqrtf(wx * wx + wy * wy);
        const float limit = bb.y;
        const float k_air = fminf(bb.x * speed, limit);
        float dfx = -wx * k_air, dfy = -wy * k_air;
        if (w.has(CE_FLAG_WATER)) {
            const float width = r0 + r1;
            const float2 p0 = t.pos(i0), p1 = t.pos(i1);
            const float wet0 = clampf((p.water - (p0.y - r0)) / (2.0f * r0), 0.0f, 1.0f);
            const float wet1 = clampf((p.water - (p1.y - r1)) / (2.0f * r1), 0.0f, 1.0f);
            const float wet = 0.5f * (wet0 + wet1);
            const float ax = (p1.x - p0.x) / ba.y, ay = (p1.y - p0.y) / ba.y;
            const float along = wx * ax + wy * ay;
            const float lx = ax * along, ly = ay * along;
            const float sx = wx - lx, sy = wy - ly;
            const float k_water = fminf(kWaterDrag * wet * ba.y * width * speed, limit);
            dfx -= sx * k_water + lx * k_water * kWaterAlong;
            dfy -= sy * k_water + ly * k_water * kWaterAlong;
        }
        const float s0 = bb.z, s1 = bb.w;
        t.vel(i0) = make_float2(v0.x + s0 * dfx, v0.y + s0 * dfy);
        t.vel(i1) = make_float2(v1.x + s1 * dfx, v1.y + s1 * dfy);
    }

    // Length of bone j (shaders/creature.cu:597-613).
    __device__ __forceinline__ void bone_item(unsigned j, const float4& ba) const {
        const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
        const float2 p0 = t.pos(i0), p1 = t.pos(i1);
        const float dx = p1.x - p0.x, dy = p1.y - p0.y;
        const float len = fmaxf(sqrtf(dx * dx + dy * dy), 1e-9f);
        const float w0 = ba.z, w1 = ba.w;
        const float s = (len - ba.y) / ((w0 + w1) * len);
        t.pos(i0) = make_float2(p0.x + w0 * s * dx, p0.y + w0 * s * dy);
        t.pos(i1) = make_float2(p1.x - w1 * s * dx, p1.y - w1 * s * dy);
    }

    // Range of joint j (shaders/creature.cu:618-634).
    __device__ __forceinline__ void limit_item(unsigned j, const float4& ra, const float4& rb) const {
        if (__float_as_uint(ra.x) == kNone) {
            return;
        }
        const Joint k = joint(j, ra, rb, true);
        float error = 0.0f;
        if (k.angle < k.lo) {
            error = k.angle - k.lo;
        }
        if (k.angle > k.hi) {
            error = k.angle - k.hi;
        }
        if (error == 0.0f) {
            return;
        }
        const float wgt = joint_weight(k);
        if (wgt > 0.0f) {
            joint_push<false>(k, -error / wgt);
        }
    }

    // Damping of joint j (shaders/creature.cu:683-702).
    __device__ __forceinline__ void damp_item(unsigned j, const float4& ra, const float4& rb) const {
        const float share = fminf(C::h * kInvJointDamping, 1.0f);
        if (__float_as_uint(ra.x) == kNone) {
            return;
        }
        const Joint k = joint(j, ra, rb, false);
        const float2 vt = t.vel(k.tip), vf = t.vel(k.far), vh = t.vel(k.hub);
        const float rate = k.g_tip.x * vt.x + k.g_tip.y * vt.y + k.g_far.x * vf.x + k.g_far.y * vf.y +
                           k.g_hub.x * vh.x + k.g_hub.y * vh.y;
        const float wgt = joint_weight(k);
        if (wgt > 0.0f) {
            joint_push<true>(k, -share * rate / wgt);
        }
    }

    // Whether joint j is past its range by more than kJointBreak
    // (shaders/creature.cu:746-759).
    __device__ __forceinline__ bool broken_item(unsigned j, const float4& ra, const float4& rb) const {
        if (__float_as_uint(ra.x) == kNone) {
            return false;
        }
        const Joint k = joint(j, ra, rb, true);
        return k.angle < k.lo - kJointBreak || k.angle > k.hi + kJointBreak;
    }

    // World force, muscle force and velocity of node i, then its predicted
    // position; the force table keeps the start position.
    __device__ __forceinline__ void integrate_item(unsigned i, const float4& nr) const {
        const float2 f = node_force(i, nr);
        float4 s = t.at(i);
        const float2 fpv = t.f(i);
        s.z += C::h * (f.x + fpv.x) * nr.y;
        s.w += C::h * (f.y + fpv.y) * nr.y;
        if (w.has(CE_FLAG_AIR)) {
            s.z *= p.air_sub;
            s.w *= p.air_sub;
        }
        t.f(i) = make_float2(s.x, s.y);
        s.x += C::h * s.z;
        s.y += C::h * s.w;
        t.set_at(i, s);
    }

    // Ground contact of node i, then its velocity from the substep's move.
    __device__ __forceinline__ void land_item(unsigned i, const float4& nr) const {
        float2 q = t.pos(i);
        const float2 f0 = t.f(i);
        solve_ground(i, nr, q, f0);
        t.vel(i) = make_float2((q.x - f0.x) * C::inv_h, (q.y - f0.y) * C::inv_h);
    }

    // ------------------------------------------------------------ passes
    // Air and water drag on the bones (shaders/creature.cu:553-593).
    __device__ __forceinline__ void bone_drag() const {
        const unsigned bones = r.nodes - 1u;
        if (w.has(CE_FLAG_WATER)) {
            // Water drag reads the bone's length and both radii as well.
            float4 na = L.get(S.bone), nb = L.get(S.bone + 1u);
            for (unsigned j = 0u; j < bones; j++) {
                const float4 ba = na, bb = nb;
                na = L.get(S.bone + 2u * j + 2u);
                nb = L.get(S.bone + 2u * j + 3u);
                const float r0 = L.get2(S.ground, __float_as_uint(ba.x)).x, r1 = L.get2(S.ground, j + 1u).x;
                drag_item(j, ba, bb, r0, r1);
            }
        } else {
            // Air drag needs only the pivot of line a.
            float na = L.get1(S.pivot, 0u);
            float4 nb = L.get(S.bone + 1u);
            for (unsigned j = 0u; j < bones; j++) {
                const float pivot = na;
                const float4 bb = nb;
                na = L.get1(S.pivot, j + 1u);
                nb = L.get(S.bone + 2u * j + 3u);
                drag_item(j, make_float4(pivot, 0.0f, 0.0f, 0.0f), bb, 0.0f, 0.0f);
            }
        }
    }

    // Bone lengths (shaders/creature.cu:597-613).
    __device__ __forceinline__ void solve_bones() const {
        const unsigned bones = r.nodes - 1u;
        float4 na = L.get(S.bone);
        for (unsigned j = 0u; j < bones; j++) {
            const float4 ba = na;
            na = L.get(S.bone + 2u * j + 2u);
            bone_item(j, ba);
        }
    }

    // Joint ranges (shaders/creature.cu:618-634).
    __device__ __forceinline__ void solve_joints() const {
        const unsigned bones = r.nodes - 1u;
        float4 na = L.get(S.joint + 2u), nb = L.get(S.joint + 3u);
        for (unsigned j = 1u; j < bones; j++) {
            const float4 ra = na, rb = nb;
            na = L.get(S.joint + 2u * j + 2u);
            nb = L.get(S.joint + 2u * j + 3u);
            limit_item(j, ra, rb);
        }
    }

    // Ground contact and friction of node i (shaders/creature.cu:640-679).
    // `q` is the node's position (updated and stored when it touches) and
    // `f0` its position at the start of the substep.
    __device__ __forceinline__ void solve_ground(unsigned i, const float4& nr, float2& q, const float2& f0) const {
        if (!w.has(CE_FLAG_GROUND)) {
            return;
        }
        const float2 g = ground(w, q.x, r.amp, r.qphase, p);
        const float secant = sqrtf(1.0f + g.y * g.y);
        const float nx = -g.y / secant, ny = 1.0f / secant;
        const float dry = (q.y - g.x) / secant - nr.z;
        float depth, mu;
        if (w.has(CE_FLAG_MUD)) {
            depth = -(dry + p.mud);
            const float sink = clampf(-dry, 0.0f, p.mud) * (1.0f / kMudFullDepth);
            mu = nr.w * p.friction * (1.0f + kMudGrip * sink) * (1.0f + kMudNormal * sink);
        } else {
            depth = -dry;
            mu = nr.w * p.friction;
        }
        if (depth <= 0.0f) {
            return;
        }
        if (w.has(CE_FLAG_ICE)) {
            mu *= 1.0f - p.patches * ice_at(q.x);
        }
        q.x += nx * depth;
        q.y += ny * depth;
        const float tx = ny, ty = -nx;
        const float slide = (q.x - f0.x) * tx + (q.y - f0.y) * ty;
        const float budget = mu * depth;
        const float back = fabsf(slide) <= budget ? slide : copysignf(budget, slide);
        q.x -= tx * back;
        q.y -= ty * back;
        t.pos(i) = q;
        if (RECORD) {
            float4 fl = L.get(S.rec_force + i);
            fl.x += nr.x * depth * C::inv_h * C::inv_h;
            fl.y += nr.x * back * C::inv_h * C::inv_h;
            L.put(S.rec_force + i, fl);
        }
    }

    // Joint damping (shaders/creature.cu:683-702).
    // Damping reads only the topology word of a joint's first line.
    __device__ __forceinline__ void damp_joints() const {
        const unsigned bones = r.nodes - 1u;
        float na = L.get1(S.topo, 1u);
        float4 nb = L.get(S.joint + 3u);
        for (unsigned j = 1u; j < bones; j++) {
            const float topo = na;
            const float4 rb = nb;
            na = L.get1(S.topo, j + 1u);
            nb = L.get(S.joint + 2u * j + 3u);
            damp_item(j, make_float4(topo, 0.0f, 0.0f, 0.0f), rb);
        }
    }

    // The per-node passes of a substep: `LAND` false integrates forces,
    // true does ground contact and velocities.
    // The force pass reads a node's (mass, 1/mass) half line, the ground
    // pass its (radius, friction) one; a world with water, mud or brambles
    // (whose forces read the radius) and a recording (whose contact forces
    // read the mass) read the whole node line.
    template <bool LAND>
    __device__ __forceinline__ void node_pass() const {
        const bool whole = LAND ? RECORD
                                : (w.has(CE_FLAG_WATER) || w.has(CE_FLAG_MUD) || w.has(CE_FLAG_BRAMBLES));
        if (whole) {
            float4 nn = L.get(S.node);
            for (unsigned i = 0u; i < r.nodes; i++) {
                const float4 nr = nn;
                nn = L.get(S.node + i + 1u);
                if (LAND) {
                    land_item(i, nr);
                } else {
                    integrate_item(i, nr);
                }
            }
        } else {
            const unsigned R = LAND ? S.ground : S.mass;
            float2 nn = L.get2(R, 0u);
            for (unsigned i = 0u; i < r.nodes; i++) {
                const float2 h = nn;
                nn = L.get2(R, i + 1u);
                if (LAND) {
                    land_item(i, make_float4(0.0f, 0.0f, h.x, h.y));
                } else {
                    integrate_item(i, make_float4(h.x, h.y, 0.0f, 0.0f));
                }
            }
        }
    }

    // One substep (shaders/creature.cu:705-742).
    __device__ __forceinline__ void substep() const {
        muscle_forces();
        bone_drag();
        node_pass<false>();
        solve_bones();
        solve_joints();
        node_pass<true>();
        damp_joints();
    }

    // Bits of the joints past their range by more than kJointBreak
    // (shaders/creature.cu:746-759).
    __device__ __forceinline__ unsigned long long broken_joints() const {
        unsigned long long bits = 0ull;
        const unsigned bones = r.nodes - 1u;
        float4 na = L.get(S.joint + 2u), nb = L.get(S.joint + 3u);
        for (unsigned j = 1u; j < bones; j++) {
            const float4 ra = na, rb = nb;
            na = L.get(S.joint + 2u * j + 2u);
            nb = L.get(S.joint + 2u * j + 3u);
            if (broken_item(j, ra, rb)) {
                bits |= 1ull << j;
            }
        }
        return bits;
    }
};

}  // namespace cek
