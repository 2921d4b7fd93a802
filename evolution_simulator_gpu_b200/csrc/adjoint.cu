// Gradients of a creature's fitness by the adjoint method, in the calm world
// (flat ground, gravity, air drag on the bones, no other effect) and in the
// effects worlds (rough and sloped ground with hurdles, optionally shaken by
// tremors, wind, thick air, water with buoyancy and drag, ice patches).
//
// Fitness is the centre of mass's x after the trial's last step (the fall
// step for a creature that falls, shaders/creature.cu:1060-1064, 1193-1194).
// The forward run is the creature kernel itself with a checkpoint of the
// state every 256 substeps (`advance_kernel<..., CKPT>`); its results are
// those of the plain kernel to the bit. The backward kernel then walks each
// creature's trial backwards a segment of 256 substeps at a time: it reruns
// the segment from its checkpoint and keeps the state at every substep start
// (the segment tape), then, substep by substep from the last, reruns the
// substep keeping what its passes need (the values each sequential
// projection saw, the positions before the ground pass, which joints were
// past their range, which nodes touched and slid) and carries the adjoint of
// the state back through damping, velocity, ground, joint limits, bone
// lengths, integration, bone drag and the muscles, adding up the gradient
// of every muscle and node parameter. Contact, stick or slip, joint-limit
// and clamp modes are the ones the forward run took: the gradient is that of
// the realised piecewise-smooth trajectory.
//
// At a clamp, min or max whose arguments are equal (common: every velocity is
// exactly zero at the start of a trial) the derivative passes to the
// argument itself, the convention of forward-mode dual numbers.
//
// Gradients are per record field (the kernel's parameters): for each muscle
// the stroke amplitude, hill factor, force cap, inverse energy capacity,
// phase, duty, 1 / duty, 1 / (1 - duty) and stiffness, for each node its
// friction, its mass and its start position. The host maps them to the genes.
#include <cuda_runtime.h>

#include <type_traits>

#include "trial.cuh"

namespace cek {

namespace {

using CalmWorld = StaticWorld<kWorldCalm>;
using EffectsWorld = StaticWorld<kWorldEffects>;
using QuakeWorld = StaticWorld<kWorldEffectsQuake>;

// d slope / d x of the ground under x: the terrain's second derivative (the
// slope, gap and hurdle terms are linear in x between their kinks).
template <class W>
__device__ __forceinline__ float ground_curvature(const W& w, float x, float amp, float qphase) {
    if (!w.has(CE_FLAG_TERRAIN)) {
        return 0.0f;
    }
    const float u0 = fracf(x * (1.0f / 1.1f) + qphase);
    const float u1 = fracf(x * (1.0f / 0.43f) + 0.3f + qphase);
    const float c0 = (1.0f - 2.0f * u0) * (1.0f - 2.0f * u0) - 2.0f * u0 * (1.0f - u0);
    const float c1 = (1.0f - 2.0f * u1) * (1.0f - 2.0f * u1) - 2.0f * u1 * (1.0f - u1);
    return amp * (0.65f * 32.0f * c0 * (1.0f / (1.1f * 1.1f)) + 0.35f * 32.0f * c1 * (1.0f / (0.43f * 0.43f)));
}

// d ice_at / d x (the smoothstep of ice_at; 0 outside its ramps).
__device__ __forceinline__ float ice_slope(float x) {
    const float w = fracf(x * kIceInv);
    const float t = fabsf(w - 0.5f) * 2.0f;
    const float z = (0.7f - t) * 2.5f;
    if (z < 0.0f || z > 1.0f) {
        return 0.0f;
    }
    const float dt = (w - 0.5f < 0.0f ? -2.0f : 2.0f) * kIceInv;
    return 6.0f * z * (1.0f - z) * -2.5f * dt;
}

// Lines of a lane's slot after the creature's constant lines (SlotLayout).
struct AdjointLayout {
    unsigned grad;    // 3 a muscle: (amp, hill, cap, 1/capacity), (phase, duty, 1/duty, 1/(1-duty)), (stiffness)
    unsigned fric;    // friction gradient, 4 nodes a line
    unsigned force;   // muscle force on each node in the substep, 2 nodes a line
    unsigned drag;    // bone j: the velocities of its ends before its drag
    unsigned bones;   // bone j: the positions of its ends before its projection
    unsigned joints;  // joint j: (parent tip, parent pivot), (tip, hub) positions before its test
    unsigned damp;    // joint j: (tip, far), (hub, -) velocities before its damping
    unsigned pj;      // positions after the joint pass, 2 nodes a line
    unsigned lines;
    __host__ __device__ static AdjointLayout make(unsigned rows, unsigned mm) {
        AdjointLayout A;
        unsigned at = SlotLayout::make(rows, mm, false).lines;
        A.grad = at;
        at += 3u * mm;
        A.fric = at;
        at += (rows + 3u) / 4u;
        A.force = at;
        at += (rows + 1u) / 2u;
        A.drag = at;
        at += rows - 1u;
        A.bones = at;
        at += rows - 1u;
        A.joints = at;
        at += 2u * (rows - 1u);
        A.damp = at;
        at += 2u * (rows - 1u);
        A.pj = at;
        at += (rows + 1u) / 2u;
        A.lines = at + 1u;  // a loop's load of the line after its last
        return A;
    }
};

// One substep's record in the segment tape: positions, velocities and
// energy stores at its start, float4 lines of a lane.
__host__ __device__ inline unsigned tape_lines(unsigned rows, unsigned mm) {
    return (checkpoint_floats(rows, mm) + 3u) / 4u;
}

struct Tape {
    float4* base;  // line 0 of substep 0 of this lane
    unsigned lines;
    __device__ __forceinline__ float* word(unsigned k, unsigned f) const {
        return reinterpret_cast<float*>(base + ((size_t)k * lines + f / 4u) * 32u) + (f % 4u);
    }
    __device__ __forceinline__ float2* pair(unsigned k, unsigned f) const {
        return reinterpret_cast<float2*>(base + ((size_t)k * lines + f / 4u) * 32u) + ((f % 4u) / 2u);
    }
};

struct AdjointArgs {
    float4* tape;           // segment tapes: warps of the grid x 256 substeps x tape lines x 32 lanes
    float* grads;           // grad_floats(rows, mm) a creature (packed index)
    const float* weights;   // dL/dfitness a creature (packed index), NULL for 1
    // The reruns' check, NULL for none: per creature (packed index) bit 0
    // when a segment's rerun from its checkpoint does not end on the next
    // checkpoint to the bit, bit 1 when a substep's kept rerun does not end
    // on the next tape state (or checkpoint).
    uint32_t* mismatch;
};

template <class W, int RATE>
struct Backward {
    using C = Clock<RATE>;
    using Body = Creature<W, RATE, false>;
    using T = Trial<W, false, RATE>;
    const Body& b;
    const NodeTables& g;  // adjoints: positions, velocities, start positions / forces, (energy, demand)
    float* gmass;         // d J / d mass of node i at gmass[i * g.stride] (shared memory)
    const AdjointLayout& A;
    const Tape& tape;
    const KernelArgs& a;
    const AdjointArgs& x;
    unsigned& end;  // steps of the trial
    unsigned& seg;  // segment to do next
    float& weight;  // d L / d fitness of the creature

    __device__ __forceinline__ void add_mass(unsigned i, float d) const { gmass[i * g.stride] += d; }

    // d J / d w for an inverse mass w = 1 / m, as d J / d m.
    __device__ __forceinline__ void add_inverse_mass(unsigned i, float w, float dw) const { add_mass(i, -dw * w * w); }

    __device__ __forceinline__ void add_line(unsigned line, float4 d) const {
        float4 v = b.L.get(line);
        v.x += d.x;
        v.y += d.y;
        v.z += d.z;
        v.w += d.w;
        b.L.put(line, v);
    }

    // Takes creature `cidx`: its constant lines, zeroed gradients and the
    // adjoint of the fitness (weight x d com_x / d position). False when the
    // trial failed or ran no step: its gradient is zero.
    __device__ __forceinline__ bool start(unsigned cidx) const {
        T::begin(b, a, cidx, 0u);
        LaneRegs& r = b.r;
        end = a.ends[cidx];
        weight = x.weights ? x.weights[cidx] : 1.0f;
        const bool usable = end > 0u && a.results[cidx].fitness > -1e19f;
        for (unsigned k = 0u; k < 3u * r.muscles; k++) {
            b.L.put(A.grad + k, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        }
        for (unsigned q = 0u; q < (r.nodes + 3u) / 4u; q++) {
            b.L.put(A.fric + q, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        }
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float m = b.L.get(b.S.node + i).x;
            g.pos(i) = make_float2(usable ? weight * m * r.inv_mass : 0.0f, 0.0f);
            g.vel(i) = make_float2(0.0f, 0.0f);
            g.f(i) = make_float2(0.0f, 0.0f);
            gmass[i * g.stride] = 0.0f;
        }
        for (unsigned k = 0u; k < r.muscles; k++) {
            g.muscle(k) = make_float2(0.0f, 0.0f);
        }
        seg = usable ? (end - 1u) / 16u : 0u;
        if (!usable) {
            finish(cidx);
        }
        return usable;
    }

    __device__ __forceinline__ void finish(unsigned cidx) const {
        const LaneRegs& r = b.r;
        float* out = x.grads + (size_t)cidx * grad_floats(a.rows, a.mm);
        for (unsigned k = 0u; k < r.muscles; k++) {
            const float4 g0 = b.L.get(A.grad + 3u * k), g1 = b.L.get(A.grad + 3u * k + 1u);
            const float g2 = b.L.get(A.grad + 3u * k + 2u).x;
            float* o = out + kGradMuscle * k;
            o[0] = g0.x;
            o[1] = g0.y;
            o[2] = g0.z;
            o[3] = g0.w;
            o[4] = g1.x;
            o[5] = g1.y;
            o[6] = g1.z;
            o[7] = g1.w;
            o[8] = g2;
        }
        for (unsigned i = 0u; i < r.nodes; i++) {
            out[kGradMuscle * a.mm + i] = b.L.word(A.fric + i / 4u, i % 4u);
            out[kGradMuscle * a.mm + a.rows + i] = gmass[i * g.stride];
            // The adjoint of the start position (the tables hold the state's
            // adjoint at the start of the trial once every segment is done).
            const float2 l0 = g.pos(i);
            out[kGradMuscle * a.mm + 2u * a.rows + 2u * i] = l0.x;
            out[kGradMuscle * a.mm + 2u * a.rows + 2u * i + 1u] = l0.y;
        }
    }

    // The segment tape streams through L2 (2.2 MB a warp at 12 node rows and
    // 20 muscle slots, each substep's state written once and read back by
    // the reverse pass up to 255 substeps later), so its stores and loads
    // carry the evict-first hint and leave L2 to the lane slots.
    __device__ __forceinline__ void load_state(unsigned k) const {
        const LaneRegs& r = b.r;
        for (unsigned i = 0u; i < r.nodes; i++) {
            b.t.pos(i) = __ldcs(tape.pair(k, 2u * i));
            b.t.vel(i) = __ldcs(tape.pair(k, 2u * a.rows + 2u * i));
        }
        for (unsigned m = 0u; m < r.muscles; m++) {
            b.t.muscle(m).x = __ldcs(tape.word(k, 4u * a.rows + m));
        }
    }

    __device__ __forceinline__ void save_state(unsigned k) const {
        const LaneRegs& r = b.r;
        for (unsigned i = 0u; i < r.nodes; i++) {
            __stcs(tape.pair(k, 2u * i), b.t.pos(i));
            __stcs(tape.pair(k, 2u * a.rows + 2u * i), b.t.vel(i));
        }
        for (unsigned m = 0u; m < r.muscles; m++) {
            __stcs(tape.word(k, 4u * a.rows + m), b.t.muscle(m).x);
        }
    }

    // Whether the tables hold tape entry k's state (positions, velocities,
    // energy stores), to the bit.
    __device__ __forceinline__ bool same_as_tape(unsigned k) const {
        const LaneRegs& r = b.r;
        bool same = true;
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float2 q = *tape.pair(k, 2u * i), v = *tape.pair(k, 2u * a.rows + 2u * i);
            const float2 tq = b.t.pos(i), tv = b.t.vel(i);
            same = same && __float_as_uint(q.x) == __float_as_uint(tq.x) && __float_as_uint(q.y) == __float_as_uint(tq.y) &&
                   __float_as_uint(v.x) == __float_as_uint(tv.x) && __float_as_uint(v.y) == __float_as_uint(tv.y);
        }
        for (unsigned m = 0u; m < r.muscles; m++) {
            same = same && __float_as_uint(*tape.word(k, 4u * a.rows + m)) == __float_as_uint(b.t.muscle(m).x);
        }
        return same;
    }

    // Whether the tables hold checkpoint s, to the bit.
    __device__ __forceinline__ bool same_as_checkpoint(unsigned s) const {
        const LaneRegs& r = b.r;
        const size_t n = a.count;
        const float* c = a.ckpt + (size_t)s * checkpoint_floats(a.rows, a.mm) * n + r.cidx;
        bool same = true;
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float2 tq = b.t.pos(i), tv = b.t.vel(i);
            same = same && __float_as_uint(c[(2u * i) * n]) == __float_as_uint(tq.x) &&
                   __float_as_uint(c[(2u * i + 1u) * n]) == __float_as_uint(tq.y) &&
                   __float_as_uint(c[(2u * a.rows + 2u * i) * n]) == __float_as_uint(tv.x) &&
                   __float_as_uint(c[(2u * a.rows + 2u * i + 1u) * n]) == __float_as_uint(tv.y);
        }
        for (unsigned m = 0u; m < r.muscles; m++) {
            same = same && __float_as_uint(c[(4u * a.rows + m) * n]) == __float_as_uint(b.t.muscle(m).x);
        }
        return same;
    }

    __device__ __forceinline__ void load_checkpoint(unsigned s) const {
        const LaneRegs& r = b.r;
        const size_t n = a.count;
        const float* c = a.ckpt + (size_t)s * checkpoint_floats(a.rows, a.mm) * n + r.cidx;
        for (unsigned i = 0u; i < r.nodes; i++) {
            b.t.pos(i) = make_float2(c[(2u * i) * n], c[(2u * i + 1u) * n]);
            b.t.vel(i) = make_float2(c[(2u * a.rows + 2u * i) * n], c[(2u * a.rows + 2u * i + 1u) * n]);
        }
        for (unsigned m = 0u; m < r.muscles; m++) {
            b.t.muscle(m).x = c[(4u * a.rows + m) * n];
        }
    }

    // The substep of Creature::substep, keeping what the reverse passes read.
    // Returns the joints past their range (bit j) and sets `touch` (nodes in
    // contact) and `slip` (contacts that slid). Its passes load the next
    // item's lines while working on the current one, as the forward passes
    // do; it must land on the forward run's states to the bit, which the
    // checked backward (AdjointArgs::mismatch) verifies.
    __device__ __forceinline__ unsigned substep_kept(unsigned& touch, unsigned& slip) const {
        const LaneRegs& r = b.r;
        const NodeTables& t = b.t;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const unsigned bones = r.nodes - 1u;
        b.muscle_forces();
        float4 ka = L.get(S.bone), kb = L.get(S.bone + 1u);
        for (unsigned j = 0u; j < bones; j++) {
            const float4 ba = ka, bb = kb;
            ka = L.get(S.bone + 2u * j + 2u);
            kb = L.get(S.bone + 2u * j + 3u);
            const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
            const float2 v0 = t.vel(i0), v1 = t.vel(i1);
            L.put(A.drag + j, make_float4(v0.x, v0.y, v1.x, v1.y));
            const float wx = 0.5f * (v0.x + v1.x), wy = 0.5f * (v0.y + v1.y);
            const float speed = sqrtf(wx * wx + wy * wy);
            const float limit = bb.y;
            const float k_air = fminf(bb.x * speed, limit);
            float dfx = -wx * k_air, dfy = -wy * k_air;
            if (b.w.has(CE_FLAG_WATER)) {
                const float r0 = L.get(S.node + i0).z, r1 = L.get(S.node + i1).z;
                const float width = r0 + r1;
                const float2 p0 = t.pos(i0), p1 = t.pos(i1);
                const float wet0 = clampf((b.p.water - (p0.y - r0)) / (2.0f * r0), 0.0f, 1.0f);
                const float wet1 = clampf((b.p.water - (p1.y - r1)) / (2.0f * r1), 0.0f, 1.0f);
                const float wet = 0.5f * (wet0 + wet1);
                const float ax = (p1.x - p0.x) / ba.y, ay = (p1.y - p0.y) / ba.y;
                const float along = wx * ax + wy * ay;
                const float lx = ax * along, ly = ay * along;
                const float sx = wx - lx, sy = wy - ly;
                const float k_water = fminf(kWaterDrag * wet * ba.y * width * speed, limit);
                dfx -= sx * k_water + lx * k_water * kWaterAlong;
                dfy -= sy * k_water + ly * k_water * kWaterAlong;
            }
            t.vel(i0) = make_float2(v0.x + bb.z * dfx, v0.y + bb.z * dfy);
            t.vel(i1) = make_float2(v1.x + bb.w * dfx, v1.y + bb.w * dfy);
        }
        float4 kn = L.get(S.node);
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float4 nr = kn;
            kn = L.get(S.node + i + 1u);
            const float2 f = b.node_force(i, nr);
            float4 s = t.at(i);
            const float2 fpv = t.f(i);
            reinterpret_cast<float2*>(&L.base[(A.force + i / 2u) * 32u])[i % 2u] = fpv;
            s.z += C::h * (f.x + fpv.x) * nr.y;
            s.w += C::h * (f.y + fpv.y) * nr.y;
            if (b.w.has(CE_FLAG_AIR)) {
                s.z *= b.p.air_sub;
                s.w *= b.p.air_sub;
            }
            t.f(i) = make_float2(s.x, s.y);
            s.x += C::h * s.z;
            s.y += C::h * s.w;
            t.set_at(i, s);
        }
        float4 kba = L.get(S.bone);
        for (unsigned j = 0u; j < bones; j++) {
            const float4 ba = kba;
            kba = L.get(S.bone + 2u * j + 2u);
            const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
            const float2 p0 = t.pos(i0), p1 = t.pos(i1);
            L.put(A.bones + j, make_float4(p0.x, p0.y, p1.x, p1.y));
            const float dx = p1.x - p0.x, dy = p1.y - p0.y;
            const float len = fmaxf(sqrtf(dx * dx + dy * dy), 1e-9f);
            const float w0 = ba.z, w1 = ba.w;
            const float sc = (len - ba.y) / ((w0 + w1) * len);
            t.pos(i0) = make_float2(p0.x + w0 * sc * dx, p0.y + w0 * sc * dy);
            t.pos(i1) = make_float2(p1.x - w1 * sc * dx, p1.y - w1 * sc * dy);
        }
        unsigned violated = 0u;
        float4 kra = L.get(S.joint + 2u), krb = L.get(S.joint + 3u);
        for (unsigned j = 1u; j < bones; j++) {
            const float4 ra = kra, rb = krb;
            kra = L.get(S.joint + 2u * j + 2u);
            krb = L.get(S.joint + 2u * j + 3u);
            if (__float_as_uint(ra.x) == kNone) {
                continue;
            }
            const unsigned topo = __float_as_uint(ra.x);
            const unsigned hub = topo & 31u, ptip = (topo >> 5u) & 31u, ppivot = (topo >> 10u) & 31u;
            const float2 pt = t.pos(ptip), pp = t.pos(ppivot), ct = t.pos(j + 1u), ch = t.pos(hub);
            L.put(A.joints + 2u * j, make_float4(pt.x, pt.y, pp.x, pp.y));
            L.put(A.joints + 2u * j + 1u, make_float4(ct.x, ct.y, ch.x, ch.y));
            const typename Body::Joint k = b.joint(j, ra, rb, true);
            float error = 0.0f;
            if (k.angle < k.lo) {
                error = k.angle - k.lo;
            }
            if (k.angle > k.hi) {
                error = k.angle - k.hi;
            }
            if (error == 0.0f) {
                continue;
            }
            const float wgt = Body::joint_weight(k);
            if (wgt > 0.0f) {
                violated |= 1u << j;
                b.template joint_push<false>(k, -error / wgt);
            }
        }
        touch = 0u;
        slip = 0u;
        float4 gn = L.get(S.node);
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float4 nr = gn;
            gn = L.get(S.node + i + 1u);
            float2 q = t.pos(i);
            const float2 f0 = t.f(i);
            float* pj = reinterpret_cast<float*>(&L.base[(A.pj + i / 2u) * 32u]) + 2u * (i % 2u);
            pj[0] = q.x;
            pj[1] = q.y;
            const float2 before = q;
            b.solve_ground(i, nr, q, f0);
            // The ground pass's contact and stick/slip tests, on the same
            // values.
            const Contact c = contact(before, f0, nr);
            if (c.depth > 0.0f) {
                touch |= 1u << i;
                if (!(fabsf(c.slide) <= c.mu * c.depth)) {
                    slip |= 1u << i;
                }
            }
            t.vel(i) = make_float2((q.x - f0.x) * C::inv_h, (q.y - f0.y) * C::inv_h);
        }
        float4 dra = L.get(S.joint + 2u), drb = L.get(S.joint + 3u);
        for (unsigned j = 1u; j < bones; j++) {
            const float4 ra = dra, rb = drb;
            dra = L.get(S.joint + 2u * j + 2u);
            drb = L.get(S.joint + 2u * j + 3u);
            if (__float_as_uint(ra.x) == kNone) {
                continue;
            }
            const typename Body::Joint k = b.joint(j, ra, rb, false);
            const float2 vt = t.vel(k.tip), vf = t.vel(k.far), vh = t.vel(k.hub);
            L.put(A.damp + 2u * j, make_float4(vt.x, vt.y, vf.x, vf.y));
            L.put(A.damp + 2u * j + 1u, make_float4(vh.x, vh.y, 0.0f, 0.0f));
            const float share = fminf(C::h * kInvJointDamping, 1.0f);
            const float rate = k.g_tip.x * vt.x + k.g_tip.y * vt.y + k.g_far.x * vf.x + k.g_far.y * vf.y +
                               k.g_hub.x * vh.x + k.g_hub.y * vh.y;
            const float wgt = Body::joint_weight(k);
            if (wgt > 0.0f) {
                b.template joint_push<true>(k, -share * rate / wgt);
            }
        }
        return violated;
    }

    // The ground pass's contact of a node at q (Creature::solve_ground's
    // arithmetic): the ground's height and slope under q.x, its secant and
    // normal, the depth, the friction coefficient and the slide along the
    // surface after the push out.
    struct Contact {
        float2 gr, n, q1;
        float secant, depth, mu, ice, slide;
    };
    __device__ __forceinline__ Contact contact(float2 q, float2 f0, const float4& nr) const {
        Contact c;
        c.gr = ground(b.w, q.x, b.r.amp, b.r.qphase, b.p);
        c.secant = sqrtf(1.0f + c.gr.y * c.gr.y);
        c.n = make_float2(-c.gr.y / c.secant, 1.0f / c.secant);
        const float dry = (q.y - c.gr.x) / c.secant - nr.z;
        c.depth = -dry;
        c.mu = nr.w * b.p.friction;
        c.ice = 1.0f;
        if (b.w.has(CE_FLAG_ICE)) {
            c.ice = 1.0f - b.p.patches * ice_at(q.x);
            c.mu *= c.ice;
        }
        c.q1 = make_float2(q.x + c.n.x * c.depth, q.y + c.n.y * c.depth);
        const float tx = c.n.y, ty = -c.n.x;
        c.slide = (c.q1.x - f0.x) * tx + (c.q1.y - f0.y) * ty;
        return c;
    }

    // Adjoint of node i's ground contact (pushed out along the normal, then
    // held or slid back along the surface) from the position before it `q`,
    // the substep's start position `f0` and the adjoint of the result in the
    // table; the start position's share goes to g.f.
    __device__ __forceinline__ void ground_back(unsigned i, const float4& nr, float2 q, float2 f0,
                                                bool slipped) const {
        const Contact c = contact(q, f0, nr);
        const float S = c.gr.y, sec = c.secant, nx = c.n.x, ny = c.n.y;
        const float tx = ny, ty = -nx;
        const float budget = c.mu * c.depth;
        const float back = slipped ? copysignf(budget, c.slide) : c.slide;
        const float2 l2 = g.pos(i);
        float2 lq1 = l2;
        float ltx = -back * l2.x, lty = -back * l2.y;
        const float lback = -(l2.x * tx + l2.y * ty);
        float ldepth = 0.0f, lmu = 0.0f, lslide = 0.0f;
        if (slipped) {
            const float lbudget = c.slide < 0.0f ? -lback : lback;
            lmu = lbudget * c.depth;
            ldepth = lbudget * c.mu;
        } else {
            lslide = lback;
        }
        lq1.x += lslide * tx;
        lq1.y += lslide * ty;
        float2 lf = g.f(i);
        lf.x -= lslide * tx;
        lf.y -= lslide * ty;
        g.f(i) = lf;
        ltx += lslide * (c.q1.x - f0.x);
        lty += lslide * (c.q1.y - f0.y);
        float lny = ltx, lnx = -lty;
        float2 lq = lq1;
        lnx += lq1.x * c.depth;
        lny += lq1.y * c.depth;
        ldepth += lq1.x * nx + lq1.y * ny;
        float lx = 0.0f;
        if (lmu != 0.0f) {
            b.L.word(A.fric + i / 4u, i % 4u) += lmu * b.p.friction * c.ice;
            if (b.w.has(CE_FLAG_ICE)) {
                lx -= lmu * nr.w * b.p.friction * b.p.patches * ice_slope(q.x);
            }
        }
        // depth = radius - (q.y - height) / secant
        lq.y -= ldepth / sec;
        const float lheight = ldepth / sec;
        float lsec = ldepth * (q.y - c.gr.x) / (sec * sec);
        // n = (-slope, 1) / secant, secant = sqrt(1 + slope^2)
        float lslope = -lnx / sec;
        lsec += (lnx * S - lny) / (sec * sec);
        lslope += lsec * S / sec;
        lx += lheight * S + lslope * ground_curvature(b.w, q.x, b.r.amp, b.r.qphase);
        lq.x += lx;
        g.pos(i) = lq;
    }

    // A push node += w lam g with lam = -e / wgt, wgt = sum w |g|^2: the
    // inverse mass w's share, from the post-push adjoint `ap` of the node
    // and the adjoint `lwgt` of wgt.
    __device__ __forceinline__ void weights_back(unsigned node, float w, float2 gv, float2 ap, float lam,
                                                 float lwgt) const {
        add_inverse_mass(node, w, lam * (gv.x * ap.x + gv.y * ap.y) + lwgt * (gv.x * gv.x + gv.y * gv.y));
    }

    // Adjoint of the joint geometry: carries the adjoints of the two
    // gradient vectors (lg_tip of g_tip = perp(v) / |v|^2 and lg_u of
    // g_u = perp(u) / |u|^2) to u = parent tip - parent pivot and
    // v = tip - hub.
    __device__ __forceinline__ static void perp_back(float2 w, float ww, float2 gw, float2 lg, float2& lw) {
        // gw = (-w.y, w.x) / ww; d gw = R dw / ww - gw (2 w . dw) / ww
        lw.x += lg.y / ww;
        lw.y += -lg.x / ww;
        if (ww >= 1e-12f && w.x * w.x + w.y * w.y >= 1e-12f) {
            const float c = 2.0f * (lg.x * gw.x + lg.y * gw.y) / ww;
            lw.x -= c * w.x;
            lw.y -= c * w.y;
        }
    }

    __device__ __forceinline__ void reverse_substep(unsigned k_tape, unsigned violated, unsigned touch,
                                                    unsigned slip) const {
        const LaneRegs& r = b.r;
        const NodeTables& t = b.t;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const ce_params& p = b.p;
        const unsigned bones = r.nodes - 1u;
        // Damping, joints from last to first; positions are those after the
        // ground pass (the table holds them). Here and in the bone, node,
        // drag and muscle loops below, the next item's lines load while the
        // current item is worked on; the extra load at a loop's end reads an
        // item of the creature's own (joint 0, bone 0) or the line after the
        // last, which the slot holds.
        const float share = fminf(C::h * kInvJointDamping, 1.0f);
        float4 na = L.get(S.joint + 2u * (bones - 1u)), nb = L.get(S.joint + 2u * (bones - 1u) + 1u);
        float4 nd0 = L.get(A.damp + 2u * (bones - 1u)), nd1 = L.get(A.damp + 2u * (bones - 1u) + 1u);
        for (unsigned j = bones; j-- > 1u;) {
            const float4 ra = na, rb = nb, d0 = nd0, d1 = nd1;
            na = L.get(S.joint + 2u * (j - 1u));
            nb = L.get(S.joint + 2u * (j - 1u) + 1u);
            nd0 = L.get(A.damp + 2u * (j - 1u));
            nd1 = L.get(A.damp + 2u * (j - 1u) + 1u);
            if (__float_as_uint(ra.x) == kNone) {
                continue;
            }
            const typename Body::Joint k = b.joint(j, ra, rb, false);
            const float wgt = Body::joint_weight(k);
            if (!(wgt > 0.0f)) {
                continue;
            }
            const float2 vt = make_float2(d0.x, d0.y), vf = make_float2(d0.z, d0.w), vh = make_float2(d1.x, d1.y);
            const float rate = k.g_tip.x * vt.x + k.g_tip.y * vt.y + k.g_far.x * vf.x + k.g_far.y * vf.y +
                               k.g_hub.x * vh.x + k.g_hub.y * vh.y;
            const float lam = -share * rate / wgt;
            const float2 at = g.vel(k.tip), af = g.vel(k.far), ah = g.vel(k.hub);
            const float llam = k.w_tip * (k.g_tip.x * at.x + k.g_tip.y * at.y) +
                               k.w_far * (k.g_far.x * af.x + k.g_far.y * af.y) +
                               k.w_hub * (k.g_hub.x * ah.x + k.g_hub.y * ah.y);
            const float lrate = -share * llam / wgt;
            const float lwgt = llam * share * rate / (wgt * wgt);
            float2 lgt = make_float2(k.w_tip * lam * at.x + lrate * vt.x + 2.0f * k.w_tip * k.g_tip.x * lwgt,
                                     k.w_tip * lam * at.y + lrate * vt.y + 2.0f * k.w_tip * k.g_tip.y * lwgt);
            float2 lgf = make_float2(k.w_far * lam * af.x + lrate * vf.x + 2.0f * k.w_far * k.g_far.x * lwgt,
                                     k.w_far * lam * af.y + lrate * vf.y + 2.0f * k.w_far * k.g_far.y * lwgt);
            const float2 lgh = make_float2(k.w_hub * lam * ah.x + lrate * vh.x + 2.0f * k.w_hub * k.g_hub.x * lwgt,
                                           k.w_hub * lam * ah.y + lrate * vh.y + 2.0f * k.w_hub * k.g_hub.y * lwgt);
            lgt.x -= lgh.x;
            lgt.y -= lgh.y;
            lgf.x -= lgh.x;
            lgf.y -= lgh.y;
            g.vel(k.tip) = make_float2(at.x + lrate * k.g_tip.x, at.y + lrate * k.g_tip.y);
            g.vel(k.far) = make_float2(af.x + lrate * k.g_far.x, af.y + lrate * k.g_far.y);
            g.vel(k.hub) = make_float2(ah.x + lrate * k.g_hub.x, ah.y + lrate * k.g_hub.y);
            weights_back(k.tip, k.w_tip, k.g_tip, at, lam, lwgt);
            weights_back(k.far, k.w_far, k.g_far, af, lam, lwgt);
            weights_back(k.hub, k.w_hub, k.g_hub, ah, lam, lwgt);
            geometry_back(ra, j, k, lgt, lgf, 0.0f);
        }
        // Velocity from the positions: v = (q - q0) / h.
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float2 lv = g.vel(i);
            float2 lq = g.pos(i);
            lq.x += lv.x * C::inv_h;
            lq.y += lv.y * C::inv_h;
            g.pos(i) = lq;
            g.f(i) = make_float2(-lv.x * C::inv_h, -lv.y * C::inv_h);
            g.vel(i) = make_float2(0.0f, 0.0f);
        }
        // Ground contact.
        // The substep's start positions come from the tape: the forward
        // force table and the adjoint force table share memory.
        float4 cn = L.get(S.node);
        float2 cq = reinterpret_cast<const float2*>(&L.base[A.pj * 32u])[0], cf = *tape.pair(k_tape, 0u);
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float4 nr = cn;
            const float2 q = cq, f0 = cf;
            cn = L.get(S.node + i + 1u);
            cq = reinterpret_cast<const float2*>(&L.base[(A.pj + (i + 1u) / 2u) * 32u])[(i + 1u) % 2u];
            cf = *tape.pair(k_tape, 2u * (i + 1u));
            if (((touch >> i) & 1u) == 0u) {
                continue;
            }
            ground_back(i, nr, q, f0, ((slip >> i) & 1u) != 0u);
        }
        // Joint limits, last to first, on the joints that were pushed.
        for (unsigned j = bones; j-- > 1u;) {
            if (((violated >> j) & 1u) == 0u) {
                continue;
            }
            const float4 ra = L.get(S.joint + 2u * j), rb = L.get(S.joint + 2u * j + 1u);
            const float4 e0 = L.get(A.joints + 2u * j), e1 = L.get(A.joints + 2u * j + 1u);
            joint_limit_back(j, ra, rb, e0, e1);
        }
        // Bone lengths, last to first.
        float4 nba = L.get(S.bone + 2u * (bones - 1u)), npre = L.get(A.bones + bones - 1u);
        for (unsigned j = bones; j-- > 0u;) {
            const float4 ba = nba, pre = npre;
            const unsigned jn = j > 0u ? j - 1u : 0u;
            nba = L.get(S.bone + 2u * jn);
            npre = L.get(A.bones + jn);
            const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
            const float dx = pre.z - pre.x, dy = pre.w - pre.y;
            const float len0 = sqrtf(dx * dx + dy * dy);
            const float len = fmaxf(len0, 1e-9f);
            const float w0 = ba.z, w1 = ba.w;
            const float sc = (len - ba.y) / ((w0 + w1) * len);
            const float2 l0 = g.pos(i0), l1 = g.pos(i1);
            const float ls = w0 * (dx * l0.x + dy * l0.y) - w1 * (dx * l1.x + dy * l1.y);
            float ldx = w0 * sc * l0.x - w1 * sc * l1.x, ldy = w0 * sc * l0.y - w1 * sc * l1.y;
            if (len0 >= 1e-9f) {
                const float llen = ls * ba.y / ((w0 + w1) * len * len);
                ldx += llen * dx / len;
                ldy += llen * dy / len;
            }
            g.pos(i0) = make_float2(l0.x - ldx, l0.y - ldy);
            g.pos(i1) = make_float2(l1.x + ldx, l1.y + ldy);
            // s = (len - L) / ((w0 + w1) len): ds/dw0 = ds/dw1 = -s / (w0 + w1).
            const float lsw = -ls * sc / (w0 + w1);
            add_inverse_mass(i0, w0, sc * (dx * l0.x + dy * l0.y) + lsw);
            add_inverse_mass(i1, w1, -sc * (dx * l1.x + dy * l1.y) + lsw);
        }
        // Integration: q1 = q0 + h v1, v1 = a (v + h (f_world + f_muscle) / m)
        // (a the thick air's retention, 1 without), and the start position
        // kept for the velocity pass. Mass: the world force is a mass times
        // an acceleration (gravity, wind, buoyancy), so the m-derivative of
        // v1 is -a h F / m^2. Buoyancy's depth goes to the start height.
        float4 nnr = L.get(S.node);
        float2 nF = reinterpret_cast<const float2*>(&L.base[A.force * 32u])[0];
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float4 nr = nnr;
            const float2 F = nF;
            nnr = L.get(S.node + i + 1u);
            nF = reinterpret_cast<const float2*>(&L.base[(A.force + (i + 1u) / 2u) * 32u])[(i + 1u) % 2u];
            const float im = nr.y;
            const float2 lq1 = g.pos(i), lq0 = g.f(i);
            float2 lp = make_float2(lq1.x + lq0.x, lq1.y + lq0.y);
            float2 lv1 = make_float2(C::h * lq1.x, C::h * lq1.y);
            if (b.w.has(CE_FLAG_AIR)) {
                lv1.x *= p.air_sub;
                lv1.y *= p.air_sub;
            }
            if (b.w.has(CE_FLAG_WATER)) {
                const float y0 = tape.pair(k_tape, 2u * i)->y;
                const float z = (p.water - (y0 - nr.z)) / (2.0f * nr.z);
                if (z >= 0.0f && z <= 1.0f) {
                    lp.y -= lv1.y * C::h * im * kWaterBuoyancy * nr.x * p.gravity / (2.0f * nr.z);
                }
            }
            g.pos(i) = lp;
            g.vel(i) = lv1;
            g.f(i) = make_float2(lv1.x * C::h * im, lv1.y * C::h * im);
            add_mass(i, -C::h * im * im * (lv1.x * F.x + lv1.y * F.y));
        }
        // Bone drag, last to first.
        float4 dba = L.get(S.bone + 2u * (bones - 1u)), dbb = L.get(S.bone + 2u * (bones - 1u) + 1u);
        float4 dpre = L.get(A.drag + bones - 1u);
        for (unsigned j = bones; j-- > 0u;) {
            const float4 ba = dba, bb = dbb, pre = dpre;
            const unsigned jn = j > 0u ? j - 1u : 0u;
            dba = L.get(S.bone + 2u * jn);
            dbb = L.get(S.bone + 2u * jn + 1u);
            dpre = L.get(A.drag + jn);
            const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
            const float wx = 0.5f * (pre.x + pre.z), wy = 0.5f * (pre.y + pre.w);
            const float speed = sqrtf(wx * wx + wy * wy);
            const float limit = bb.y;
            const float k_air = fminf(bb.x * speed, limit);
            const float2 l0 = g.vel(i0), l1 = g.vel(i1);
            const float ldx = bb.z * l0.x + bb.w * l1.x, ldy = bb.z * l0.y + bb.w * l1.y;
            float lwx = -k_air * ldx, lwy = -k_air * ldy;
            const float lk = -(wx * ldx + wy * ldy);
            float lspeed = 0.0f, llimit = 0.0f;
            if (bb.x * speed <= limit) {
                lspeed += lk * bb.x;
            } else {
                llimit += lk;
            }
            float dfx = -wx * k_air, dfy = -wy * k_air;
            if (b.w.has(CE_FLAG_WATER)) {
                // Water drag from the bone's wet share at the substep's start
                // positions: across the bone in full, along it by kWaterAlong.
                const float r0 = L.get(S.node + i0).z, r1 = L.get(S.node + i1).z;
                const float width = r0 + r1;
                const float2 p0 = *tape.pair(k_tape, 2u * i0), p1 = *tape.pair(k_tape, 2u * i1);
                const float z0 = (p.water - (p0.y - r0)) / (2.0f * r0);
                const float z1 = (p.water - (p1.y - r1)) / (2.0f * r1);
                const float wet = 0.5f * (clampf(z0, 0.0f, 1.0f) + clampf(z1, 0.0f, 1.0f));
                const float ax = (p1.x - p0.x) / ba.y, ay = (p1.y - p0.y) / ba.y;
                const float along = wx * ax + wy * ay;
                const float lx = ax * along, ly = ay * along;
                const float sx = wx - lx, sy = wy - ly;
                const float xw = kWaterDrag * wet * ba.y * width * speed;
                const float k_water = fminf(xw, limit);
                dfx -= sx * k_water + lx * k_water * kWaterAlong;
                dfy -= sy * k_water + ly * k_water * kWaterAlong;
                const float lkw = -(sx * ldx + sy * ldy) - kWaterAlong * (lx * ldx + ly * ldy);
                // s = w - l, l = a (w . a)
                const float lsx = -k_water * ldx, lsy = -k_water * ldy;
                const float llx = -k_water * kWaterAlong * ldx - lsx, lly = -k_water * kWaterAlong * ldy - lsy;
                lwx += lsx;
                lwy += lsy;
                const float lalong = llx * ax + lly * ay;
                lwx += lalong * ax;
                lwy += lalong * ay;
                const float lax = llx * along + lalong * wx, lay = lly * along + lalong * wy;
                float lwet = 0.0f;
                if (xw <= limit) {
                    lwet = lkw * kWaterDrag * ba.y * width * speed;
                    lspeed += lkw * kWaterDrag * wet * ba.y * width;
                } else {
                    llimit += lkw;
                }
                float2 e = g.pos(i0);
                e.x -= lax / ba.y;
                e.y -= lay / ba.y;
                if (z0 >= 0.0f && z0 <= 1.0f) {
                    e.y -= 0.5f * lwet / (2.0f * r0);
                }
                g.pos(i0) = e;
                e = g.pos(i1);
                e.x += lax / ba.y;
                e.y += lay / ba.y;
                if (z1 >= 0.0f && z1 <= 1.0f) {
                    e.y -= 0.5f * lwet / (2.0f * r1);
                }
                g.pos(i1) = e;
            }
            if (speed > 0.0f) {
                lwx += lspeed * wx / speed;
                lwy += lspeed * wy / speed;
            }
            if (llimit != 0.0f) {
                // The limit 0.5 (m0 + m1) / h.
                add_mass(i0, 0.5f * C::inv_h * llimit);
                add_mass(i1, 0.5f * C::inv_h * llimit);
            }
            // The scales 0.5 h / m of the two ends.
            add_inverse_mass(i0, L.get(S.node + i0).y, 0.5f * C::h * (l0.x * dfx + l0.y * dfy));
            add_inverse_mass(i1, L.get(S.node + i1).y, 0.5f * C::h * (l1.x * dfx + l1.y * dfy));
            g.vel(i0) = make_float2(l0.x + 0.5f * lwx, l0.y + 0.5f * lwy);
            g.vel(i1) = make_float2(l1.x + 0.5f * lwx, l1.y + 0.5f * lwy);
        }
        // Muscles, from the substep's start state.
        load_state(k_tape);
        muscles_back();
    }

    // Adjoint of a joint's geometry given the adjoints of its gradient
    // vectors g_tip (lgt) and g_far (lgf, g_hub's share already folded in),
    // and of its angle (lturn, 0 for damping).
    __device__ __forceinline__ void geometry_back(const float4& ra, unsigned j, const typename Body::Joint& k,
                                                  float2 lgt, float2 lgf, float lturn) const {
        const NodeTables& t = b.t;
        const unsigned topo = __float_as_uint(ra.x);
        const unsigned ptip = (topo >> 5u) & 31u, ppivot = (topo >> 10u) & 31u;
        const bool at_head = ((topo >> 20u) & 1u) != 0u;
        const float2 pt = t.pos(ptip), pp = t.pos(ppivot), ct = t.pos(k.tip), ch = t.pos(k.hub);
        geometry_back_at(pt, pp, ct, ch, ptip, ppivot, k.tip, k.hub, at_head, lgt, lgf, lturn);
    }

    __device__ __forceinline__ void geometry_back_at(float2 pt, float2 pp, float2 ct, float2 ch, unsigned ptip,
                                                     unsigned ppivot, unsigned tip, unsigned hub, bool at_head,
                                                     float2 lgt, float2 lgf, float lturn) const {
        const float2 u = make_float2(pt.x - pp.x, pt.y - pp.y);
        const float2 v = make_float2(ct.x - ch.x, ct.y - ch.y);
        const float uu = fmaxf(u.x * u.x + u.y * u.y, 1e-12f), vv = fmaxf(v.x * v.x + v.y * v.y, 1e-12f);
        const float2 g_tip = make_float2(-v.y / vv, v.x / vv);
        const float2 g_u = make_float2(-u.y / uu, u.x / uu);
        const float2 lgu = at_head ? make_float2(-lgf.x, -lgf.y) : lgf;
        float2 lu = make_float2(0.0f, 0.0f), lv = make_float2(0.0f, 0.0f);
        perp_back(v, vv, g_tip, lgt, lv);
        perp_back(u, uu, g_u, lgu, lu);
        if (lturn != 0.0f) {
            const float cr = u.x * v.y - u.y * v.x, dt = u.x * v.x + u.y * v.y;
            const float den = cr * cr + dt * dt;
            if (den > 0.0f) {
                const float lc = lturn * dt / den, ld = -lturn * cr / den;
                lu.x += lc * v.y + ld * v.x;
                lu.y += -lc * v.x + ld * v.y;
                lv.x += -lc * u.y + ld * u.x;
                lv.y += lc * u.x + ld * u.y;
            }
        }
        float2 e = g.pos(ptip);
        g.pos(ptip) = make_float2(e.x + lu.x, e.y + lu.y);
        e = g.pos(ppivot);
        g.pos(ppivot) = make_float2(e.x - lu.x, e.y - lu.y);
        e = g.pos(tip);
        g.pos(tip) = make_float2(e.x + lv.x, e.y + lv.y);
        e = g.pos(hub);
        g.pos(hub) = make_float2(e.x - lv.x, e.y - lv.y);
    }

    // Adjoint of a joint-limit push from the positions its test saw.
    __device__ __forceinline__ void joint_limit_back(unsigned j, const float4& ra, const float4& rb, const float4& e0,
                                                     const float4& e1) const {
        const unsigned topo = __float_as_uint(ra.x);
        const unsigned hub = topo & 31u, ptip = (topo >> 5u) & 31u, ppivot = (topo >> 10u) & 31u;
        const unsigned far = (topo >> 15u) & 31u, tip = j + 1u;
        const bool at_head = ((topo >> 20u) & 1u) != 0u;
        const float2 pt = make_float2(e0.x, e0.y), pp = make_float2(e0.z, e0.w);
        const float2 ct = make_float2(e1.x, e1.y), ch = make_float2(e1.z, e1.w);
        const float2 u = make_float2(pt.x - pp.x, pt.y - pp.y);
        const float2 v = make_float2(ct.x - ch.x, ct.y - ch.y);
        const float uu = fmaxf(u.x * u.x + u.y * u.y, 1e-12f), vv = fmaxf(v.x * v.x + v.y * v.y, 1e-12f);
        const float turn = atan2f(u.x * v.y - u.y * v.x, u.x * v.x + u.y * v.y);
        const float mid = ra.w;
        const float angle = mid + wrapf(turn - mid);
        const float lo = ra.y, hi = ra.z;
        float error = 0.0f;
        if (angle < lo) {
            error = angle - lo;
        }
        if (angle > hi) {
            error = angle - hi;
        }
        const float2 g_tip = make_float2(-v.y / vv, v.x / vv);
        const float2 g_u = make_float2(-u.y / uu, u.x / uu);
        const float2 g_far = at_head ? make_float2(-g_u.x, -g_u.y) : g_u;
        const float2 g_hub = make_float2(-(g_tip.x + g_far.x), -(g_tip.y + g_far.y));
        const float w_tip = rb.x, w_far = rb.y, w_hub = rb.z;
        const float wgt = w_tip * (g_tip.x * g_tip.x + g_tip.y * g_tip.y) +
                          w_far * (g_far.x * g_far.x + g_far.y * g_far.y) +
                          w_hub * (g_hub.x * g_hub.x + g_hub.y * g_hub.y);
        const float lam = -error / wgt;
        const float2 at = g.pos(tip), af = g.pos(far), ah = g.pos(hub);
        const float llam = w_tip * (g_tip.x * at.x + g_tip.y * at.y) + w_far * (g_far.x * af.x + g_far.y * af.y) +
                           w_hub * (g_hub.x * ah.x + g_hub.y * ah.y);
        const float lerr = -llam / wgt;
        const float lwgt = llam * error / (wgt * wgt);
        float2 lgt = make_float2(w_tip * lam * at.x + 2.0f * w_tip * g_tip.x * lwgt,
                                 w_tip * lam * at.y + 2.0f * w_tip * g_tip.y * lwgt);
        float2 lgf = make_float2(w_far * lam * af.x + 2.0f * w_far * g_far.x * lwgt,
                                 w_far * lam * af.y + 2.0f * w_far * g_far.y * lwgt);
        const float2 lgh = make_float2(w_hub * lam * ah.x + 2.0f * w_hub * g_hub.x * lwgt,
                                       w_hub * lam * ah.y + 2.0f * w_hub * g_hub.y * lwgt);
        lgt.x -= lgh.x;
        lgt.y -= lgh.y;
        lgf.x -= lgh.x;
        lgf.y -= lgh.y;
        weights_back(tip, w_tip, g_tip, at, lam, lwgt);
        weights_back(far, w_far, g_far, af, lam, lwgt);
        weights_back(hub, w_hub, g_hub, ah, lam, lwgt);
        geometry_back_at(pt, pp, ct, ch, ptip, ppivot, tip, hub, at_head, lgt, lgf, lerr);
    }

    // Adjoint of the muscle pass (shaders/creature.cu:455-508) from the
    // substep's start state in the tables, the adjoints of the forces in
    // g.f and of the new energy stores in g.muscle().x.
    __device__ __forceinline__ void muscles_back() const {
        const LaneRegs& r = b.r;
        const NodeTables& t = b.t;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const ce_params& p = b.p;
        const float c = kMuscleRecovery * p.muscle_recovery * C::h;
        float4 n0 = L.get(S.muscle + kPull0), nacc = L.get(A.grad);
        float2 nc = L.get2(S.cap, 0u), nt = r.tendon ? L.get2(S.tendon, 0u) : make_float2(0.0f, 0.0f);
        for (unsigned k = 0u; k < r.muscles; k++) {
            const float4 q0 = n0, acc = nacc;
            const float2 qc = nc, qt = nt;
            n0 = L.get(S.muscle + 5u * (k + 1u) + kPull0);
            nacc = L.get(A.grad + 3u * (k + 1u));
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
            const float len0 = sqrtf(dx * dx + dy * dy);
            const float len = fmaxf(len0, 1e-6f);
            const float ex = dx / len, ey = dy / len;
            const float rvx = bvx - avx, rvy = bvy - avy;
            const float lengthening = rvx * ex + rvy * ey;
            const float drive0 = ms.y * ms.x;
            float drive = drive0, hc = 1.0f, hz = 0.0f;
            if (hill > 0.0f) {
                hz = 1.0f + lengthening * hill;
                hc = clampf(hz, 0.0f, 1.0f);
                drive = drive0 * hc;
            }
            const float ya = drive + lengthening * 0.15f;
            const float active = clampf(ya, -cap, cap);
            const float m1 = fminf(drive, cap), m2 = fmaxf(-lengthening, 0.0f);
            const float work = m1 * m2 * C::h;
            const float z = ms.x - work * inv_capacity * p.inv_muscle_energy + c * (1.0f - ms.x);
            const float tendon = tendon_k * fmaxf(len - slack, 0.0f);
            const float pull = active + tendon;
            // Adjoint of the pull from the forces on its four nodes.
            const float2 fa0 = g.f(a0), fa1 = g.f(a1), fb0 = g.f(b0), fb1 = g.f(b1);
            const float lfx = (1.0f - anchor_a) * fa0.x + anchor_a * fa1.x - (1.0f - anchor_b) * fb0.x -
                              anchor_b * fb1.x;
            const float lfy = (1.0f - anchor_a) * fa0.y + anchor_a * fa1.y - (1.0f - anchor_b) * fb0.y -
                              anchor_b * fb1.y;
            const float lpull = lfx * ex + lfy * ey;
            float lex = lfx * pull, ley = lfy * pull;
            const float2 lm = g.muscle(k);
            // Energy store: e1 = clamp(z, 0, 1).
            const float lz = (z >= 0.0f && z <= 1.0f) ? lm.x : 0.0f;
            float le = lz * (1.0f - c);
            const float lwork = -lz * inv_capacity * p.inv_muscle_energy;
            float g_icap = -lz * work * p.inv_muscle_energy;
            float g_cap = 0.0f, g_hill = 0.0f;
            float ldrive = 0.0f, llg = 0.0f, llen = 0.0f;
            const float lm1 = lwork * m2 * C::h, lm2 = lwork * m1 * C::h;
            if (drive <= cap) {
                ldrive += lm1;
            } else {
                g_cap += lm1;
            }
            if (-lengthening >= 0.0f) {
                llg -= lm2;
            }
            if (len - slack >= 0.0f) {
                llen += lpull * tendon_k;
            }
            if (ya >= -cap && ya <= cap) {
                ldrive += lpull;
                llg += 0.15f * lpull;
            } else if (ya > cap) {
                g_cap += lpull;
            } else {
                g_cap -= lpull;
            }
            float ldrive0 = ldrive;
            if (hill > 0.0f) {
                ldrive0 = ldrive * hc;
                if (hz >= 0.0f && hz <= 1.0f) {
                    const float lhc = ldrive * drive0;
                    llg += lhc * hill;
                    g_hill += lhc * lengthening;
                }
            }
            const float ld = ldrive0 * ms.x;
            le += ldrive0 * ms.y;
            // Lengthening speed along the unit direction.
            const float lrvx = llg * ex, lrvy = llg * ey;
            lex += llg * rvx;
            ley += llg * rvy;
            // e = d / len
            float ldx = lex / len, ldy = ley / len;
            llen -= (lex * ex + ley * ey) / len;
            if (len0 >= 1e-6f) {
                ldx += llen * dx / len;
                ldy += llen * dy / len;
            }
            // Anchors on the two bones.
            float2 e;
            e = g.pos(a0);
            g.pos(a0) = make_float2(e.x - (1.0f - anchor_a) * ldx, e.y - (1.0f - anchor_a) * ldy);
            e = g.pos(a1);
            g.pos(a1) = make_float2(e.x - anchor_a * ldx, e.y - anchor_a * ldy);
            e = g.pos(b0);
            g.pos(b0) = make_float2(e.x + (1.0f - anchor_b) * ldx, e.y + (1.0f - anchor_b) * ldy);
            e = g.pos(b1);
            g.pos(b1) = make_float2(e.x + anchor_b * ldx, e.y + anchor_b * ldy);
            e = g.vel(a0);
            g.vel(a0) = make_float2(e.x - (1.0f - anchor_a) * lrvx, e.y - (1.0f - anchor_a) * lrvy);
            e = g.vel(a1);
            g.vel(a1) = make_float2(e.x - anchor_a * lrvx, e.y - anchor_a * lrvy);
            e = g.vel(b0);
            g.vel(b0) = make_float2(e.x + (1.0f - anchor_b) * lrvx, e.y + (1.0f - anchor_b) * lrvy);
            e = g.vel(b1);
            g.vel(b1) = make_float2(e.x + anchor_b * lrvx, e.y + anchor_b * lrvy);
            g.muscle(k) = make_float2(le, lm.y + ld);
            L.put(A.grad + 3u * k, make_float4(acc.x + 0.0f, acc.y + g_hill, acc.z + g_cap, acc.w + g_icap));
        }
    }

    // Adjoint of the step's muscle demands (shaders/creature.cu:442-451)
    // from the demands' adjoints summed over its substeps.
    __device__ __forceinline__ void demands_back(float t_now) const {
        const LaneRegs& r = b.r;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        for (unsigned k = 0u; k < r.muscles; k++) {
            const float ld = g.muscle(k).y;
            g.muscle(k).y = 0.0f;
            const unsigned m0 = S.muscle + 5u * k;
            const float4 r0 = L.get_cold(m0 + kRhythm0), r1 = L.get_cold(m0 + kRhythm1);
            const float offset = L.word_cold(m0 + kMState, 2);
            const float before = rhythm(t_now, r0.y, r0.z, offset, r0.w, r1.x, r1.y);
            const float after = rhythm(t_now + C::dt, r0.y, r0.z, offset, r0.w, r1.x, r1.y);
            const float shortening = r0.x * (after - before) * C::rate;
            const float xd = shortening * r1.z * 0.25f;
            if (r.limp || xd < 0.0f || ld == 0.0f) {
                continue;
            }
            const float lsh = ld * r1.z * 0.25f;
            const float g_stiff = ld * shortening * 0.25f;
            const float g_amp = lsh * (after - before) * C::rate;
            const float lr = lsh * r0.x * C::rate;
            float4 g1 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            rhythm_back(t_now + C::dt, r0, r1, offset, lr, g1);
            rhythm_back(t_now, r0, r1, offset, -lr, g1);
            add_line(A.grad + 3u * k, make_float4(g_amp, 0.0f, 0.0f, 0.0f));
            add_line(A.grad + 3u * k + 1u, g1);
            add_line(A.grad + 3u * k + 2u, make_float4(g_stiff, 0.0f, 0.0f, 0.0f));
        }
    }

    // d rhythm(t) into (phase, duty, 1/duty, 1/(1-duty)) times `lr`.
    __device__ __forceinline__ static void rhythm_back(float t, const float4& r0, const float4& r1, float offset,
                                                       float lr, float4& g1) {
        const float ph = fracf(t * r0.y + r0.z + offset);
        const float duty = r0.w, inv_duty = r1.x, inv_comp = r1.y;
        if (ph < duty) {
            const float arg = kPiF * ph * inv_duty;
            const float sn = __sinf(arg);
            g1.x += lr * 0.5f * kPiF * inv_duty * sn;  // d/d phase
            g1.z += lr * 0.5f * kPiF * ph * sn;        // d/d (1/duty)
        } else {
            const float arg = kPiF * (ph - duty) * inv_comp;
            const float sn = __sinf(arg);
            g1.x += -lr * 0.5f * kPiF * inv_comp * sn;
            g1.y += lr * 0.5f * kPiF * inv_comp * sn;          // d/d duty
            g1.w += -lr * 0.5f * kPiF * (ph - duty) * sn;      // d/d (1/(1-duty))
        }
    }

    // One segment, backwards. Returns whether segments remain.
    __device__ __forceinline__ bool segment() const {
        const unsigned s0 = seg * 16u, s1 = min(s0 + 16u, end);
        load_checkpoint(seg);
        for (unsigned s = s0; s < s1; s++) {
            b.muscle_demands((float)s * C::dt);
            for (unsigned q = 0u; q < 16u; q++) {
                save_state((s - s0) * 16u + q);
                b.substep();
            }
        }
        if (x.mismatch && s1 < end && !same_as_checkpoint(s1 / 16u)) {
            atomicOr(x.mismatch + b.r.cidx, 1u);
        }
        if (s1 == end) {
            // Fitness com_x = sum m x / sum m: d/dm_i = (x_i - com_x) / sum m.
            const LaneRegs& r = b.r;
            float com_x = 0.0f;
            for (unsigned i = 0u; i < r.nodes; i++) {
                com_x += b.L.get(b.S.node + i).x * b.t.pos(i).x;
            }
            com_x *= r.inv_mass;
            for (unsigned i = 0u; i < r.nodes; i++) {
                add_mass(i, weight * r.inv_mass * (b.t.pos(i).x - com_x));
            }
        }
        for (unsigned s = s1; s-- > s0;) {
            const float t_now = (float)s * C::dt;
            b.muscle_demands(t_now);
            for (unsigned q = 16u; q-- > 0u;) {
                const unsigned k = (s - s0) * 16u + q;
                load_state(k);
                unsigned touch, slip;
                const unsigned violated = substep_kept(touch, slip);
                if (x.mismatch) {
                    const bool last = k + 1u == (s1 - s0) * 16u;
                    if (last ? (s1 < end && !same_as_checkpoint(s1 / 16u)) : !same_as_tape(k + 1u)) {
                        atomicOr(x.mismatch + b.r.cidx, 2u);
                    }
                }
                reverse_substep(k, violated, touch, slip);
            }
            demands_back(t_now);
        }
        if (seg == 0u) {
            return false;
        }
        seg--;
        return true;
    }
};

// The tangent-linear run (Tangent, tangent_kernel), the adjoint's check.
#include "tangent.cuh"

template <class W, int RATE>
__global__ void __launch_bounds__(kBlock, 2) adjoint_kernel(const KernelArgs a, const ce_params p,
                                                            const AdjointArgs x) {
    extern __shared__ float4 smem[];
    using B = Backward<W, RATE>;
    const unsigned threads = blockDim.x;
    float2* const tables = reinterpret_cast<float2*>(smem) + threadIdx.x;
    // Tables of rows x threads entries: positions, velocities, the adjoints
    // of both, one force table (the forward passes' forces and start
    // positions, then the reverse passes' adjoints of those: each is dead
    // while the other is in use), the mass gradients (one float an entry),
    // then the muscles' (energy, demand) pairs and their adjoints.
    const size_t node_table = (size_t)a.rows * threads, muscle_table = (size_t)(a.mm > 0u ? a.mm : 1u) * threads;
    float2* const forces = tables + 4u * node_table;
    float* const gmass = reinterpret_cast<float*>(reinterpret_cast<float2*>(smem) + 5u * node_table) + threadIdx.x;
    float2* const muscles = reinterpret_cast<float2*>(smem) + 5u * node_table + node_table / 2u + threadIdx.x;
    const NodeTables tab{tables, tables + node_table, forces, muscles};
    const NodeTables adj{tables + 2u * node_table, tables + 3u * node_table, forces, muscles + muscle_table};
    const SlotLayout S = SlotLayout::make(a.rows, a.mm, false);
    const AdjointLayout A = AdjointLayout::make(a.rows, a.mm);
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = (blockIdx.x * threads + threadIdx.x) >> 5u;
    const unsigned warps_total = gridDim.x * (threads >> 5u);
    const Lines L = Lines::make(a.scratch + (size_t)warp * A.lines * 32u, lane);
    const unsigned tl = tape_lines(a.rows, a.mm);
    const Tape tape{x.tape + (size_t)warp * 256u * tl * 32u + lane, tl};
    const W w{};
    LaneRegs r;
    const typename B::Body body{w, p, tab, L, S, r};
    unsigned end = 0u, seg = 0u;
    float weight = 1.0f;
    const B back{body, adj, gmass, A, tape, a, x, end, seg, weight};
    bool live = false;
    Claim claim(a, lane, warp, warps_total);
    for (;;) {
        const unsigned mine = claim.next(live);
        unsigned done_cidx = kNone;
        if (mine != kNone) {
            const unsigned cidx = a.order ? __ldg(a.order + mine) : p.base + mine;
            live = back.start(cidx);
        }
        if (__ballot_sync(kFull, live) == 0u) {
            if (claim.drained) {
                break;
            }
            continue;
        }
        if (live) {
            live = back.segment();
            if (!live) {
                done_cidx = r.cidx;
            }
        }
        if (done_cidx != kNone) {
            back.finish(done_cidx);
        }
    }
}

}  // namespace

size_t adjoint_smem_bytes(unsigned rows, unsigned mm, unsigned block) {
    return (size_t)block * (rows * 44u + (mm > 0u ? mm : 1u) * 16u);
}

size_t adjoint_slot_bytes(unsigned grid, unsigned rows, unsigned mm) {
    const size_t warps = (size_t)grid * (kBlock / 32u);
    return warps * (size_t)AdjointLayout::make(rows, mm).lines * 32u * 16u;
}

size_t adjoint_tape_bytes(unsigned grid, unsigned rows, unsigned mm) {
    const size_t warps = (size_t)grid * (kBlock / 32u);
    return warps * 256u * (size_t)tape_lines(rows, mm) * 32u * 16u;
}

// The worlds with gradients, as compile-time worlds: f(world, rate).
template <class F>
cudaError_t with_gradient_world(uint32_t flags, int rate, F&& f) {
    auto at = [&](auto w) -> cudaError_t {
        if (rate == 60) return f(w, std::integral_constant<int, 60>{});
        if (rate == 120) return f(w, std::integral_constant<int, 120>{});
        return cudaErrorInvalidValue;
    };
    switch (flags) {
        case kWorldCalm: return at(CalmWorld{});
        case kWorldEffects: return at(EffectsWorld{});
        case kWorldEffectsQuake: return at(QuakeWorld{});
        default: return cudaErrorInvalidValue;
    }
}

bool gradient_world(uint32_t flags) {
    return flags == kWorldCalm || flags == kWorldEffects || flags == kWorldEffectsQuake;
}

cudaError_t adjoint_occupancy(unsigned rows, unsigned mm, uint32_t flags, int rate, int* blocks) {
    const size_t smem = adjoint_smem_bytes(rows, mm, kBlock);
    return with_gradient_world(flags, rate, [&](auto w, auto r) -> cudaError_t {
        auto kern = adjoint_kernel<decltype(w), decltype(r)::value>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, kern, (int)kBlock, smem);
    });
}

cudaError_t launch_forward_ckpt(const LaunchSpec& s, const KernelArgs& a, const ce_params& p) {
    if (s.record || a.rows != s.rows || a.mm != s.mm) return cudaErrorInvalidValue;
    const size_t smem = smem_bytes(s.rows, s.mm, s.block);
    return with_gradient_world(s.flags, s.rate, [&](auto w, auto r) -> cudaError_t {
        auto kern = advance_kernel<decltype(w), false, decltype(r)::value, true>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<s.grid, s.block, smem, s.stream>>>(a, p, w);
        return cudaGetLastError();
    });
}

size_t tangent_smem_bytes(unsigned rows, unsigned mm, unsigned block) {
    return (size_t)block * (rows * 48u + (mm > 0u ? mm : 1u) * 16u);
}

bool tangent_world(uint32_t flags) { return gradient_world(flags); }

cudaError_t launch_tangent(const LaunchSpec& s, const KernelArgs& a, const ce_params& p, const float* dstart,
                           const float* dmuscle, const float* dfriction, const float* dmass, float* dfitness) {
    if (s.record || a.rows != s.rows || a.mm != s.mm || !tangent_world(s.flags)) return cudaErrorInvalidValue;
    const size_t smem = tangent_smem_bytes(s.rows, s.mm, s.block);
    return with_gradient_world(s.flags, s.rate, [&](auto w, auto r) -> cudaError_t {
        auto kern = tangent_kernel<decltype(w), decltype(r)::value>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<s.grid, s.block, smem, s.stream>>>(a, p, dstart, dmuscle, dfriction, dmass, dfitness);
        return cudaGetLastError();
    });
}

cudaError_t launch_adjoint(const LaunchSpec& s, const KernelArgs& a, const ce_params& p, float4* tape, float* grads,
                           const float* weights, uint32_t* mismatch) {
    if (s.record || a.rows != s.rows || a.mm != s.mm) return cudaErrorInvalidValue;
    const size_t smem = adjoint_smem_bytes(s.rows, s.mm, s.block);
    const AdjointArgs x{tape, grads, weights, mismatch};
    return with_gradient_world(s.flags, s.rate, [&](auto w, auto r) -> cudaError_t {
        auto kern = adjoint_kernel<decltype(w), decltype(r)::value>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<s.grid, s.block, smem, s.stream>>>(a, p, x);
        return cudaGetLastError();
    });
}

}  // namespace cek
