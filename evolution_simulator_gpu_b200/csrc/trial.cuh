// One creature's trial on one lane (begin and step) and the persistent
// launch that runs them: the creature kernel family, included by the
// launchers of the plain kernels and of the gradient kernels.
#pragma once
#include <cuda_runtime.h>

#include "advance.cuh"
#include "kernels.h"

namespace cek {

constexpr unsigned kFull = 0xffffffffu;
static_assert(NodeTables::stride == kBlock, "node table rows are one block wide");

template <class W, bool RECORD, int RATE, bool CKPT = false>
struct Trial {
    using C = Clock<RATE>;
    using Body = Creature<W, RATE, RECORD>;

    // Frame t of a recording (shaders/creature.cu:767-779): the reference's
    // frame slots, stored frame-major and creature-minor (slot s of frame t
    // of recorded creature c at (t * stride + s) * count + c), so the lanes
    // of a warp, which record consecutive creatures in step with each other,
    // store each slot as one coalesced run. frames_to_creature_major turns
    // them into the reference's creature-major layout.
    __device__ __forceinline__ static void record_frame(const Body& b, const KernelArgs& a, unsigned t) {
        const unsigned stride = b.p.stride;
        const size_t k = a.count;
        float2* fr = a.frames + (size_t)t * stride * k + b.r.rec_slot;
        for (unsigned i = 0u; i < b.r.nodes; i++) {
            const float4 fl = b.L.get(b.S.rec_force + i);
            fr[i * k] = b.t.pos(i);
            fr[(CE_MAX_NODES + b.r.muscles + i) * k] = make_float2(fl.x, fl.y);
        }
        for (unsigned m = 0u; m < b.r.muscles; m++) {
            fr[(CE_MAX_NODES + m) * k] = make_float2(b.t.muscle(m).x, b.L.word(b.S.rec_pull + m / 4u, m % 4u));
        }
        const unsigned long long broken = b.broken_joints();
        fr[(stride - 1u) * k] =
            make_float2(__uint_as_float((unsigned)broken), __uint_as_float((unsigned)(broken >> 32)));
    }

    // Checkpoint `k` of the creature (the state at substep 256 k): positions,
    // velocities and energy stores, the whole state that the substeps carry
    // from one step to the next in a world without touch sensors. Stored
    // creature-minor, so that the lanes of a warp (creatures claimed in
    // packed order) write neighbouring words.
    __device__ __forceinline__ static void save_checkpoint(const Body& b, const KernelArgs& a, unsigned k) {
        const size_t n = a.count;
        float* c = a.ckpt + (size_t)k * checkpoint_floats(a.rows, a.mm) * n + b.r.cidx;
        for (unsigned i = 0u; i < b.r.nodes; i++) {
            const float2 q = b.t.pos(i), v = b.t.vel(i);
            __stcs(c + (2u * i) * n, q.x);
            __stcs(c + (2u * i + 1u) * n, q.y);
            __stcs(c + (2u * a.rows + 2u * i) * n, v.x);
            __stcs(c + (2u * a.rows + 2u * i + 1u) * n, v.y);
        }
        for (unsigned k2 = 0u; k2 < b.r.muscles; k2++) {
            __stcs(c + (4u * a.rows + k2) * n, b.t.muscle(k2).x);
        }
    }

    // Starts creature `cidx` on this lane (shaders/creature.cu:845-950).
    __device__ __forceinline__ static void begin(const Body& b, const KernelArgs& a, unsigned cidx,
                                                 unsigned slot) {
        LaneRegs& r = b.r;
        const ce_params& p = b.p;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const uint4 h0 = __ldcs(&a.heads[2u * cidx]);
        const uint4 h1 = __ldcs(&a.heads[2u * cidx + 1u]);
        r.cidx = cidx;
        r.rec_slot = slot;
        r.nodes = h0.x & 255u;
        r.muscles = h0.y;
        const uint32_t* rec = a.records + h0.w;
        const float* mus = a.muscles + h1.x;
        r.inv_mass = __uint_as_float(h1.z);
        r.flags = h1.w >> 16u;
        r.period_f = h2f(h1.w & 0xffffu);
        if (b.w.has(CE_FLAG_QUAKE)) {
            r.qphase = (float)(h0.z & 0xffffu) * (1.0f / 65536.0f);
            r.amp = p.terrain + p.quake * (0.6f + (float)((h0.z >> 16u) & 0xffffu) * (0.8f / 65536.0f));
        } else {
            r.qphase = 0.0f;
            r.amp = p.terrain;
        }
        r.feet = 0u;
        for (unsigned i = 0u; i < r.nodes; i++) {
            const uint32_t* q = rec + i * CE_NODE_WORDS;
            const float m = __uint_as_float(__ldcs(q + 0));
            const float radius = __uint_as_float(__ldcs(q + 1)), friction = __uint_as_float(__ldcs(q + 2));
            L.put(S.node + i, make_float4(m, 1.0f / m, radius, friction));
            L.put2(S.mass, i, make_float2(m, 1.0f / m));
            L.put2(S.ground, i, make_float2(radius, friction));
            b.t.set_at(i, make_float4(__uint_as_float(__ldcs(q + 3)), __uint_as_float(__ldcs(q + 4)), 0.0f, 0.0f));
            r.feet |= (__ldcs(q + 5) & 1u) << i;
            if (RECORD) {
                L.put(S.rec_force + i, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
            }
        }
        const uint32_t* bone_rec = rec + r.nodes * CE_NODE_WORDS;
        const unsigned bones = r.nodes - 1u;
        for (unsigned j = 0u; j < bones; j++) {
            const uint32_t* q = bone_rec + j * CE_BONE_WORDS;
            const unsigned i0 = __ldcs(q + 0), i1 = j + 1u;
            const float length = __uint_as_float(__ldcs(q + 1));
            const float4 n0 = L.get(S.node + i0), n1 = L.get(S.node + i1);
            const float width = n0.z + n1.z;
            const float bone_mass = n0.x + n1.x;
            L.put(S.bone + 2u * j, make_float4(__uint_as_float(i0), length, n0.y, n1.y));
            L.put(S.bone + 2u * j + 1u, make_float4(kAirDrag * length * width, 0.5f * bone_mass * C::inv_h,
                                                    0.5f * C::h * n0.y, 0.5f * C::h * n1.y));
            float4 ra = make_float4(__uint_as_float(kNone), 0.0f, 0.0f, 0.0f);
            float4 rb = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const unsigned pj = __ldcs(q + 2);
            if (j > 0u && pj != kNone) {
                const unsigned hub = i0, parent_pivot = __ldcs(bone_rec + pj * CE_BONE_WORDS);
                const bool at_head = hub == parent_pivot;
                const unsigned far = at_head ? pj + 1u : parent_pivot;
                const unsigned topo =
                    hub | ((pj + 1u) << 5u) | (parent_pivot << 10u) | (far << 15u) | ((at_head ? 1u : 0u) << 20u);
                const float lo = __uint_as_float(__ldcs(q + 3)), hi = __uint_as_float(__ldcs(q + 4));
                ra = make_float4(__uint_as_float(topo), lo, hi, 0.5f * (lo + hi));
                rb = make_float4(n1.y, L.get(S.node + far).y, n0.y, 0.0f);
            }
            L.put(S.joint + 2u * j, ra);
            L.put(S.joint + 2u * j + 1u, rb);
            L.put1(S.pivot, j, __uint_as_float(i0));
            L.put1(S.topo, j, ra.x);
        }
        r.tendon = false;
        for (unsigned k = 0u; k < r.muscles; k++) {
            const float4* q = reinterpret_cast<const float4*>(mus + k * CE_MUSCLE_FIELDS);
            const unsigned m0 = S.muscle + 5u * k;
            const float4 pull1 = __ldcs(q + 1);
            L.put(m0 + kPull0, __ldcs(q + 0));
            L.put(m0 + kPull1, pull1);
            L.put2(S.cap, k, make_float2(pull1.x, pull1.y));
            L.put2(S.tendon, k, make_float2(pull1.z, pull1.w));
            r.tendon = r.tendon || pull1.z != 0.0f;
            L.put_cold(m0 + kRhythm0, __ldcs(q + 2));
            L.put_cold(m0 + kRhythm1, __ldcs(q + 3));
            L.put_cold(m0 + kMState, make_float4(0.0f, 0.0f, 0.0f, __ldcs(q + 4).x));
            b.t.muscle(k) = make_float2(1.0f, 0.0f);
            if (RECORD) {
                L.word(S.rec_pull + k / 4u, k % 4u) = 0.0f;
            }
        }
        // The result starts at 0 except the lowest and highest mean height.
        const float2 head = b.t.pos(0u);
        float lw[36];
#pragma unroll
        for (unsigned q = 0u; q < 36u; q++) {
            lw[q] = 0.0f;
        }
        lw[2] = 1e20f;
        lw[3] = -1e20f;
        lw[kWHeadAt] = head.x;
        lw[kWHeadAt + 1u] = head.y;
#pragma unroll
        for (unsigned q = 0u; q < 9u; q++) {
            L.put_cold(S.lane + q, make_float4(lw[4u * q], lw[4u * q + 1u], lw[4u * q + 2u], lw[4u * q + 3u]));
        }
        r.limp = false;
        r.scoring = true;
        r.step = 0u;
        if (RECORD) {
            for (unsigned t = 0u; t <= C::settle; t++) {
                record_frame(b, a, t);
            }
        }
    }

    // Centre of mass x, centre height, lowest and highest point and the
    // contact and lift bits of the step's end (shaders/creature.cu:1000-1023).
    struct Tally {
        bool failed;
        float center_y, com_x, low, high;
        unsigned touching, lifted;
    };
    __device__ __forceinline__ static void tally_node(const Body& b, Tally& y, unsigned i, const float4& nr) {
        const float2 q = b.t.pos(i);
        y.failed = y.failed || !(fabsf(q.x) <= 1e6f && fabsf(q.y) <= 1e6f);
        y.center_y += q.y;
        y.com_x += nr.x * q.x;
        y.low = fminf(y.low, q.y - nr.z);
        y.high = fmaxf(y.high, q.y + nr.z);
        if (b.w.has(CE_FLAG_GROUND)) {
            const float2 g = ground_tally(b.w, q.x, b.r.amp, b.r.qphase, b.p);
            const float floor_y = __fmaf_rn(nr.z, sqrtf(__fmaf_rn(g.y, g.y, 1.0f)), g.x);
            if (q.y <= floor_y + kContactSlack) {
                y.touching |= 1u << i;
            }
            if (q.y > floor_y + kLiftClearance) {
                y.lifted |= 1u << i;
            }
        }
    }
    __device__ __forceinline__ static Tally tally(const Body& b) {
        Tally y{false, 0.0f, 0.0f, 1e20f, -1e20f, 0u, 0u};
        for (unsigned i = 0u; i < b.r.nodes; i++) {
            tally_node(b, y, i, b.L.get(b.S.node + i));
        }
        return y;
    }

    // The trial's metrics row and niche cell, from its 19 result words
    // (niche.cuh: the host's to_metrics and cell index to the bit).
    __device__ __forceinline__ static void niche_epilogue(const KernelArgs& a, const LaneRegs& r, const float* m) {
        const ce_result res{m[0],  m[1],  m[2],  m[3],  m[4],  m[5],  m[6],  m[7],  m[8], m[9],
                            m[10], m[11], m[12], m[13], m[14], m[15], m[16], m[17], m[18]};
        const ce_metrics mt = to_metrics(res, r.nodes, a.niche);
        if (a.metrics) {
            a.metrics[r.cidx] = mt;
        }
        a.cells[r.cidx] = cell_of(mt, r.nodes, a.shapes[r.cidx], a.niche);
    }

    // One step of the creature on this lane (shaders/creature.cu:956-1248).
    // Returns whether the lane still has a creature.
    __device__ __forceinline__ static bool step(const Body& b, const KernelArgs& a) {
        LaneRegs& r = b.r;
        const ce_params& p = b.p;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const unsigned step = r.step;
        const unsigned flags = r.flags;
        const unsigned rung1 = (unsigned)(C::rate) - 1u, rung2 = (unsigned)(2.5f * C::rate) - 1u;
        const unsigned rung3 = (unsigned)(5.0f * C::rate) - 1u, rung4 = (unsigned)(10.0f * C::rate) - 1u;
        const unsigned half_s = (unsigned)(0.5f * C::rate);
        const float t_now = (float)step * C::dt;
        if (RECORD) {
            for (unsigned i = 0u; i < r.nodes; i++) {
                L.put(S.rec_force + i, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
            }
        }
        if (CKPT && (step & 15u) == 0u) {
            save_checkpoint(b, a, step >> 4u);
        }
        b.muscle_demands(t_now);
        for (unsigned s = 0u; s < 16u; s++) {
            b.substep();
        }
        if (RECORD) {
            for (unsigned i = 0u; i < r.nodes; i++) {
                float4 fl = L.get(S.rec_force + i);
                fl.x *= 1.0f / 16u;
                fl.y *= 1.0f / 16u;
                L.put(S.rec_force + i, fl);
            }
        }
        const Tally y = tally(b);
        const bool broken = b.broken_joints() != 0ull;
        const bool failed = y.failed;
        float center_y = y.center_y, com_x = y.com_x;
        const float low = y.low, high = y.high;
        const unsigned touching = y.touching, lifted = y.lifted;
        center_y /= (float)r.nodes;
        com_x *= r.inv_mass;
        // The result and tallies, from the lane lines.
        // Words 0-18 are the result, 19-31 the tallies.
        float lw[32];
#pragma unroll
        for (unsigned q = 0u; q < 8u; q++) {
            const float4 v = L.get_cold(S.lane + q);
            lw[4u * q] = v.x;
            lw[4u * q + 1u] = v.y;
            lw[4u * q + 2u] = v.z;
            lw[4u * q + 3u] = v.w;
        }
        float* const m = lw;
        auto LW = [&](unsigned q) -> float& { return lw[q]; };
        unsigned contact_bits = __float_as_uint(LW(kWContact));
        unsigned lift_bits = __float_as_uint(LW(kWLift));
        unsigned ground_bits = __float_as_uint(LW(kWGround));
        float head_shake = LW(kWHeadShake);
        float2 head_at = make_float2(LW(kWHeadAt), LW(kWHeadAt + 1u));
        float2 head_vel = make_float2(LW(kWHeadVel), LW(kWHeadVel + 1u));
        unsigned rung_x = __float_as_uint(LW(kWRungX));
        unsigned rung_speed = __float_as_uint(LW(kWRungSpeed));
        unsigned rung_early = __float_as_uint(LW(kWRungEarly));
        unsigned rung_late = __float_as_uint(LW(kWRungLate));
        unsigned rung_bits = __float_as_uint(LW(kWRungBits));
        float& fitness = m[0];
        float& ground_contact = m[1];
        float& vertical_oscillation = m[2];
        float& gait_frequency = m[3];
        float& previous_center_y = m[4];
        float& vertical_extremum = m[5];
        float& vertical_trend = m[6];
        float& gait_turns = m[7];
        float& height_sum = m[8];
        float& contact_lo = m[9];
        float& contact_hi = m[10];
        float& lift_lo = m[11];
        float& lift_hi = m[12];
        float& ground_lo = m[13];
        float& ground_hi = m[14];
        float& fall_time = m[15];
        float& head_shake_r = m[16];
        float& screen_x = m[17];
        float& screened = m[18];

        contact_bits |= touching;
        lift_bits |= contact_bits & lifted;
        const unsigned down = touching & ~ground_bits;
        ground_bits = touching;
        if (down != 0u && step > 0u) {
            const float next = t_now + C::dt;
            for (unsigned k = 0u; k < r.muscles; k++) {
                const unsigned m0 = S.muscle + 5u * k;
                const unsigned sensor = __float_as_uint(L.word_cold(m0 + kMState, 3));
                if (sensor != kNone && ((down >> sensor) & 1u)) {
                    const float4 r0 = L.get_cold(m0 + kRhythm0), r1 = L.get_cold(m0 + kRhythm1);
                    L.set_cold(m0 + kMState, 2, fracf(r1.w - (next * r0.y + r0.z)));
                }
            }
        }
        if ((step + 1u) % C::head_sample == 0u) {
            const float2 h = b.t.pos(0u);
            const float2 v = make_float2((h.x - head_at.x) * 60.0f, (h.y - head_at.y) * 60.0f);
            const float ax = (v.x - head_vel.x) * 60.0f, ay = (v.y - head_vel.y) * 60.0f;
            if (t_now >= kHeadShakeWindow) {
                const float accel = sqrtf(ax * ax + ay * ay);
                head_shake += (accel - head_shake) * fminf(1.0f / (kHeadShakeWindow * 60.0f), 1.0f);
            }
            head_at = h;
            head_vel = v;
        }
        bool done = false;
        if (!RECORD || r.scoring) {
            contact_lo = __uint_as_float(contact_bits);
            lift_lo = __uint_as_float(lift_bits);
            ground_lo = __uint_as_float(ground_bits);
            head_shake_r = head_shake;
            const bool fell = b.t.pos(0u).y < b.t.pos(1u).y || broken || head_shake > kHeadShakeLimit || failed;
            bool ended = false;
            if (fell) {
                fall_time = t_now + C::dt;
                fitness = failed ? -1e20f : com_x;
                if (step <= p.screen_step) {
                    screen_x = fitness;
                }
                ended = true;
            }
            ground_contact += (float)__popc(touching);
            height_sum += high - low;
            vertical_oscillation = fminf(vertical_oscillation, center_y);
            gait_frequency = fmaxf(gait_frequency, center_y);
            if (step == 0u) {
                previous_center_y = center_y;
                vertical_extremum = center_y;
                vertical_trend = 0.0f;
                gait_turns = 0.0f;
            } else if (step % C::sample == 0u) {
                const float delta = center_y - previous_center_y;
                if (vertical_trend == 0.0f) {
                    if (fabsf(delta) > 0.0005f) {
                        vertical_trend = delta > 0.0f ? 1.0f : -1.0f;
                        vertical_extremum = center_y;
                    }
                } else if (vertical_trend > 0.0f) {
                    if (center_y > vertical_extremum) {
                        vertical_extremum = center_y;
                    } else if (vertical_extremum - center_y > 0.005f) {
                        gait_turns += 1.0f;
                        vertical_trend = -1.0f;
                        vertical_extremum = center_y;
                    }
                } else {
                    if (center_y < vertical_extremum) {
                        vertical_extremum = center_y;
                    } else if (center_y - vertical_extremum > 0.005f) {
                        gait_turns += 1.0f;
                        vertical_trend = 1.0f;
                        vertical_extremum = center_y;
                    }
                }
                previous_center_y = center_y;
            }
            if (step + half_s == rung1 || step + half_s == rung2) {
                rung_x = __float_as_uint(com_x);
            }
            if (step == rung1 || step == rung2) {
                const bool second = step == rung2;
                const unsigned sh = second ? 16u : 0u;
                const unsigned keep = second ? 0x0000ffffu : 0xffff0000u;
                const float speed = (com_x - __uint_as_float(rung_x)) * (C::rate / (float)half_s);
                const float touched = (float)__popc(contact_bits) / (float)r.nodes;
                float en_mean = 0.0f;
                for (unsigned k = 0u; k < r.muscles; k++) {
                    en_mean += b.t.muscle(k).x;
                }
                en_mean /= (float)max(r.muscles, 1u);
                contact_hi = __uint_as_float((__float_as_uint(contact_hi) & keep) | (f2h(com_x) << sh));
                ground_hi = __uint_as_float((__float_as_uint(ground_hi) & keep) | (f2h(head_shake) << sh));
                rung_speed = (rung_speed & keep) | (f2h(speed) << sh);
                const unsigned pair = f2h(touched) | (f2h(en_mean) << 16u);
                if (second) {
                    rung_late = pair;
                } else {
                    rung_early = pair;
                }
                const unsigned rr = second ? 1u : 0u;
                const float gait_now = gait_turns * (0.5f / (t_now + C::dt));
                const unsigned band = min((unsigned)(gait_now * (8.0f / 6.0f)), 7u);
                rung_bits |= band << (8u + 3u * rr);
                if (!ended && (flags & (second ? 0xbu : 0x7u)) == 0u) {
                    const ce_rung& rp = second ? p.r2 : p.r1;
                    const float fv[6] = {h2f(f2h(com_x)),      h2f(f2h(speed)),   h2f(f2h(touched)),
                                         h2f(f2h(head_shake)), h2f(f2h(en_mean)), r.period_f};
                    float score = 0.0f;
                    bool finite = true;
                    for (int i = 0; i < 6; i++) {
                        score = fmaf(rp.w[i], fv[i], score);
                        finite = finite && isfinite(fv[i]);
                    }
                    if (finite && score < rp.bias && ((rp.off >> band) & 1u) == 0u) {
                        screened = t_now + C::dt;
                        screen_x = com_x;
                        fitness = com_x;
                        rung_bits |= (rr + 1u) << 6u;
                        ended = true;
                    }
                }
            }
            if (step == rung3 || step == rung4) {
                const bool second = step == rung4;
                const unsigned keep = second ? 0x0000ffffu : 0xffff0000u;
                lift_hi = __uint_as_float((__float_as_uint(lift_hi) & keep) | (f2h(com_x) << (second ? 16u : 0u)));
            }
            if (step == p.screen_step && !ended) {
                screen_x = com_x;
                const float bar = (flags & 32u) != 0u   ? p.screen_bar_reshaped
                                  : (flags & 16u) != 0u ? p.screen_bar_young
                                                        : p.screen_bar;
                if (com_x < bar && (flags & 1u) == 0u) {
                    screened = t_now + C::dt;
                    fitness = com_x;
                    ended = true;
                }
            }
            bool last = false;
            if (ended) {
                vertical_oscillation = fmaxf(gait_frequency - vertical_oscillation, 0.0f);
                gait_frequency = gait_turns * 0.5f / (t_now + C::dt);
            } else if (step + 1u >= p.steps) {
                fitness = com_x;
                vertical_oscillation = fmaxf(gait_frequency - vertical_oscillation, 0.0f);
                gait_frequency = gait_turns * 0.5f / fmaxf((float)(step + 1u) * C::dt, C::dt);
                last = true;
            }
            if (ended || last) {
                const unsigned fin = f2h(fitness);
                unsigned d = __float_as_uint(contact_hi);
                if (step < rung1) {
                    d = (d & 0xffff0000u) | fin;
                }
                if (step < rung2) {
                    d = (d & 0x0000ffffu) | (fin << 16u);
                }
                contact_hi = __uint_as_float(d);
                d = __float_as_uint(lift_hi);
                if (step < rung3) {
                    d = (d & 0xffff0000u) | fin;
                }
                if (step < rung4) {
                    d = (d & 0x0000ffffu) | (fin << 16u);
                }
                lift_hi = __uint_as_float(d);
                const unsigned code = (fell ? 16u : 0u) | (failed ? 32u : 0u) | (screened > 0.0f ? 3u : 0u) |
                                      (rung_bits & 0x3fc0u) | ((flags & 1u) << 14u);
                previous_center_y = __uint_as_float(rung_speed);
                vertical_extremum = __uint_as_float(rung_early);
                vertical_trend = __uint_as_float(rung_late);
                gait_turns = ground_hi;
                ground_hi = __uint_as_float(code | (min(step + 1u, 65535u) << 16u));
                if (RECORD) {
                    for (unsigned q = 0u; q < 19u; q++) {
                        L.word(S.rec_kept + q / 4u, q % 4u) = m[q];
                    }
                    r.scoring = false;
                    r.limp = true;
                } else {
                    float* out = reinterpret_cast<float*>(a.results + r.cidx);
                    for (unsigned q = 0u; q < 19u; q++) {
                        __stcs(out + q, m[q]);
                    }
                    if (!CKPT && a.cells) {
                        niche_epilogue(a, r, m);
                    }
                    if (CKPT) {
                        a.ends[r.cidx] = step + 1u;
                    }
                    done = true;
                }
            }
        }
        if (done) {
            return false;
        }
        LW(kWContact) = __uint_as_float(contact_bits);
        LW(kWLift) = __uint_as_float(lift_bits);
        LW(kWGround) = __uint_as_float(ground_bits);
        LW(kWHeadShake) = head_shake;
        LW(kWHeadAt) = head_at.x;
        LW(kWHeadAt + 1u) = head_at.y;
        LW(kWHeadVel) = head_vel.x;
        LW(kWHeadVel + 1u) = head_vel.y;
        LW(kWRungX) = __uint_as_float(rung_x);
        LW(kWRungSpeed) = __uint_as_float(rung_speed);
        LW(kWRungEarly) = __uint_as_float(rung_early);
        LW(kWRungLate) = __uint_as_float(rung_late);
        LW(kWRungBits) = __uint_as_float(rung_bits);
#pragma unroll
        for (unsigned q = 0u; q < 8u; q++) {
            L.put_cold(S.lane + q, make_float4(lw[4u * q], lw[4u * q + 1u], lw[4u * q + 2u], lw[4u * q + 3u]));
        }
        if (RECORD) {
            record_frame(b, a, C::settle + step + 1u);
            if (step + 1u >= p.steps) {
                float* out = reinterpret_cast<float*>(a.results + r.cidx);
                for (unsigned q = 0u; q < 19u; q++) {
                    out[q] = L.word(S.rec_kept + q / 4u, q % 4u);
                }
                return false;
            }
        }
        r.step = step + 1u;
        return true;
    }
};

// The work claiming of a persistent warp: a run (window) of positions of
// the launch's order claimed at a time from the warp's queue, handed to the
// lanes that need a creature. The warps split between the queues by
// estimated work, and a warp whose queue runs dry moves on to the next one.
struct Claim {
    const KernelArgs& a;
    unsigned lane, warps_total, queues, queue = 0u, win_cur = 0u, win_end = 0u;
    unsigned long long total_work = 1ull;
    bool drained = false;

    __device__ __forceinline__ Claim(const KernelArgs& args, unsigned lane_, unsigned warp, unsigned warps)
        : a(args), lane(lane_), warps_total(warps), queues(args.queues > 0u ? args.queues : 1u) {
        if (a.queues > 1u) {
            total_work = max(a.work[a.queues] - a.work[0], 1ull);
            const unsigned long long target =
                a.work[0] + total_work * (2ull * warp + 1ull) / (2ull * warps_total);
            while (queue + 1u < a.queues && a.work[queue + 1u] <= target) {
                queue++;
            }
        }
    }

    // The next position of the order for each lane whose `live` is false
    // (kNone for a lane that gets none: all queues are exhausted).
    __device__ __forceinline__ unsigned next(bool live) {
        const unsigned below = (1u << lane) - 1u;
        unsigned need = ~__ballot_sync(kFull, live);
        unsigned mine = kNone;
        while (need != 0u) {
            if (win_cur >= win_end) {
                if (drained) {
                    break;
                }
                unsigned c0 = kNone, c1 = 0u, got_queue = queue;
                if (lane == 0u) {
                    for (unsigned t = 0u; t < queues; t++) {
                        const unsigned q = queue + t < queues ? queue + t : queue + t - queues;
                        const unsigned lo = a.queues > 0u ? a.bounds[q] : 0u;
                        const unsigned n = (a.queues > 0u ? a.bounds[q + 1u] : a.count) - lo;
                        const unsigned seen = *reinterpret_cast<volatile unsigned*>(a.counter + q);
                        if (seen >= n) {
                            continue;
                        }
                        unsigned share = warps_total;
                        if (a.queues > 1u) {
                            share = (unsigned)max(1ull, warps_total * (a.work[q + 1u] - a.work[q]) / total_work);
                        }
                        const unsigned want = min(max((n - seen) / (a.chunk_k * share), 1u), kChunk);
                        const unsigned got = atomicAdd(a.counter + q, want);
                        if (got >= n) {
                            continue;
                        }
                        c0 = lo + got;
                        c1 = lo + min(got + want, n);
                        got_queue = q;
                        break;
                    }
                }
                c0 = __shfl_sync(kFull, c0, 0);
                c1 = __shfl_sync(kFull, c1, 0);
                queue = __shfl_sync(kFull, got_queue, 0);
                if (c0 == kNone) {
                    drained = true;
                    break;
                }
                win_cur = c0;
                win_end = c1;
            }
            const unsigned rank = (unsigned)__popc(need & below);
            const bool take = ((need >> lane) & 1u) != 0u && rank < win_end - win_cur;
            if (take) {
                mine = win_cur + rank;
            }
            const unsigned taken = __ballot_sync(kFull, take);
            need &= ~taken;
            win_cur += (unsigned)__popc(taken);
        }
        return mine;
    }
};

template <class W, bool RECORD, int RATE, bool CKPT = false>
__global__ void __launch_bounds__(kBlock, kMinBlocks) advance_kernel(const KernelArgs a, const ce_params p,
                                                                      const W w) {
    extern __shared__ float4 smem[];
    using T = Trial<W, RECORD, RATE, CKPT>;
    const unsigned threads = blockDim.x;
    // Tables of rows x threads entries: positions, velocities, forces, then
    // the muscles' (energy, demand) pairs.
    float2* const tables = reinterpret_cast<float2*>(smem) + threadIdx.x;
    const size_t table = (size_t)a.rows * threads;
    const NodeTables tab{tables, tables + table, tables + 2u * table, tables + 3u * table};
    const SlotLayout S = SlotLayout::make(a.rows, a.mm, RECORD);
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = (blockIdx.x * threads + threadIdx.x) >> 5u;
    const unsigned warps_total = gridDim.x * (threads >> 5u);
    const Lines L = Lines::make(a.scratch + (size_t)warp * S.lines * 32u, lane);
    LaneRegs r;
    const typename T::Body b{w, p, tab, L, S, r};
    bool live = false;
    Claim claim(a, lane, warp, warps_total);
    for (;;) {
        const unsigned mine = claim.next(live);
        if (mine != kNone) {
            const unsigned cidx = a.order ? __ldg(a.order + mine) : p.base + mine;
            T::begin(b, a, cidx, mine);
            live = true;
        }
        if (__ballot_sync(kFull, live) == 0u) {
            break;
        }
        if (live) {
            live = T::step(b, a);
        }
    }
}

}  // namespace cek
