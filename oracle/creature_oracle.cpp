// Test infrastructure: the CPU oracle of the creature path (see
// creature_oracle.hpp). Each function cites the lines of the reference
// kernel, shaders/creature.cu, whose computation it restates.
#include "creature_oracle.hpp"

#include <omp.h>

#include <algorithm>
#include <chrono>

namespace oracle {

thread_local OpCount g_ops;

namespace {

inline float fbits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t ubits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Round to the nearest half and back (cvt.rn.f16.f32, creature.cu:138-147).
uint32_t f2h(float v) {
    const uint32_t bits = ubits(v);
    const uint32_t sign = (bits >> 16) & 0x8000u;
    const int32_t exponent = (int32_t)((bits >> 23) & 0xffu);
    const uint32_t mantissa = bits & 0x7fffffu;
    if (exponent == 0xff) return sign | 0x7c00u | (mantissa ? 0x200u : 0u);
    const int32_t e = exponent - 127 + 15;
    if (e >= 31) return sign | 0x7c00u;
    if (e <= 0) {
        if (e < -10) return sign;
        const uint32_t m = mantissa | 0x800000u;
        const uint32_t shift = (uint32_t)(14 - e);
        const uint32_t half = 1u << (shift - 1);
        const uint32_t rest = m & ((1u << shift) - 1u);
        uint32_t o = m >> shift;
        if (rest > half || (rest == half && (o & 1u))) o += 1;
        return sign | o;
    }
    const uint32_t rest = mantissa & 0x1fffu;
    uint32_t o = ((uint32_t)e << 10) | (mantissa >> 13);
    if (rest > 0x1000u || (rest == 0x1000u && (o & 1u))) o += 1;
    return sign | o;
}
float h2f(uint32_t h) {
    const uint32_t sign = (h >> 15) << 31, exponent = (h >> 10) & 0x1fu, mantissa = h & 0x3ffu;
    uint32_t bits;
    if (exponent == 0 && mantissa == 0) {
        bits = sign;
    } else if (exponent == 0) {
        const uint32_t shift = (uint32_t)__builtin_clz(mantissa) - 21;
        bits = sign | ((113 - shift) << 23) | (((mantissa << shift) & 0x3ffu) << 13);
    } else if (exponent == 31) {
        bits = sign | 0x7f800000u | (mantissa ? (0x400000u | (mantissa << 13)) : 0u);
    } else {
        bits = sign | ((exponent + 112) << 23) | (mantissa << 13);
    }
    return fbits(bits);
}

template <class T>
struct Sim {
    // Constants (the #define block of src/kernel.rs:268-317).
    const T PI = T(3.14159265359f), TAU = T(6.28318530718f);
    const uint32_t NONE = 0xffffffffu;

    const Params& p;
    uint32_t flags;
    T rate, dt, h, inv_h;
    uint32_t settle, sample, head_sample;

    struct Node {
        T m, im, r, mu;
    };
    struct Bone {
        uint32_t i0;
        T len, w0, w1, kair, limit, s0, s1;
    };
    struct Joint {
        bool has;
        uint32_t hub, ptip, ppivot, far;
        bool at_head;
        T lo, hi, mid, wt, wf, wh;
    };
    T fit_t = T(0.0f);  // the fitness as a T (its derivative parts for a dual T)
    const double* seed_mass = nullptr;  // dual T: node-mass directions set in begin
    const double* seed_start = nullptr; // dual T: start-position directions (x, y a node) set in begin
    // Checkpoints of another run of the same trial (positions, velocities,
    // energy stores every `resync_every` substeps, rows x 4 + mm floats
    // each): when set, the state's values are reset to them at each
    // checkpoint, its derivative parts kept, so the run follows that
    // trajectory.
    const float* resync = nullptr;
    uint32_t resync_rows = 0, resync_mm = 0, resync_count = 0, resync_every = 256;
    void resync_state(const float* c) {
        for (uint32_t i = 0; i < N; i++) {
            set_value(px[i], c[2 * i]);
            set_value(py[i], c[2 * i + 1]);
            set_value(vx[i], c[2 * resync_rows + 2 * i]);
            set_value(vy[i], c[2 * resync_rows + 2 * i + 1]);
        }
        for (uint32_t k = 0; k < M; k++) set_value(mus[k].energy, c[4 * resync_rows + k]);
    }
    struct Muscle {
        uint32_t a0, a1, b0, b1, sensor;
        T aa, ab, hill, cap, icap, tk, slack, amp, iper, phase, duty, iduty, icomp, stiff, reset;
        T energy, demand, offset;
    };
    uint32_t N = 0, M = 0, feet = 0, cflags = 0;
    T inv_mass, amp, qphase, period_f;
    std::vector<Node> node;
    std::vector<Bone> bone;
    std::vector<Joint> joint;
    std::vector<Muscle> mus;
    std::vector<T> px, py, vx, vy, fx, fy;

    Sim(const Params& params, uint32_t f, int r) : p(params), flags(f) {
        rate = T((float)r);
        dt = T(1.0f) / rate;
        h = T(1.0f) / (rate * T(16.0f));
        inv_h = rate * T(16.0f);
        settle = (200u * (uint32_t)r + 119u) / 120u;
        sample = std::max((uint32_t)r / 30u, 1u);
        head_sample = (uint32_t)((float)r / 60.0f + 0.5f);
    }
    bool has(uint32_t bit) const { return (flags & bit) != 0u; }
    T clamp(T x, T lo, T hi) const { return min_(max_(x, lo), hi); }
    T frac(T x) const { return x - floor_(x); }
    T wrap(T a) const { return a - TAU * floor_((a + PI) * (T(1.0f) / TAU)); }

    // creature.cu:153-159
    T rhythm(T t, const Muscle& u, T offset) const {
        const T ph = frac(t * u.iper + u.phase + offset);
        if (ph < u.duty) return T(0.5f) - T(0.5f) * cos_(PI * ph * u.iduty);
        return T(0.5f) + T(0.5f) * cos_(PI * (ph - u.duty) * u.icomp);
    }

    // creature.cu:166-226
    void ground(T x, T& height, T& slope) const {
        height = T(0.0f);
        slope = T(0.0f);
        if (has(TERRAIN)) {
            const T t0 = x * (T(1.0f) / T(1.1f)) + qphase;
            const T u0 = frac(t0);
            const T w0 = u0 * (T(1.0f) - u0);
            const T t1 = x * (T(1.0f) / T(0.43f)) + T(0.3f) + qphase;
            const T u1 = frac(t1);
            const T w1 = u1 * (T(1.0f) - u1);
            height = amp * (T(0.65f) * T(16.0f) * w0 * w0 + T(0.35f) * T(16.0f) * w1 * w1);
            slope = amp * (T(0.65f) * T(32.0f) * w0 * (T(1.0f) - T(2.0f) * u0) * (T(1.0f) / T(1.1f)) +
                           T(0.35f) * T(32.0f) * w1 * (T(1.0f) - T(2.0f) * u1) * (T(1.0f) / T(0.43f)));
        }
        if (has(SLOPE)) {
            height += T(p.slope) * x;
            slope += T(p.slope);
        }
        if (has(GAPS)) {
            const T spacing = T(2.0f) + T(4.0f) * T(p.gaps);
            const T center = spacing * T(0.5f);
            const T r = x - floor_(x / spacing) * spacing;
            const T distance = abs_(r - center);
            const T half_w = T(0.5f) * T(p.gaps);
            const T run = max_(min_(T(0.15f), half_w), T(1e-6f));
            T factor = clamp((half_w - distance) / run, T(0.0f), T(1.0f));
            if (distance <= half_w - run) factor = T(1.0f);
            else if (distance >= half_w) factor = T(0.0f);
            height -= T(2.0f) * factor;
            if (distance > half_w - run && distance < half_w) {
                slope -= T(2.0f) * ((r < center ? T(1.0f) : T(-1.0f)) / run);
            }
        }
        if (has(HURDLES)) {
            const T spacing = T(3.0f);
            const T center = spacing * T(0.5f);
            const T r = x - floor_(x / spacing) * spacing;
            const T distance = abs_(r - center);
            const T half_w = T(0.5f) * T(1.2f);
            const T run = T(0.2f);
            T factor = clamp((half_w + run - distance) / run, T(0.0f), T(1.0f));
            if (distance <= half_w) factor = T(1.0f);
            else if (distance >= half_w + run) factor = T(0.0f);
            height += T(p.hurdles) * factor;
            if (distance > half_w && distance < half_w + run) {
                slope += T(p.hurdles) * ((r < center ? T(1.0f) : T(-1.0f)) / run);
            }
        }
    }

    // creature.cu:230-235
    T ice_at(T x) const {
        const T w = frac(x * T(0.16666667f));
        const T t = abs_(w - T(0.5f)) * T(2.0f);
        const T s = clamp((T(0.7f) - t) * T(2.5f), T(0.0f), T(1.0f));
        return s * s * (T(3.0f) - T(2.0f) * s);
    }

    // creature.cu:845-929: constants and the start pose from the records.
    void begin(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t cidx) {
        const uint32_t* h0 = heads + 8 * cidx;
        const uint32_t* h1 = h0 + 4;
        N = h0[0] & 255u;
        M = h0[1];
        const uint32_t* rec = records + h0[3];
        const float* mrec = muscles + h1[0];
        inv_mass = T(fbits(h1[2]));
        cflags = h1[3] >> 16;
        period_f = T(h2f(h1[3] & 0xffffu));
        if (has(QUAKE)) {
            qphase = T((float)(h0[2] & 0xffffu) * (1.0f / 65536.0f));
            amp = T(p.terrain) + T(p.quake) * (T(0.6f) + T((float)((h0[2] >> 16) & 0xffffu)) * T(0.8f / 65536.0f));
        } else {
            qphase = T(0.0f);
            amp = T(p.terrain);
        }
        node.resize(N);
        px.assign(N, T(0.0f));
        py.assign(N, T(0.0f));
        vx.assign(N, T(0.0f));
        vy.assign(N, T(0.0f));
        fx.assign(N, T(0.0f));
        fy.assign(N, T(0.0f));
        feet = 0;
        for (uint32_t i = 0; i < N; i++) {
            const uint32_t* r = rec + i * 6;
            T m = T(fbits(r[0]));
            if (seed_mass) set_deriv(m, seed_mass[i]);
            node[i] = Node{m, T(1.0f) / m, T(fbits(r[1])), T(fbits(r[2]))};
            px[i] = T(fbits(r[3]));
            py[i] = T(fbits(r[4]));
            if (seed_start) {
                set_deriv(px[i], seed_start[2 * i]);
                set_deriv(py[i], seed_start[2 * i + 1]);
            }
            feet |= (r[5] & 1u) << i;
        }
        if (seed_mass) {
            // inv_mass = 1 / sum of node masses.
            double dsum = 0.0;
            for (uint32_t i = 0; i < N; i++) dsum += seed_mass[i];
            set_deriv(inv_mass, -dsum * (double)fbits(h1[2]) * (double)fbits(h1[2]));
        }
        const uint32_t* bone_rec = rec + N * 6;
        const uint32_t B = N - 1;
        bone.resize(B);
        joint.assign(B, Joint{});
        for (uint32_t j = 0; j < B; j++) {
            const uint32_t* r = bone_rec + j * 6;
            const uint32_t i0 = r[0], i1 = j + 1;
            const T length = T(fbits(r[1]));
            const T width = node[i0].r + node[i1].r;
            const T bone_mass = node[i0].m + node[i1].m;
            bone[j] = Bone{i0, length, node[i0].im, node[i1].im, T(0.6f) * length * width,
                           T(0.5f) * bone_mass * inv_h, T(0.5f) * h * node[i0].im, T(0.5f) * h * node[i1].im};
            const uint32_t pj = r[2];
            if (j > 0 && pj != NONE) {
                Joint& k = joint[j];
                k.has = true;
                k.hub = i0;
                k.ppivot = bone_rec[pj * 6];
                k.ptip = pj + 1;
                k.at_head = k.hub == k.ppivot;
                k.far = k.at_head ? pj + 1 : k.ppivot;
                k.lo = T(fbits(r[3]));
                k.hi = T(fbits(r[4]));
                k.mid = T(0.5f) * (k.lo + k.hi);
                k.wt = node[i1].im;
                k.wf = node[k.far].im;
                k.wh = node[k.hub].im;
            }
        }
        mus.resize(M);
        for (uint32_t k = 0; k < M; k++) {
            const float* q = mrec + k * 20;
            const uint32_t nodes = ubits(q[0]);
            Muscle& u = mus[k];
            u.a0 = nodes & 255u;
            u.a1 = (nodes >> 8) & 255u;
            u.b0 = (nodes >> 16) & 255u;
            u.b1 = nodes >> 24;
            u.aa = T(q[1]);
            u.ab = T(q[2]);
            u.hill = T(q[3]);
            u.cap = T(q[4]);
            u.icap = T(q[5]);
            u.tk = T(q[6]);
            u.slack = T(q[7]);
            u.amp = T(q[8]);
            u.iper = T(q[9]);
            u.phase = T(q[10]);
            u.duty = T(q[11]);
            u.iduty = T(q[12]);
            u.icomp = T(q[13]);
            u.stiff = T(q[14]);
            u.reset = T(q[15]);
            u.sensor = ubits(q[16]);
            u.energy = T(1.0f);
            u.demand = T(0.0f);
            u.offset = T(0.0f);
        }
    }

    // creature.cu:322-356: the joint's angle and its gradients.
    void joint_eval(const Joint& k, uint32_t tip, bool with_angle, T& angle, T g[6]) const {
        const T ux = px[k.ptip] - px[k.ppivot], uy = py[k.ptip] - py[k.ppivot];
        const T vx_ = px[tip] - px[k.hub], vy_ = py[tip] - py[k.hub];
        const T uu = max_(ux * ux + uy * uy, T(1e-12f)), vv = max_(vx_ * vx_ + vy_ * vy_, T(1e-12f));
        angle = T(0.0f);
        if (with_angle) {
            const T turn = atan2_(ux * vy_ - uy * vx_, ux * vx_ + uy * vy_);
            angle = k.mid + wrap(turn - k.mid);
        }
        g[0] = -vy_ / vv;
        g[1] = vx_ / vv;
        T gux = -uy / uu, guy = ux / uu;
        if (k.at_head) {
            gux = -gux;
            guy = -guy;
        }
        g[2] = gux;
        g[3] = guy;
        g[4] = -(g[0] + g[2]);
        g[5] = -(g[1] + g[3]);
    }
    T joint_weight(const Joint& k, const T g[6]) const {
        return k.wt * (g[0] * g[0] + g[1] * g[1]) + k.wf * (g[2] * g[2] + g[3] * g[3]) +
               k.wh * (g[4] * g[4] + g[5] * g[5]);
    }
    void joint_push(const Joint& k, uint32_t tip, const T g[6], T lambda, std::vector<T>& X, std::vector<T>& Y) {
        X[tip] += k.wt * lambda * g[0];
        Y[tip] += k.wt * lambda * g[1];
        X[k.far] += k.wf * lambda * g[2];
        Y[k.far] += k.wf * lambda * g[3];
        X[k.hub] += k.wh * lambda * g[4];
        Y[k.hub] += k.wh * lambda * g[5];
    }

    // creature.cu:442-451
    void muscle_demands(T t, bool limp) {
        for (Muscle& u : mus) {
            const T before = rhythm(t, u, u.offset);
            const T after = rhythm(t + dt, u, u.offset);
            const T shortening = u.amp * (after - before) * rate;
            u.demand = limp ? T(0.0f) : max_(shortening * u.stiff * T(0.25f), T(0.0f));
        }
    }

    // creature.cu:455-508
    void muscle_forces() {
        for (uint32_t i = 0; i < N; i++) {
            fx[i] = T(0.0f);
            fy[i] = T(0.0f);
        }
        for (Muscle& u : mus) {
            const T ax = px[u.a0] + (px[u.a1] - px[u.a0]) * u.aa;
            const T ay = py[u.a0] + (py[u.a1] - py[u.a0]) * u.aa;
            const T avx = vx[u.a0] + (vx[u.a1] - vx[u.a0]) * u.aa;
            const T avy = vy[u.a0] + (vy[u.a1] - vy[u.a0]) * u.aa;
            const T bx = px[u.b0] + (px[u.b1] - px[u.b0]) * u.ab;
            const T by = py[u.b0] + (py[u.b1] - py[u.b0]) * u.ab;
            const T bvx = vx[u.b0] + (vx[u.b1] - vx[u.b0]) * u.ab;
            const T bvy = vy[u.b0] + (vy[u.b1] - vy[u.b0]) * u.ab;
            const T dx = bx - ax, dy = by - ay;
            const T len = max_(sqrt_(dx * dx + dy * dy), T(1e-6f));
            const T ex = dx / len, ey = dy / len;
            const T lengthening = (bvx - avx) * ex + (bvy - avy) * ey;
            T drive = u.demand * u.energy;
            if (u.hill > T(0.0f)) drive *= clamp(T(1.0f) + lengthening * u.hill, T(0.0f), T(1.0f));
            const T active = clamp(drive + lengthening * T(0.15f), -u.cap, u.cap);
            const T work = min_(drive, u.cap) * max_(-lengthening, T(0.0f)) * h;
            u.energy = clamp(u.energy - work * u.icap * T(p.inv_muscle_energy) +
                                 T(0.5f) * T(p.muscle_recovery) * h * (T(1.0f) - u.energy),
                             T(0.0f), T(1.0f));
            const T tendon = u.tk * max_(len - u.slack, T(0.0f));
            const T pull = active + tendon;
            const T fxm = ex * pull, fym = ey * pull;
            fx[u.a0] += fxm * (T(1.0f) - u.aa);
            fy[u.a0] += fym * (T(1.0f) - u.aa);
            fx[u.a1] += fxm * u.aa;
            fy[u.a1] += fym * u.aa;
            fx[u.b0] -= fxm * (T(1.0f) - u.ab);
            fy[u.b0] -= fym * (T(1.0f) - u.ab);
            fx[u.b1] -= fxm * u.ab;
            fy[u.b1] -= fym * u.ab;
        }
    }

    // creature.cu:511-546
    void node_force(uint32_t i, T& ffx, T& ffy) const {
        const Node& nr = node[i];
        const T m = nr.m;
        ffx = T(0.0f);
        ffy = -T(p.gravity) * m;
        if (has(WIND)) ffx += T(p.wind) * m;
        T dry = T(0.0f);
        if (has(MUD) || has(BRAMBLES)) {
            T gh, gs;
            ground(px[i], gh, gs);
            dry = (py[i] - gh) / sqrt_(T(1.0f) + gs * gs) - nr.r;
        }
        if (has(MUD)) ffx -= m * T(2.0f) * (clamp(-dry, T(0.0f), T(p.mud)) * (T(1.0f) / T(0.1f))) * vx[i];
        if (has(BRAMBLES)) {
            if (((feet >> i) & 1u) == 0u && dry < T(0.01f)) ffx -= m * T(p.brambles) * vx[i];
        }
        if (has(WATER)) {
            const T wet = clamp((T(p.water) - (py[i] - nr.r)) / (T(2.0f) * nr.r), T(0.0f), T(1.0f));
            ffy += T(0.7f) * m * T(p.gravity) * wet;
        }
    }

    // creature.cu:553-593
    void bone_drag() {
        for (uint32_t j = 0; j + 1 < N; j++) {
            const Bone& b = bone[j];
            const uint32_t i0 = b.i0, i1 = j + 1;
            const T wx = T(0.5f) * (vx[i0] + vx[i1]), wy = T(0.5f) * (vy[i0] + vy[i1]);
            const T speed = sqrt_(wx * wx + wy * wy);
            const T k_air = min_(b.kair * speed, b.limit);
            T dfx = -wx * k_air, dfy = -wy * k_air;
            if (has(WATER)) {
                const T r0 = node[i0].r, r1 = node[i1].r;
                const T width = r0 + r1;
                const T wet0 = clamp((T(p.water) - (py[i0] - r0)) / (T(2.0f) * r0), T(0.0f), T(1.0f));
                const T wet1 = clamp((T(p.water) - (py[i1] - r1)) / (T(2.0f) * r1), T(0.0f), T(1.0f));
                const T wet = T(0.5f) * (wet0 + wet1);
                const T ax = (px[i1] - px[i0]) / b.len, ay = (py[i1] - py[i0]) / b.len;
                const T along = wx * ax + wy * ay;
                const T lx = ax * along, ly = ay * along;
                const T sx = wx - lx, sy = wy - ly;
                const T k_water = min_(T(100.0f) * wet * b.len * width * speed, b.limit);
                dfx -= sx * k_water + lx * k_water * T(0.25f);
                dfy -= sy * k_water + ly * k_water * T(0.25f);
            }
            vx[i0] += b.s0 * dfx;
            vy[i0] += b.s0 * dfy;
            vx[i1] += b.s1 * dfx;
            vy[i1] += b.s1 * dfy;
        }
    }

    // creature.cu:597-613
    void solve_bones() {
        for (uint32_t j = 0; j + 1 < N; j++) {
            const Bone& b = bone[j];
            const uint32_t i0 = b.i0, i1 = j + 1;
            const T dx = px[i1] - px[i0], dy = py[i1] - py[i0];
            const T len = max_(sqrt_(dx * dx + dy * dy), T(1e-9f));
            const T s = (len - b.len) / ((b.w0 + b.w1) * len);
            px[i0] += b.w0 * s * dx;
            py[i0] += b.w0 * s * dy;
            px[i1] -= b.w1 * s * dx;
            py[i1] -= b.w1 * s * dy;
        }
    }

    // creature.cu:618-634
    void solve_joints() {
        for (uint32_t j = 1; j + 1 < N; j++) {
            const Joint& k = joint[j];
            if (!k.has) continue;
            T angle, g[6];
            joint_eval(k, j + 1, true, angle, g);
            T error = T(0.0f);
            if (angle < k.lo) error = angle - k.lo;
            if (angle > k.hi) error = angle - k.hi;
            if (error == T(0.0f)) continue;
            const T w = joint_weight(k, g);
            if (w > T(0.0f)) joint_push(k, j + 1, g, -error / w, px, py);
        }
    }

    // creature.cu:640-679 (normal/friction out for a recording)
    void solve_ground(uint32_t i) {
        if (!has(GROUND)) return;
        const Node& nr = node[i];
        T gh, gs;
        ground(px[i], gh, gs);
        const T secant = sqrt_(T(1.0f) + gs * gs);
        const T nx = -gs / secant, ny = T(1.0f) / secant;
        const T dry = (py[i] - gh) / secant - nr.r;
        T depth, mu;
        if (has(MUD)) {
            depth = -(dry + T(p.mud));
            const T sink = clamp(-dry, T(0.0f), T(p.mud)) * (T(1.0f) / T(0.1f));
            mu = nr.mu * T(p.friction) * (T(1.0f) + T(2.0f) * sink) * (T(1.0f) + T(2.0f) * sink);
        } else {
            depth = -dry;
            mu = nr.mu * T(p.friction);
        }
        if (depth <= T(0.0f)) return;
        if (has(ICE)) mu *= T(1.0f) - T(p.patches) * ice_at(px[i]);
        px[i] += nx * depth;
        py[i] += ny * depth;
        const T tx = ny, ty = -nx;
        const T slide = (px[i] - fx[i]) * tx + (py[i] - fy[i]) * ty;
        const T budget = mu * depth;
        const T back = abs_(slide) <= budget ? slide : copysign_(budget, slide);
        px[i] -= tx * back;
        py[i] -= ty * back;
    }

    // creature.cu:683-702
    void damp_joints() {
        const T share = min_(h * T(10.0f), T(1.0f));
        for (uint32_t j = 1; j + 1 < N; j++) {
            const Joint& k = joint[j];
            if (!k.has) continue;
            T angle, g[6];
            joint_eval(k, j + 1, false, angle, g);
            const T rate_ = g[0] * vx[j + 1] + g[1] * vy[j + 1] + g[2] * vx[k.far] + g[3] * vy[k.far] +
                            g[4] * vx[k.hub] + g[5] * vy[k.hub];
            const T w = joint_weight(k, g);
            if (w > T(0.0f)) joint_push(k, j + 1, g, -share * rate_ / w, vx, vy);
        }
    }

    // creature.cu:705-742
    void substep() {
        muscle_forces();
        bone_drag();
        for (uint32_t i = 0; i < N; i++) {
            T ffx, ffy;
            node_force(i, ffx, ffy);
            vx[i] += h * (ffx + fx[i]) * node[i].im;
            vy[i] += h * (ffy + fy[i]) * node[i].im;
            if (has(AIR)) {
                vx[i] *= T(p.air_sub);
                vy[i] *= T(p.air_sub);
            }
            fx[i] = px[i];
            fy[i] = py[i];
            px[i] += h * vx[i];
            py[i] += h * vy[i];
        }
        solve_bones();
        solve_joints();
        for (uint32_t i = 0; i < N; i++) {
            solve_ground(i);
            vx[i] = (px[i] - fx[i]) * inv_h;
            vy[i] = (py[i] - fy[i]) * inv_h;
        }
        damp_joints();
    }

    // creature.cu:746-759
    bool any_broken() const {
        for (uint32_t j = 1; j + 1 < N; j++) {
            const Joint& k = joint[j];
            if (!k.has) continue;
            T angle, g[6];
            joint_eval(k, j + 1, true, angle, g);
            if (angle < k.lo - T(0.5f) || angle > k.hi + T(0.5f)) return true;
        }
        return false;
    }

    // creature.cu:956-1235 for a scoring trial.
    void run(Result& mt, float* trace, size_t trace_steps) {
        std::memset(&mt, 0, sizeof mt);
        mt.vertical_oscillation = 1e20f;
        mt.gait_frequency = -1e20f;
        uint32_t contact_bits = 0, lift_bits = 0, ground_bits = 0;
        T head_shake = T(0.0f), hax = px[0], hay = py[0], hvx = T(0.0f), hvy = T(0.0f);
        uint32_t rung_x = 0, rung_speed = 0, rung_early = 0, rung_late = 0, rung_bits = 0;
        T vo = T(1e20f), gf = T(-1e20f), prev = T(0.0f), ext = T(0.0f), trend = T(0.0f), turns = T(0.0f);
        T height_sum = T(0.0f), ground_contact = T(0.0f);
        const uint32_t r = (uint32_t)to_f(rate);
        const uint32_t rung1 = r - 1, rung2 = (uint32_t)(2.5f * (float)r) - 1;
        const uint32_t rung3 = (uint32_t)(5.0f * (float)r) - 1, rung4 = (uint32_t)(10.0f * (float)r) - 1;
        const uint32_t half_s = (uint32_t)(0.5f * (float)r);
        for (uint32_t step = 0;; step++) {
            const T t_now = T((float)step) * dt;
            muscle_demands(t_now, false);
            for (uint32_t s = 0; s < 16u; s++) {
                const uint32_t k = step * 16u + s;
                if (resync && k % resync_every == 0u && k / resync_every < resync_count) {
                    resync_state(resync + (size_t)(k / resync_every) * (4u * resync_rows + resync_mm));
                }
                substep();
            }
            if (trace && step < trace_steps) {
                for (uint32_t i = 0; i < N; i++) {
                    trace[(step * 32 + i) * 2] = to_f(px[i]);
                    trace[(step * 32 + i) * 2 + 1] = to_f(py[i]);
                }
            }
            bool failed = false;
            T center_y = T(0.0f), com_x = T(0.0f), low = T(1e20f), high = T(-1e20f);
            uint32_t touching = 0, lifted = 0;
            for (uint32_t i = 0; i < N; i++) {
                failed = failed || !(abs_(px[i]) <= T(1e6f) && abs_(py[i]) <= T(1e6f));
                center_y += py[i];
                com_x += node[i].m * px[i];
                low = min_(low, py[i] - node[i].r);
                high = max_(high, py[i] + node[i].r);
                if (has(GROUND)) {
                    T gh, gs;
                    ground(px[i], gh, gs);
                    const T floor_y = gh + node[i].r * sqrt_(T(1.0f) + gs * gs);
                    if (py[i] <= floor_y + T(0.002f)) touching |= 1u << i;
                    if (py[i] > floor_y + T(0.01f)) lifted |= 1u << i;
                }
            }
            center_y /= T((float)N);
            com_x *= inv_mass;
            contact_bits |= touching;
            lift_bits |= contact_bits & lifted;
            const uint32_t down = touching & ~ground_bits;
            ground_bits = touching;
            if (down != 0 && step > 0) {
                const T next = t_now + dt;
                for (Muscle& u : mus) {
                    if (u.sensor != NONE && ((down >> u.sensor) & 1u)) {
                        u.offset = frac(u.reset - (next * u.iper + u.phase));
                    }
                }
            }
            if ((step + 1) % head_sample == 0) {
                const T vxh = (px[0] - hax) * T(60.0f), vyh = (py[0] - hay) * T(60.0f);
                const T ax = (vxh - hvx) * T(60.0f), ay = (vyh - hvy) * T(60.0f);
                if (t_now >= T(0.1f)) {
                    const T accel = sqrt_(ax * ax + ay * ay);
                    head_shake += (accel - head_shake) * min_(T(1.0f) / (T(0.1f) * T(60.0f)), T(1.0f));
                }
                hax = px[0];
                hay = py[0];
                hvx = vxh;
                hvy = vyh;
            }
            const bool broken = any_broken();
            mt.contact_lo = fbits(contact_bits);
            mt.lift_lo = fbits(lift_bits);
            mt.ground_lo = fbits(ground_bits);
            mt.head_shake = to_f(head_shake);
            const bool fell = py[0] < py[1] || broken || head_shake > T(78.4f) || failed;
            bool ended = false;
            if (fell) {
                mt.fall_time = to_f(t_now + dt);
                mt.fitness = failed ? -1e20f : to_f(com_x);
                fit_t = failed ? T(0.0f) : com_x;
                if (step <= p.screen_step) mt.screen_x = mt.fitness;
                ended = true;
            }
            ground_contact += T((float)__builtin_popcount(touching));
            height_sum += high - low;
            vo = min_(vo, center_y);
            gf = max_(gf, center_y);
            if (step == 0) {
                prev = center_y;
                ext = center_y;
                trend = T(0.0f);
                turns = T(0.0f);
            } else if (step % sample == 0) {
                const T delta = center_y - prev;
                if (trend == T(0.0f)) {
                    if (abs_(delta) > T(0.0005f)) {
                        trend = delta > T(0.0f) ? T(1.0f) : T(-1.0f);
                        ext = center_y;
                    }
                } else if (trend > T(0.0f)) {
                    if (center_y > ext) {
                        ext = center_y;
                    } else if (ext - center_y > T(0.005f)) {
                        turns += T(1.0f);
                        trend = T(-1.0f);
                        ext = center_y;
                    }
                } else {
                    if (center_y < ext) {
                        ext = center_y;
                    } else if (center_y - ext > T(0.005f)) {
                        turns += T(1.0f);
                        trend = T(1.0f);
                        ext = center_y;
                    }
                }
                prev = center_y;
            }
            const float comf = to_f(com_x);
            if (step + half_s == rung1 || step + half_s == rung2) rung_x = ubits(comf);
            if (step == rung1 || step == rung2) {
                const bool second = step == rung2;
                const uint32_t sh = second ? 16 : 0;
                const uint32_t keep = second ? 0x0000ffffu : 0xffff0000u;
                const float speed = (comf - fbits(rung_x)) * ((float)r / (float)half_s);
                const float touched = (float)__builtin_popcount(contact_bits) / (float)N;
                T en = T(0.0f);
                for (const Muscle& u : mus) en += u.energy;
                en /= T((float)std::max(M, 1u));
                const float en_mean = to_f(en);
                const float hs = to_f(head_shake);
                mt.contact_hi = fbits((ubits(mt.contact_hi) & keep) | (f2h(comf) << sh));
                mt.ground_hi = fbits((ubits(mt.ground_hi) & keep) | (f2h(hs) << sh));
                rung_speed = (rung_speed & keep) | (f2h(speed) << sh);
                const uint32_t pair = f2h(touched) | (f2h(en_mean) << 16);
                if (second) rung_late = pair;
                else rung_early = pair;
                const uint32_t rr = second ? 1 : 0;
                const float gait_now = to_f(turns) * (0.5f / to_f(t_now + dt));
                const uint32_t band = std::min((uint32_t)(gait_now * (8.0f / 6.0f)), 7u);
                rung_bits |= band << (8 + 3 * rr);
                if (!ended && (cflags & (second ? 0xbu : 0x7u)) == 0u) {
                    const RungParams& rp = second ? p.r2 : p.r1;
                    const float fv[6] = {h2f(f2h(comf)), h2f(f2h(speed)), h2f(f2h(touched)), h2f(f2h(hs)),
                                         h2f(f2h(en_mean)), to_f(period_f)};
                    float score = 0.0f;
                    bool finite = true;
                    for (int i = 0; i < 6; i++) {
                        score = std::fma(rp.w[i], fv[i], score);
                        finite = finite && std::isfinite(fv[i]);
                    }
                    if (finite && score < rp.bias && ((rp.off >> band) & 1u) == 0u) {
                        mt.screened = to_f(t_now + dt);
                        mt.screen_x = comf;
                        mt.fitness = comf;
                        fit_t = com_x;
                        rung_bits |= (rr + 1) << 6;
                        ended = true;
                    }
                }
            }
            if (step == rung3 || step == rung4) {
                const bool second = step == rung4;
                const uint32_t keep = second ? 0x0000ffffu : 0xffff0000u;
                mt.lift_hi = fbits((ubits(mt.lift_hi) & keep) | (f2h(comf) << (second ? 16 : 0)));
            }
            if (step == p.screen_step && !ended) {
                mt.screen_x = comf;
                const float bar = (cflags & 32u) ? p.screen_bar_reshaped
                                  : (cflags & 16u) ? p.screen_bar_young
                                                   : p.screen_bar;
                if (comf < bar && (cflags & 1u) == 0u) {
                    mt.screened = to_f(t_now + dt);
                    mt.fitness = comf;
                    fit_t = com_x;
                    ended = true;
                }
            }
            bool last = false;
            if (ended) {
                vo = max_(gf - vo, T(0.0f));
                gf = turns * T(0.5f) / (t_now + dt);
            } else if (step + 1 >= p.steps) {
                mt.fitness = comf;
                fit_t = com_x;
                vo = max_(gf - vo, T(0.0f));
                gf = turns * T(0.5f) / max_(T((float)(step + 1)) * dt, dt);
                last = true;
            }
            if (ended || last) {
                const uint32_t fin = f2h(mt.fitness);
                uint32_t d = ubits(mt.contact_hi);
                if (step < rung1) d = (d & 0xffff0000u) | fin;
                if (step < rung2) d = (d & 0x0000ffffu) | (fin << 16);
                mt.contact_hi = fbits(d);
                d = ubits(mt.lift_hi);
                if (step < rung3) d = (d & 0xffff0000u) | fin;
                if (step < rung4) d = (d & 0x0000ffffu) | (fin << 16);
                mt.lift_hi = fbits(d);
                const uint32_t code = (fell ? 16u : 0u) | (failed ? 32u : 0u) | (mt.screened > 0.0f ? 3u : 0u) |
                                      (rung_bits & 0x3fc0u) | ((cflags & 1u) << 14);
                mt.ground_contact = to_f(ground_contact);
                mt.vertical_oscillation = to_f(vo);
                mt.gait_frequency = to_f(gf);
                mt.height_sum = to_f(height_sum);
                mt.previous_center_y = fbits(rung_speed);
                mt.vertical_extremum = fbits(rung_early);
                mt.vertical_trend = fbits(rung_late);
                mt.gait_turns = mt.ground_hi;
                mt.ground_hi = fbits(code | (std::min(step + 1, 65535u) << 16));
                return;
            }
        }
    }
};

}  // namespace

template <class T>
void simulate(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t cidx, const Params& p,
              uint32_t flags, int rate, Result* out, float* trace, size_t trace_steps) {
    Sim<T> s(p, flags, rate);
    s.begin(records, muscles, heads, cidx);
    s.run(*out, trace, trace_steps);
}

double tangent(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t cidx, const Params& p,
               uint32_t flags, int rate, const double* dmuscle, const double* dnode, Result* out,
               const float* resync, uint32_t rows, uint32_t mm, uint32_t count, uint32_t every, double* fitness,
               const double* dmass, const double* dstart) {
    Sim<Dual> s(p, flags, rate);
    s.seed_mass = dmass;
    s.seed_start = dstart;
    s.begin(records, muscles, heads, cidx);
    s.resync_every = every > 0 ? every : 256u;
    s.resync = resync;
    s.resync_rows = rows;
    s.resync_mm = mm;
    s.resync_count = count;
    for (size_t k = 0; k < s.mus.size(); k++) {
        auto& u = s.mus[k];
        const double* d = dmuscle + 9 * k;
        u.amp.d = d[0];
        u.hill.d = d[1];
        u.cap.d = d[2];
        u.icap.d = d[3];
        u.phase.d = d[4];
        u.duty.d = d[5];
        u.iduty.d = d[6];
        u.icomp.d = d[7];
        u.stiff.d = d[8];
    }
    for (size_t i = 0; i < s.node.size(); i++) {
        s.node[i].mu.d = dnode[i];
    }
    s.run(*out, nullptr, 0);
    if (fitness) *fitness = s.fit_t.v;
    return s.fit_t.d;
}

template void simulate<float>(const uint32_t*, const float*, const uint32_t*, size_t, const Params&, uint32_t, int,
                              Result*, float*, size_t);
template void simulate<double>(const uint32_t*, const float*, const uint32_t*, size_t, const Params&, uint32_t, int,
                               Result*, float*, size_t);
template void simulate<Counted>(const uint32_t*, const float*, const uint32_t*, size_t, const Params&, uint32_t,
                                int, Result*, float*, size_t);

}  // namespace oracle

// ------------------------------------------------------------------ C ABI
extern "C" {

// Runs creatures [first, first + n) of a packed batch in FP32 (precision 0)
// or FP64 (precision 1) on `threads` host threads (0: all). Returns the wall
// seconds.
double oracle_run(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t first, size_t n,
                  const oracle::Params* p, uint32_t flags, int rate, int precision, oracle::Result* out,
                  int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 16)
    for (long long i = 0; i < (long long)n; i++) {
        if (precision == 1) {
            oracle::simulate<double>(records, muscles, heads, first + i, *p, flags, rate, out + i, nullptr, 0);
        } else {
            oracle::simulate<float>(records, muscles, heads, first + i, *p, flags, rate, out + i, nullptr, 0);
        }
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Positions after every step of creature `cidx` (32 pairs a step).
void oracle_trace(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t cidx,
                  const oracle::Params* p, uint32_t flags, int rate, int precision, oracle::Result* out,
                  float* trace, size_t trace_steps) {
    if (precision == 1) {
        oracle::simulate<double>(records, muscles, heads, cidx, *p, flags, rate, out, trace, trace_steps);
    } else {
        oracle::simulate<float>(records, muscles, heads, cidx, *p, flags, rate, out, trace, trace_steps);
    }
}

// FP64 tangents of creatures [first, first + n): for creature c the record
// directions sit at dmuscle + c * 9 * mm and dnode + c * rows; d fitness goes
// to dfit[c] and the FP64 fitness to fit[c] (when not NULL). `dmass` (NULL
// for none, else rows a creature) moves the node masses too, and `dstart`
// (NULL for none, else 2 x rows a creature) the start positions. Returns the
// wall seconds.
double oracle_tangent(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t first, size_t n,
                      const oracle::Params* p, uint32_t flags, int rate, const double* dmuscle, const double* dnode,
                      uint32_t rows, uint32_t mm, double* dfit, double* fit, oracle::Result* out, int threads,
                      const double* dmass, const double* dstart) {
    if (threads > 0) omp_set_num_threads(threads);
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < (long long)n; i++) {
        dfit[i] = oracle::tangent(records, muscles, heads, first + i, *p, flags, rate, dmuscle + i * 9 * mm,
                                  dnode + i * rows, out + i, nullptr, 0, 0, 0, 256, fit ? fit + i : nullptr,
                                  dmass ? dmass + i * rows : nullptr, dstart ? dstart + 2 * i * rows : nullptr);
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// As oracle_tangent, the state reset at every checkpoint to `ckpt` (per
// creature `count` checkpoints of rows x 4 + mm floats, one every `every`
// substeps, creature c's at ckpt + c * ckpt_stride): the FP64 tangent along
// another run's trajectory.
double oracle_tangent_along(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t first,
                            size_t n, const oracle::Params* p, uint32_t flags, int rate, const double* dmuscle,
                            const double* dnode, uint32_t rows, uint32_t mm, const float* ckpt, size_t ckpt_stride,
                            uint32_t count, uint32_t every, double* dfit, double* fit, oracle::Result* out,
                            int threads, const double* dmass) {
    if (threads > 0) omp_set_num_threads(threads);
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < (long long)n; i++) {
        dfit[i] = oracle::tangent(records, muscles, heads, first + i, *p, flags, rate, dmuscle + i * 9 * mm,
                                  dnode + i * rows, out + i, ckpt + (first + i) * ckpt_stride, rows, mm, count,
                                  every, fit ? fit + i : nullptr, dmass ? dmass + i * rows : nullptr, nullptr);
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Counts the arithmetic of creature `cidx`'s trial: out[0..7] = add, mul,
// div, sqrt, transcendental, min/max, compare, other.
void oracle_count(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t cidx,
                  const oracle::Params* p, uint32_t flags, int rate, oracle::Result* out, uint64_t counts[8]) {
    oracle::g_ops = oracle::OpCount{};
    oracle::simulate<oracle::Counted>(records, muscles, heads, cidx, *p, flags, rate, out, nullptr, 0);
    const oracle::OpCount& c = oracle::g_ops;
    const uint64_t v[8] = {c.add, c.mul, c.div, c.sqrt, c.trans, c.minmax, c.cmp, c.other};
    for (int i = 0; i < 8; i++) counts[i] = v[i];
}
}
