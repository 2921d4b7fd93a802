// Test infrastructure: the CPU oracle of the creature path.
//
// A restatement of the reference kernel's per-creature simulation
// (shaders/creature.cu:130-1248) on the host, templated on the scalar type:
//   float    -- the FP32 oracle, with the C library's cosf/atan2f and IEEE
//               division and square root where the kernel uses __cosf,
//               atan2f and approximate division and square root, and no
//               fused multiply-adds; it agrees with the GPU to a tolerance
//               over short horizons, not to the bit;
//   double   -- the FP64 reference of the same trial;
//   Counted  -- float arithmetic that counts its operations, which gives the
//               algorithmic FP32 operations per creature-substep.
// It reads the same packed records as the kernels (src/kernel.rs:336-593).
// Only the tests, the smoke check and the benchmark's CPU baseline use it.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {

// Operation counts of a Counted run, by kind.
struct OpCount {
    uint64_t add = 0, mul = 0, div = 0, sqrt = 0, trans = 0, minmax = 0, cmp = 0, other = 0;
    uint64_t total() const { return add + mul + div + sqrt + trans + minmax + cmp + other; }
};
extern thread_local OpCount g_ops;

struct Counted {
    float v;
    Counted() : v(0.0f) {}
    Counted(float x) : v(x) {}
    explicit operator float() const { return v; }
};
inline Counted operator+(Counted a, Counted b) { g_ops.add++; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { g_ops.add++; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { g_ops.mul++; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { g_ops.div++; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted& operator+=(Counted& a, Counted b) { a = a + b; return a; }
inline Counted& operator-=(Counted& a, Counted b) { a = a - b; return a; }
inline Counted& operator*=(Counted& a, Counted b) { a = a * b; return a; }
inline Counted& operator/=(Counted& a, Counted b) { a = a / b; return a; }
inline bool operator<(Counted a, Counted b) { g_ops.cmp++; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { g_ops.cmp++; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { g_ops.cmp++; return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { g_ops.cmp++; return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { g_ops.cmp++; return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { g_ops.cmp++; return a.v != b.v; }

// Scalar functions for each scalar type.
inline float sqrt_(float x) { return std::sqrt(x); }
inline double sqrt_(double x) { return std::sqrt(x); }
inline Counted sqrt_(Counted x) { g_ops.sqrt++; return Counted(std::sqrt(x.v)); }
inline float cos_(float x) { return std::cos(x); }
inline double cos_(double x) { return std::cos(x); }
inline Counted cos_(Counted x) { g_ops.trans++; return Counted(std::cos(x.v)); }
inline float atan2_(float y, float x) { return std::atan2(y, x); }
inline double atan2_(double y, double x) { return std::atan2(y, x); }
inline Counted atan2_(Counted y, Counted x) { g_ops.trans++; return Counted(std::atan2(y.v, x.v)); }
inline float floor_(float x) { return std::floor(x); }
inline double floor_(double x) { return std::floor(x); }
inline Counted floor_(Counted x) { g_ops.other++; return Counted(std::floor(x.v)); }
inline float abs_(float x) { return std::fabs(x); }
inline double abs_(double x) { return std::fabs(x); }
inline Counted abs_(Counted x) { g_ops.other++; return Counted(std::fabs(x.v)); }
inline float min_(float a, float b) { return std::fmin(a, b); }
inline double min_(double a, double b) { return std::fmin(a, b); }
inline Counted min_(Counted a, Counted b) { g_ops.minmax++; return Counted(std::fmin(a.v, b.v)); }
inline float max_(float a, float b) { return std::fmax(a, b); }
inline double max_(double a, double b) { return std::fmax(a, b); }
inline Counted max_(Counted a, Counted b) { g_ops.minmax++; return Counted(std::fmax(a.v, b.v)); }
inline float copysign_(float a, float b) { return std::copysign(a, b); }
inline double copysign_(double a, double b) { return std::copysign(a, b); }
inline Counted copysign_(Counted a, Counted b) { g_ops.other++; return Counted(std::copysign(a.v, b.v)); }
// FP64 dual number: value and one directional derivative (forward mode).
struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double x) : v(x), d(0.0) {}
    Dual(double x, double dx) : v(x), d(dx) {}
};
inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) { return Dual(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
inline Dual& operator-=(Dual& a, Dual b) { a = a - b; return a; }
inline Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }
inline Dual& operator/=(Dual& a, Dual b) { a = a / b; return a; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }
inline Dual sqrt_(Dual x) {
    const double s = std::sqrt(x.v);
    return Dual(s, s > 0.0 ? x.d / (2.0 * s) : 0.0);
}
inline Dual cos_(Dual x) { return Dual(std::cos(x.v), -std::sin(x.v) * x.d); }
inline Dual atan2_(Dual y, Dual x) {
    const double r = x.v * x.v + y.v * y.v;
    return Dual(std::atan2(y.v, x.v), r > 0.0 ? (x.v * y.d - y.v * x.d) / r : 0.0);
}
inline Dual floor_(Dual x) { return Dual(std::floor(x.v), 0.0); }
inline Dual abs_(Dual x) { return x.v < 0.0 ? -x : x; }
inline Dual min_(Dual a, Dual b) { return b.v < a.v ? b : a; }
inline Dual max_(Dual a, Dual b) { return b.v > a.v ? b : a; }
inline Dual copysign_(Dual a, Dual b) { return std::signbit(a.v) == std::signbit(b.v) ? a : -a; }
inline float to_f(Dual x) { return (float)x.v; }
inline bool finite_(Dual x) { return std::isfinite(x.v); }

inline float to_f(float x) { return x; }
inline float to_f(double x) { return (float)x; }
inline float to_f(Counted x) { return x.v; }
inline bool finite_(float x) { return std::isfinite(x); }
inline bool finite_(double x) { return std::isfinite(x); }
inline bool finite_(Counted x) { return std::isfinite(x.v); }

// Launch parameters with the layout of the kernels' Params
// (shaders/creature.cu:75-103).
struct RungParams {
    float w[6];
    float bias;
    uint32_t off;
};
struct Params {
    uint32_t count, base, steps, screen_step, stride;
    float gravity, air, friction, terrain, muscle_energy, muscle_recovery, slope, wind, mud, gaps, hurdles, quake;
    float screen_bar, screen_bar_young, screen_bar_reshaped, water, patches, air_sub, inv_muscle_energy, brambles;
    RungParams r1, r2;
};
struct Result {
    float fitness, ground_contact, vertical_oscillation, gait_frequency, previous_center_y, vertical_extremum,
        vertical_trend, gait_turns, height_sum, contact_lo, contact_hi, lift_lo, lift_hi, ground_lo, ground_hi,
        fall_time, head_shake, screen_x, screened;
};

enum : uint32_t {
    GROUND = 1u << 0, TERRAIN = 1u << 1, SLOPE = 1u << 2, GAPS = 1u << 3, HURDLES = 1u << 4, QUAKE = 1u << 5,
    MUD = 1u << 6, WATER = 1u << 7, ICE = 1u << 8, WIND = 1u << 9, AIR = 1u << 10, BRAMBLES = 1u << 11
};

// Runs creature `cidx` of a packed batch. `trace` (optional) receives the node
// positions after every step, 32 pairs a step (unused pairs left as they are);
// `trace_steps` is its room in steps.
template <class T>
void simulate(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t cidx, const Params& p,
              uint32_t flags, int rate, Result* out, float* trace, size_t trace_steps);

// FP64 tangent of creature `cidx`'s fitness: the trial run in dual numbers
// with the record fields moved along `dmuscle` (9 a muscle: amplitude, hill,
// cap, 1/capacity, phase, duty, 1/duty, 1/(1-duty), stiffness) and `dnode`
// (friction a node row) and, when not NULL, the node masses along `dmass`
// (a node row each; 1/m, the bone and joint weights and 1/total mass follow).
// Returns d fitness; `out` gets the FP64 trial's result and `fitness` (when
// not NULL) its fitness in FP64.
// With `resync` (count checkpoints of rows x 4 + mm floats: positions,
// velocities, energy stores every `every` substeps) the state's values are
// reset to them at each checkpoint and their derivative parts kept.
double tangent(const uint32_t* records, const float* muscles, const uint32_t* heads, size_t cidx, const Params& p,
               uint32_t flags, int rate, const double* dmuscle, const double* dnode, Result* out,
               const float* resync, uint32_t rows, uint32_t mm, uint32_t count, uint32_t every,
               double* fitness, const double* dmass, const double* dstart = nullptr);

// The value part of a scalar of the oracle (for dual numbers: keeps the
// derivative).
inline void set_value(float& x, float v) { x = v; }
inline void set_value(double& x, float v) { x = v; }
inline void set_value(Counted& x, float v) { x = Counted(v); }
inline void set_value(Dual& x, float v) { x.v = v; }
// The derivative part of a scalar (dual numbers only).
inline void set_deriv(float&, double) {}
inline void set_deriv(double&, double) {}
inline void set_deriv(Counted&, double) {}
inline void set_deriv(Dual& x, double d) { x.d = d; }

}  // namespace oracle
