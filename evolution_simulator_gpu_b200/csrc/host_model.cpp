// Host side of the creature path: the body model and its packing into the
// kernel records, the launch parameters, the result metrics and niche cells,
// and the seeded synthetic population generator.
//
// The packing restates the reference's host model so that a body packs into
// the same words the reference would upload:
//   physics::node_mass / body / add_muscle_masses  src/physics.rs:182-296
//   physics2::Model::new / start / kinematics      src/physics2.rs:186-428
//   kernel::fill_creature / pack_reusing           src/kernel.rs:336-593
//   kernel::params / world_flags                   src/kernel.rs:82-251
//   physics ground, quake hash                     src/physics.rs:523-714
//   f32 -> f16                                      src/creature_kernel.rs:242-274
// The reference host is Rust, whose f32 arithmetic is IEEE single with no
// contraction of multiply-adds. This file is built with -ffp-contract=off and
// calls the C library's single-precision functions (atan2f, sinf, cosf, powf,
// logf) that Rust's f32 methods call on Linux, so each value rounds as there.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/creature_engine.h"
#include "host_model.h"
#include "packer.h"

namespace ce {

thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

// The host's arctangent, sine and cosine: the C library's single-precision
// functions, as Rust's f32::atan2, sin and cos call them.
struct HostAngle {
    float operator()(size_t, float dy, float dx) const { return std::atan2(dy, dx); }
};
struct HostTrig {
    void operator()(size_t, float th, float& sn, float& cs) const {
        sn = std::sin(th);
        cs = std::cos(th);
    }
};
static Model make_model(const ce_node_gene* g, size_t n, const ce_bone_gene* bones, size_t nb,
                        const ce_muscle_gene* mg, size_t nm, uint64_t id, const ce_world& w) {
    return make_model(g, n, bones, nb, mg, nm, id, w, HostAngle{});
}
static State start_state(const Model& M, const ce_world& w) { return start_state(M, w, HostTrig{}); }
void fill_creature(const ce_population& pop, size_t i, const ce_world& w, uint32_t* record, float* muscles,
                   uint32_t* head, uint32_t record_at, uint32_t muscle_at) {
    fill_creature(pop, i, w, record, muscles, head, record_at, muscle_at, HostAngle{}, HostTrig{});
}

float f16_to_f32(uint16_t h) {
    const uint32_t sign = (uint32_t)(h >> 15) << 31;
    const uint32_t exponent = (h >> 10) & 0x1fu;
    const uint32_t mantissa = h & 0x3ffu;
    uint32_t bits;
    if (exponent == 0 && mantissa == 0) {
        bits = sign;
    } else if (exponent == 0) {
        uint32_t shift = (uint32_t)__builtin_clz(mantissa) - 21;
        const uint32_t m = (mantissa << shift) & 0x3ffu;
        bits = sign | ((113 - shift) << 23) | (m << 13);
    } else if (exponent == 31) {
        bits = sign | 0x7f800000u | (mantissa ? (0x00400000u | (mantissa << 13)) : 0u);
    } else {
        bits = sign | ((exponent + 112) << 23) | (mantissa << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// ------------------------------------------------------------- validation
bool validate_body(const ce_population& pop, size_t i, std::string* why) {
    const ce_genome& gm = pop.genomes[i];
    const size_t n = gm.node_count, nb = gm.bone_count, nm = gm.muscle_count;
    if (n < 2 || n > CE_MAX_NODES || nm > CE_MAX_MUSCLES) {
        if (why) *why = "Unsupported body for the CUDA kernel: " + std::to_string(n) + " nodes, " +
                        std::to_string(nm) + " muscles";
        return false;
    }
    if (nb != n - 1) {
        if (why) *why = "a body of n nodes needs n - 1 bones";
        return false;
    }
    const ce_bone_gene* bones = pop.bones + gm.bone_start;
    std::vector<char> seen(n, 0);
    seen[0] = 1;
    for (size_t j = 0; j < nb; j++) {
        if (bones[j].a >= n || bones[j].b >= n || bones[j].b == 0 || !seen[bones[j].a] || seen[bones[j].b]) {
            if (why) *why = "bones are not a parent-first tree rooted at node 0";
            return false;
        }
        seen[bones[j].b] = 1;
    }
    if (nb > 0 && bones[0].a != 0) {
        if (why) *why = "bone 0 must leave the head";
        return false;
    }
    const ce_muscle_gene* ms = pop.muscles + gm.muscle_start;
    for (size_t k = 0; k < nm; k++) {
        if (ms[k].bone_a >= nb || ms[k].bone_b >= nb || (ms[k].sensor != CE_NO_SENSOR && ms[k].sensor > 3)) {
            if (why) *why = "a muscle names a missing bone or sensor";
            return false;
        }
    }
    return true;
}

// Fidelity (src/physics.rs:76-101) of a world.
uint32_t world_rate(const ce_world& w) { return w.rate ? w.rate : 60u; }
uint32_t world_settle(const ce_world& w) { return (200u * world_rate(w) + 119u) / 120u; }
uint32_t world_sample(const ce_world& w) { return std::max(world_rate(w) / 30u, 1u); }
uint32_t world_steps(const ce_world& w) { return (uint32_t)std::round(w.duration * (float)world_rate(w)); }
float world_air_per_step(const ce_world& w) {
    return std::pow(w.air_retention, 60.0f / (float)world_rate(w));
}

}  // namespace ce

using namespace ce;

// ---------------------------------------------------------------- C ABI
extern "C" uint32_t ce_world_flags(const ce_world* w) {
    const bool g = w->ground != 0;
    uint32_t flags = 0;
    auto set = [&](int bit, bool on) {
        if (on) flags |= 1u << bit;
    };
    set(0, g);
    set(1, g && (terrain_amplitude(w->terrain) != 0.0f || w->quake > 0.0f));
    set(2, g && w->slope != 0.0f);
    set(3, g && w->gaps > 0.0f);
    set(4, g && w->hurdles > 0.0f);
    set(5, g && w->quake > 0.0f);
    set(6, g && w->mud > 0.0f);
    set(7, w->water > 0.0f);
    set(8, g && w->patches > 0.0f);
    set(9, w->wind != 0.0f);
    set(10, world_air_per_step(*w) != 1.0f);
    set(11, g && w->brambles > 0.0f);
    return flags;
}

extern "C" ce_status ce_make_params(const ce_world* w, uint32_t base, uint32_t count, uint32_t stride,
                                    ce_params* out) {
    if (!w || !out) {
        set_error("ce_make_params: null argument");
        return CE_ERR_INVALID;
    }
    const bool g = w->ground != 0;
    const float air = world_air_per_step(*w);
    const float ninf = -std::numeric_limits<float>::infinity();
    ce_params p;
    std::memset(&p, 0, sizeof p);
    p.count = count;
    p.base = base;
    p.steps = world_steps(*w);
    if (w->has_screen) {
        const uint32_t r = world_rate(*w);
        const uint32_t tick = std::max((uint32_t)std::round(w->screen_seconds * (float)r), 1u) - 1u;
        p.screen_step = tick;
    } else {
        p.screen_step = 0xffffffffu;
    }
    p.stride = stride;
    p.gravity = w->gravity;
    p.air = air;
    p.friction = w->ground_friction;
    p.terrain = terrain_amplitude(w->terrain);
    p.muscle_energy = w->muscle_energy;
    p.muscle_recovery = w->muscle_recovery;
    p.slope = g ? w->slope : 0.0f;
    p.wind = w->wind;
    p.mud = g ? w->mud : 0.0f;
    p.gaps = g ? w->gaps : 0.0f;
    p.hurdles = g ? w->hurdles : 0.0f;
    p.quake = g ? w->quake : 0.0f;
    p.screen_bar = w->has_screen ? w->screen_bar : ninf;
    p.screen_bar_young = w->has_screen ? w->screen_bar_young : ninf;
    p.screen_bar_reshaped = w->has_screen ? w->screen_bar_reshaped : ninf;
    p.water = w->water;
    p.patches = g ? w->patches : 0.0f;
    p.air_sub = std::pow(air, 1.0f / (float)CE_SUBSTEPS);
    p.inv_muscle_energy = 1.0f / w->muscle_energy;
    p.brambles = g ? w->brambles : 0.0f;
    ce_rung never;
    std::memset(&never, 0, sizeof never);
    never.bias = ninf;
    p.r1 = w->has_rungs ? w->rungs[0] : never;
    p.r2 = w->has_rungs ? w->rungs[1] : never;
    *out = p;
    return CE_OK;
}

extern "C" uint32_t ce_frame_stride(uint32_t max_muscles) { return 2u * CE_MAX_NODES + max_muscles + 1u; }

static bool pack_order(const ce_population* pop, const uint32_t* indices, size_t n,
                       std::vector<uint32_t>& sorted_slot) {
    sorted_slot.resize(n);
    auto idx = [&](size_t s) -> size_t { return indices ? indices[s] : s; };
    // Validation in parallel; the first failing slot's reason is kept.
    long long bad = -1;
#pragma omp parallel for schedule(dynamic, 1024)
    for (long long s = 0; s < (long long)n; s++) {
        if (idx((size_t)s) >= pop->count || !validate_body(*pop, idx((size_t)s), nullptr)) {
#pragma omp critical(ce_pack_bad)
            if (bad < 0 || s < bad) bad = s;
        }
    }
    if (bad >= 0) {
        if (idx((size_t)bad) >= pop->count) {
            set_error("ce_pack: index out of range");
        } else {
            std::string why;
            validate_body(*pop, idx((size_t)bad), &why);
            set_error(why);
        }
        return false;
    }
    // Order: muscle count, then node count, then population index. With the
    // population indices ascending (or none given) a counting sort over the
    // (muscles, nodes) key in slot order gives exactly that order.
    bool ascending = true;
    for (size_t s = 1; indices && s < n && ascending; s++) ascending = indices[s - 1] < indices[s];
    if (!ascending) {
        std::iota(sorted_slot.begin(), sorted_slot.end(), 0u);
        std::stable_sort(sorted_slot.begin(), sorted_slot.end(), [&](uint32_t x, uint32_t y) {
            const ce_genome& a = pop->genomes[idx(x)];
            const ce_genome& b = pop->genomes[idx(y)];
            if (a.muscle_count != b.muscle_count) return a.muscle_count < b.muscle_count;
            if (a.node_count != b.node_count) return a.node_count < b.node_count;
            return idx(x) < idx(y);
        });
        return true;
    }
    constexpr size_t kNodeKeys = CE_MAX_NODES + 1;
    const size_t keys = (CE_MAX_MUSCLES + 1) * kNodeKeys;
    std::vector<size_t> start(keys + 1, 0);
    auto key = [&](size_t s) {
        const ce_genome& g = pop->genomes[idx(s)];
        return (size_t)g.muscle_count * kNodeKeys + g.node_count;
    };
    for (size_t s = 0; s < n; s++) start[key(s) + 1]++;
    for (size_t k = 0; k < keys; k++) start[k + 1] += start[k];
    for (size_t s = 0; s < n; s++) sorted_slot[start[key(s)]++] = (uint32_t)s;
    return true;
}

extern "C" ce_status ce_pack_size(const ce_population* pop, const uint32_t* indices, size_t n,
                                  size_t* lanes_len, size_t* muscles_len) {
    if (!pop || !lanes_len || !muscles_len) {
        set_error("ce_pack_size: null argument");
        return CE_ERR_INVALID;
    }
    size_t r = 0, m = 0;
    for (size_t s = 0; s < n; s++) {
        const size_t i = indices ? indices[s] : s;
        if (i >= pop->count) {
            set_error("ce_pack_size: index out of range");
            return CE_ERR_INVALID;
        }
        const ce_genome& g = pop->genomes[i];
        r += (size_t)g.node_count * CE_NODE_WORDS + (size_t)g.bone_count * CE_BONE_WORDS;
        m += (size_t)g.muscle_count * CE_MUSCLE_FIELDS;
    }
    *lanes_len = std::max<size_t>(r, 1);
    *muscles_len = std::max<size_t>(m, 1);
    return CE_OK;
}

extern "C" ce_status ce_pack(const ce_population* pop, const uint32_t* indices, size_t n,
                             const ce_world* w, uint32_t* lanes, float* muscles, uint32_t* heads,
                             uint32_t* slots, uint32_t* info) {
    if (!pop || !w || !lanes || !muscles || !heads) {
        set_error("ce_pack: null argument");
        return CE_ERR_INVALID;
    }
    std::vector<uint32_t> order;
    if (!pack_order(pop, indices, n, order)) return CE_ERR_INVALID;
    std::vector<size_t> record_at(n), muscle_at(n);
    size_t rl = 0, ml = 0;
    for (size_t c = 0; c < n; c++) {
        const ce_genome& g = pop->genomes[indices ? indices[order[c]] : order[c]];
        record_at[c] = rl;
        muscle_at[c] = ml;
        rl += (size_t)g.node_count * CE_NODE_WORDS + (size_t)g.bone_count * CE_BONE_WORDS;
        ml += (size_t)g.muscle_count * CE_MUSCLE_FIELDS;
    }
    if (rl > 0xffffffffull || ml > 0xffffffffull) {
        set_error("ce_pack: batch too large for 32-bit record offsets");
        return CE_ERR_INVALID;
    }
    lanes[0] = 0;
    muscles[0] = 0.0f;
    // Each creature writes only its own ranges; the fill runs in parallel.
#pragma omp parallel for schedule(dynamic, 256)
    for (long long c = 0; c < (long long)n; c++) {
        const size_t i = indices ? indices[order[c]] : order[c];
        fill_creature(*pop, i, *w, lanes + record_at[c], muscles + muscle_at[c], heads + 8 * c,
                      (uint32_t)record_at[c], (uint32_t)muscle_at[c]);
        if (info) {
            const ce_genome& g = pop->genomes[i];
            info[4 * c + 0] = g.node_count;
            info[4 * c + 1] = g.bone_count;
            info[4 * c + 2] = g.muscle_count;
            info[4 * c + 3] = quake_hash(g.id);
        }
    }
    if (slots) {
        for (size_t c = 0; c < n; c++) slots[c] = order[c];
    }
    return CE_OK;
}

// The host half of a device packing: the packed order and record offsets
// (as ce_pack lays them out) and, per bone gene, the three single-precision
// library values the device cannot reproduce: the bone's gene-pose
// direction atan2(dy, dx) and the sine and cosine of its start-pose angle
// (make_model and start_state call them; recording them here gives the
// device the same values). They depend on the node genes alone.
namespace {
struct RecordAngle {
    float* out;
    float operator()(size_t j, float dy, float dx) const {
        const float a = std::atan2(dy, dx);
        out[3 * j] = a;
        return a;
    }
};
struct RecordTrig {
    float* out;
    void operator()(size_t j, float th, float& sn, float& cs) const {
        sn = std::sin(th);
        cs = std::cos(th);
        out[3 * j + 1] = sn;
        out[3 * j + 2] = cs;
    }
};
}  // namespace

extern "C" ce_status ce_pack_plan(const ce_population* pop, const uint32_t* indices, size_t n, const ce_world* w,
                                  size_t bones_len, uint32_t* order, uint32_t* record_at, uint32_t* muscle_at,
                                  float* trig) {
    if (!pop || !w || !order || !record_at || !muscle_at || !trig) {
        set_error("ce_pack_plan: null argument");
        return CE_ERR_INVALID;
    }
    std::vector<uint32_t> slot;
    if (!pack_order(pop, indices, n, slot)) return CE_ERR_INVALID;
    size_t rl = 0, ml = 0;
    for (size_t c = 0; c < n; c++) {
        const uint32_t i = indices ? indices[slot[c]] : slot[c];
        const ce_genome& g = pop->genomes[i];
        if ((size_t)g.bone_start + g.bone_count > bones_len) {
            set_error("ce_pack_plan: a genome's bones lie past bones_len");
            return CE_ERR_INVALID;
        }
        order[c] = i;
        record_at[c] = (uint32_t)rl;
        muscle_at[c] = (uint32_t)ml;
        rl += (size_t)g.node_count * CE_NODE_WORDS + (size_t)g.bone_count * CE_BONE_WORDS;
        ml += (size_t)g.muscle_count * CE_MUSCLE_FIELDS;
        if (rl > 0xffffffffull || ml > 0xffffffffull) {
            set_error("ce_pack_plan: batch too large for 32-bit record offsets");
            return CE_ERR_INVALID;
        }
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (long long c = 0; c < (long long)n; c++) {
        const ce_genome& gm = pop->genomes[order[c]];
        float* t = trig + 3 * (size_t)gm.bone_start;
        const Model M = make_model(pop->nodes + gm.node_start, gm.node_count, pop->bones + gm.bone_start,
                                   gm.bone_count, pop->muscles + gm.muscle_start, gm.muscle_count, gm.id, *w,
                                   RecordAngle{t});
        (void)start_state(M, *w, RecordTrig{t});
    }
    return CE_OK;
}

// ---------------------------------------------------------------- metrics
// scheduler::trial_steps and to_metrics (src/scheduler.rs:859-923).
extern "C" ce_status ce_to_metrics(const ce_result* r, uint32_t node_count, const ce_world* w,
                                   ce_metrics* out) {
    if (!r || !w || !out) {
        set_error("ce_to_metrics: null argument");
        return CE_ERR_INVALID;
    }
    const uint32_t all = std::max(world_steps(*w), 1u);
    const float ended = r->fall_time > 0.0f ? r->fall_time : r->screened;
    uint32_t steps = all;
    if (ended > 0.0f) {
        const float x = std::round(ended * (float)world_rate(*w));
        const uint32_t s = x <= 0.0f ? 0u : (x >= 4294967295.0f ? 0xffffffffu : (uint32_t)x);
        steps = std::min(std::max(s, 1u), all);
    }
    const float denom = (float)(steps * node_count);
    ce_metrics m;
    m.fitness = r->fitness;
    m.ground_contact = clampf(r->ground_contact / denom, 0.0f, 1.0f);
    m.vertical_oscillation = std::isfinite(r->vertical_oscillation) ? fmax_(r->vertical_oscillation, 0.0f) : 0.0f;
    m.gait_frequency = std::isfinite(r->gait_frequency) ? fmax_(r->gait_frequency, 0.0f) : 0.0f;
    m.mean_height = fmax_(r->height_sum / (float)steps, 0.0f);
    m.feet = (float)__builtin_popcount(fbits(r->lift_lo));
    m.screen_x = r->screen_x;
    m.screened = r->screened > 0.0f ? 1u : 0u;
    m.steps = steps;
    *out = m;
    return CE_OK;
}

static uint8_t qd_bin(float value, float low, float high, uint8_t count) {
    const float f = std::floor((clampf(value, low, high) - low) / (high - low) * (float)count);
    const uint8_t b = f <= 0.0f ? 0 : (f >= 255.0f ? 255 : (uint8_t)f);
    return std::min<uint8_t>(b, count - 1);
}
static float height_axis(float h) {
    const float low = 0.15f;
    const float high = fmax_(0.6f * lim::max_bone, 2.0f * low);
    return clampf(std::log(fmax_(h, low) / low) / std::log(high / low), 0.0f, 1.0f);
}

// The shape class of a body (qd.rs:762-790): its gene extent's aspect
// against the layout's edges.
static uint8_t shape_class(const ce_node_gene* nodes, uint32_t node_count, int global_layout) {
    float min_x = std::numeric_limits<float>::infinity(), max_x = -min_x;
    float min_y = min_x, max_y = -min_x;
    for (uint32_t i = 0; i < node_count; i++) {
        min_x = fmin_(min_x, nodes[i].x);
        max_x = fmax_(max_x, nodes[i].x);
        min_y = fmin_(min_y, nodes[i].y);
        max_y = fmax_(max_y, nodes[i].y);
    }
    const float aspect = clampf(fmax_(max_x - min_x, 0.01f) / fmax_(max_y - min_y, 0.01f), 0.0625f, 16.0f);
    static const float g_aspect[3] = {0.9f, 1.4f, 2.5f};
    static const float i_aspect[2] = {1.2f, 2.0f};
    const float* ae = global_layout ? g_aspect : i_aspect;
    const int edges = global_layout ? 3 : 2;
    uint8_t shape = 0;
    for (int e = 0; e < edges; e++) shape += aspect >= ae[e] ? 1 : 0;
    return shape;
}

extern "C" int64_t ce_niche(const ce_node_gene* nodes, uint32_t node_count, uint32_t muscle_count,
                            const ce_metrics* m, int global_layout, uint8_t niche_out[6]) {
    (void)muscle_count;
    if (!nodes || !m) return -1;
    const float gc = clampf(m->ground_contact, 0.0f, 1.0f);
    const float gf = clampf(m->gait_frequency, 0.0f, 20.0f);
    const float mh = fmax_(m->mean_height, 0.0f);
    const float feet = fmax_(m->feet, 0.0f);
    static const uint16_t g_nodes[3] = {9, 11, 14};
    static const uint16_t i_nodes[2] = {9, 12};
    const uint16_t* ne = global_layout ? g_nodes : i_nodes;
    const int edges = global_layout ? 3 : 2;
    const uint8_t shape = shape_class(nodes, node_count, global_layout);
    uint8_t size = 0;
    for (int e = 0; e < edges; e++) {
        size += (uint16_t)node_count >= ne[e] ? 1 : 0;
    }
    const float fr = std::round(feet);
    int32_t fi = fr >= 2147483647.0f ? 2147483647 : (fr <= -2147483648.0f ? (-2147483647 - 1) : (int32_t)fr);
    fi = std::min(std::max(fi, 1), 5);
    uint8_t niche[6] = {qd_bin(gc, 0.0f, 1.0f, 6), qd_bin(gf, 0.0f, 6.0f, 8), shape,
                        qd_bin(height_axis(mh), 0.0f, 1.0f, 6), (uint8_t)(fi - 1), size};
    const uint8_t bins[6] = {6, 8, (uint8_t)(edges + 1), 6, 5, (uint8_t)(edges + 1)};
    if (niche_out) std::memcpy(niche_out, niche, 6);
    int64_t index = 0;
    for (int a = 0; a < 6; a++) {
        if (niche[a] >= bins[a]) return -1;
        index = index * bins[a] + niche[a];
    }
    return index;
}

extern "C" ce_status ce_to_metrics_batch(const ce_result* r, const uint32_t* node_counts, size_t n,
                                         const ce_world* w, ce_metrics* out) {
    if (!r || !node_counts || !w || !out) {
        set_error("ce_to_metrics_batch: null argument");
        return CE_ERR_INVALID;
    }
    for (size_t i = 0; i < n; i++) {
        const ce_status s = ce_to_metrics(r + i, node_counts[i], w, out + i);
        if (s != CE_OK) return s;
    }
    return CE_OK;
}

extern "C" ce_status ce_niche_batch(const ce_population* pop, const uint32_t* indices, size_t n,
                                    const ce_metrics* m, int global_layout, int64_t* cells) {
    if (!pop || !m || !cells) {
        set_error("ce_niche_batch: null argument");
        return CE_ERR_INVALID;
    }
#pragma omp parallel for schedule(static, 4096)
    for (long long k = 0; k < (long long)n; k++) {
        const size_t i = indices ? indices[k] : (size_t)k;
        const ce_genome& g = pop->genomes[i];
        cells[k] = ce_niche(pop->nodes + g.node_start, g.node_count, g.muscle_count, m + k, global_layout, nullptr);
    }
    return CE_OK;
}

static_assert(sizeof(ce_dump_head) == 32, "ce_dump_head is 32 bytes");

// storage::dump::Dump::write_rows (src/storage/dump.rs:409-455) for
// `count` results: the caller's heads, the behaviour cell (dump::cell,
// storage/dump.rs:151-158) of each result's niche, its fitness and its rung
// trace words.
extern "C" ce_status ce_dump_rows(const ce_result* results, const uint32_t* heads, const ce_dump_head* dump,
                                  const float* archive_fitness, size_t count, const ce_world* w, uint8_t* rows) {
    if (!results || !heads || !dump || !w || !rows) {
        set_error("ce_dump_rows: null argument");
        return CE_ERR_INVALID;
    }
    for (size_t c = 0; c < count; c++) {
        const ce_result& r = results[c];
        const ce_dump_head& h = dump[c];
        ce_metrics m;
        ce_status s = ce_to_metrics(&r, heads[8 * c] & 255u, w, &m);
        if (s != CE_OK) return s;
        const uint8_t gc = qd_bin(clampf(m.ground_contact, 0.0f, 1.0f), 0.0f, 1.0f, 6);
        const uint8_t gf = qd_bin(clampf(m.gait_frequency, 0.0f, 20.0f), 0.0f, 6.0f, 8);
        const uint8_t hb = qd_bin(height_axis(fmax_(m.mean_height, 0.0f)), 0.0f, 1.0f, 6);
        const float fr = std::round(fmax_(m.feet, 0.0f));
        int32_t fi = fr >= 2147483647.0f ? 2147483647 : (fr <= -2147483648.0f ? (-2147483647 - 1) : (int32_t)fr);
        fi = std::min(std::max(fi, 1), 5);
        const uint16_t cell = (uint16_t)(((gc * 8u + gf) * 6u + hb) * 5u + (uint32_t)(fi - 1));
        uint8_t* b = rows + (size_t)CE_DUMP_ROW_BYTES * c;
        auto put = [&](size_t at, const void* v, size_t n) { std::memcpy(b + at, v, n); };
        put(0, &h.slot, 4);
        b[4] = h.emitter;
        b[5] = (uint8_t)(h.op & 0xffu);
        b[6] = (uint8_t)(h.flags | (m.screened ? CE_DUMP_SCREENED : 0u));
        b[7] = (uint8_t)((h.kind & 15u) | (((h.op >> 8) & 15u) << 4));
        put(8, &h.parent, 8);
        put(16, &h.parent_cell, 2);
        put(18, &cell, 2);
        put(20, &h.cma, 2);
        b[22] = h.nodes;
        b[23] = h.muscles;
        b[24] = h.parent_nodes;
        b[25] = h.parent_muscles;
        put(26, &h.period, 2);
        put(28, &r.fitness, 4);
        const float archive = archive_fitness ? archive_fitness[c] : r.fitness;
        put(32, &archive, 4);
        const float words[7] = {r.contact_hi,        r.lift_hi,           r.ground_hi, r.previous_center_y,
                                r.vertical_extremum, r.vertical_trend,    r.gait_turns};
        put(36, words, 28);
    }
    return CE_OK;
}

extern "C" void ce_ground(float x, float amplitude, float tilt, float width, float hurdle, float phase, float* height,
                          float* slope) {
    float h = 0.0f, sl = 0.0f;
    ce::ground(x, amplitude, tilt, width, hurdle, phase, h, sl);
    if (height) *height = h;
    if (slope) *slope = sl;
}

extern "C" uint32_t ce_quake_hash(uint64_t id) { return ce::quake_hash(id); }

// -------------------------------------------------------------- gradients
// Record-field gradients (ce_backward) to gene gradients by the chain rule
// through the packing arithmetic of make_model and fill_creature:
//   amplitude = min(long - short, 2 * speed * period * min(duty, 1 - duty) / pi)
//   hill = 1 / (8 * max(long, 0.05)), cap = force * strength * scale,
//   1 / capacity = 1 / (energy * strength * scale), phase = frac(-t_on / period),
//   duty = clamp(frac((t_off - t_on) / period), 0.05, 0.95), node friction as is;
// and, for the long length, through the body's masses: a muscle weighs
// base + per_m * max(long, span), half on each of its two bones split
// between their ends by the anchor (body_nodes), and the masses reach the
// kernel (the record gradient's mass rows), the muscles' strengths
// min(200 * driven / force, 1) / share, `driven` the lighter subtree mass,
// and the start pose, which is moved by minus the centre of mass's x.
// The gene-level parameters are, per muscle, (short, long, strength scale,
// on time, off time) with the period fixed, and per node its friction.
extern "C" ce_status ce_gene_gradients(const ce_population* pop, const uint32_t* indices, size_t n,
                                       const ce_world* world, const uint32_t* slots, const float* grads,
                                       uint32_t rows, uint32_t mm, double* muscle_grads, double* node_grads) {
    if (!pop || !world || !slots || !grads || !muscle_grads || !node_grads) {
        set_error("ce_gene_gradients: null argument");
        return CE_ERR_INVALID;
    }
    const size_t per = (size_t)9 * mm + 4 * (size_t)rows;
    for (size_t c = 0; c < n; c++) {
        const size_t i = indices ? indices[slots[c]] : slots[c];
        const ce_genome& gm = pop->genomes[i];
        if (gm.node_count > rows || gm.muscle_count > mm) {
            set_error("ce_gene_gradients: creature larger than the gradient rows");
            return CE_ERR_INVALID;
        }
        gene_gradients_one(*pop, (uint32_t)i, *world, grads + c * per, rows, mm, muscle_grads, node_grads,
                           HostAngle{}, HostTrig{});
    }
    return CE_OK;
}

// ------------------------------------------------------------------ replay
// engine::recorded (src/engine.rs:1062-1127): the frames of one recorded
// creature (ce_record's layout, `stride` float2 slots a frame, kernel node
// rows first) in the creature's own node numbering (row 0 is node 0, row
// j + 1 is bone j's far node), and, when the frames carry them, the forces:
// each muscle's energy store and pull, each node's ground and friction force,
// and the broken-joint bits.
extern "C" ce_status ce_replay_decode(const ce_bone_gene* bones, uint32_t node_count, uint32_t muscles,
                                      const float* frames, uint32_t count, uint32_t stride, float* positions,
                                      float* energy, float* pull, float* ground, float* friction,
                                      uint64_t* broken) {
    if (!bones || !frames || !positions || node_count < 1 || node_count > CE_MAX_NODES) {
        set_error("ce_replay_decode: null argument or bad node count");
        return CE_ERR_INVALID;
    }
    if (stride < node_count) {
        set_error("ce_replay_decode: frames narrower than the body");
        return CE_ERR_INVALID;
    }
    std::vector<uint32_t> order(node_count);
    order[0] = 0;
    for (uint32_t j = 0; j + 1 < node_count; j++) {
        if (bones[j].b >= node_count) {
            set_error("ce_replay_decode: bone end outside the body");
            return CE_ERR_INVALID;
        }
        order[j + 1] = bones[j].b;
    }
    const uint32_t capacity = CE_MAX_NODES;
    const bool forces = stride > capacity + muscles + node_count;
    if ((energy || pull || ground || friction || broken) && !forces) {
        set_error("ce_replay_decode: the frames carry no forces");
        return CE_ERR_INVALID;
    }
    for (uint32_t t = 0; t < count; t++) {
        const float* f = frames + (size_t)t * stride * 2;
        for (uint32_t k = 0; k < node_count; k++) {
            positions[((size_t)t * node_count + order[k]) * 2] = f[2 * k];
            positions[((size_t)t * node_count + order[k]) * 2 + 1] = f[2 * k + 1];
        }
        if (!forces) continue;
        const float* slot = f + 2 * capacity;
        for (uint32_t m = 0; m < muscles; m++) {
            if (energy) energy[(size_t)t * muscles + m] = slot[2 * m];
            if (pull) pull[(size_t)t * muscles + m] = slot[2 * m + 1];
        }
        for (uint32_t k = 0; k < node_count; k++) {
            if (ground) ground[(size_t)t * node_count + order[k]] = slot[2 * (muscles + k)];
            if (friction) friction[(size_t)t * node_count + order[k]] = slot[2 * (muscles + k) + 1];
        }
        if (broken) {
            uint32_t lo, hi;
            std::memcpy(&lo, f + 2 * (stride - 1), 4);
            std::memcpy(&hi, f + 2 * (stride - 1) + 1, 4);
            broken[t] = (uint64_t)lo | ((uint64_t)hi << 32);
        }
    }
    return CE_OK;
}

// --------------------------------------------------- metrics on the device
// Shape classes of a packed batch (packed order), for the device epilogue.
extern "C" ce_status ce_shape_classes(const ce_population* pop, const uint32_t* indices, size_t n,
                                      const uint32_t* slots, int global_layout, uint8_t* out) {
    if (!pop || !slots || !out) {
        set_error("ce_shape_classes: null argument");
        return CE_ERR_INVALID;
    }
    for (size_t c = 0; c < n; c++) {
        const size_t i = indices ? indices[slots[c]] : slots[c];
        const ce_genome& g = pop->genomes[i];
        out[c] = shape_class(pop->nodes + g.node_start, g.node_count, global_layout);
    }
    return CE_OK;
}

namespace ce {
// The mean heights where the niche's height bin steps up: bin(h) is the
// number of thresholds at or below h. The bin is monotone in h, so the
// smallest float reaching each bin, found by bisection over the float bits
// with the host's own arithmetic, reproduces it exactly.
void height_bin_thresholds(float out[5]) {
    auto bin = [](float h) { return qd_bin(height_axis(fmax_(h, 0.0f)), 0.0f, 1.0f, 6); };
    const uint32_t inf_bits = 0x7f800000u;
    for (int b = 1; b <= 5; b++) {
        uint32_t lo = 0, hi = inf_bits;  // bin(lo) < b <= bin(hi), or none
        float v;
        if (bin(std::numeric_limits<float>::max()) < b) {
            out[b - 1] = std::numeric_limits<float>::infinity();
            continue;
        }
        hi = 0x7f7fffffu;
        if (bin(0.0f) >= b) {
            out[b - 1] = 0.0f;
            continue;
        }
        while (hi - lo > 1) {
            const uint32_t mid = lo + (hi - lo) / 2;
            std::memcpy(&v, &mid, 4);
            if (bin(v) >= b) hi = mid; else lo = mid;
        }
        std::memcpy(&out[b - 1], &hi, 4);
    }
}
}  // namespace ce
