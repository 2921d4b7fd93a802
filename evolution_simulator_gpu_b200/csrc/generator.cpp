// Seeded synthetic creature populations.
//
// The reference benchmarks on saved populations that are not available, so
// the engine's workloads are generated: every creature is a function of
// (seed, creature index) alone, drawn from a counter-based stream (the
// SplitMix64 finaliser of Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014, applied to a keyed
// counter). The bodies follow the reference's conventions for a repaired
// creature: node 0 is the head and the highest node, the head sits on one
// neck bone (src/evolution.rs:1198-1227), and bones are in parent-first
// order with bone j ending at node j + 1 (src/evolution.rs:942-1042). Bone
// lengths are the node distances clamped to [0.03, 2] m
// (src/evolution.rs:1045-1054).
//
// Muscles: one per joint between the parent bone and the bone, anchored at
// the two ends away from the shared node (the node pair two hops apart),
// plus extra muscles between bones touching two random nodes, anchored at
// those nodes. Lengths are drawn relative to the anchor distance d: short
// c*d with c ~ U(0.8, 1), long e*d with e ~ U(1, 1.3). A rhythm of period
// T ~ U(0.5, 1.5) s switches on at t_on and off at t_off, both U(0, T):
// phase = frac(-t_on / T) and duty = clamp(frac((t_off - t_on) / T), 0.05,
// 0.95) (the clamp of src/evolution.rs:1316-1320). A strength factor
// U(0.5, 1.5) scales the force cap and the energy store. Stiffness is 90,
// no tendon, no sensor. Creature ids are first_id + index.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/creature_engine.h"
#include "host_model.h"

namespace {

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// A stream of uniform draws for one creature.
struct Stream {
    uint64_t key;
    uint64_t n = 0;
    Stream(uint64_t seed, uint64_t index) {
        key = mix64(seed * 0x9e3779b97f4a7c15ull + 0x2545f4914f6cdd1dull);
        key = mix64(key ^ (index + 1) * 0xd1342543de82ef95ull);
    }
    uint64_t next() { return mix64(key + (++n) * 0x9e3779b97f4a7c15ull); }
    // Uniform in [0, 1) with 24 random bits.
    float unit() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
    float range(float lo, float hi) { return lo + (hi - lo) * unit(); }
    uint32_t below(uint32_t n_) { return (uint32_t)((next() >> 32) * (uint64_t)n_ >> 32); }
    uint32_t between(uint32_t lo, uint32_t hi) { return lo + below(hi - lo + 1); }
};

float frac(float x) { return x - std::floor(x); }

struct Body {
    std::vector<ce_node_gene> nodes;
    std::vector<ce_bone_gene> bones;
    std::vector<ce_muscle_gene> muscles;
    std::vector<float> strength;
};

uint32_t draw_nodes(const ce_gen_spec& s, Stream& r) {
    const uint32_t lo = std::max(s.min_nodes, 3u), hi = std::min(std::max(s.max_nodes, lo), 32u);
    if (s.node_dist == 1) {
        // Geometric on lo, lo+1, ... with the given mean, clipped to hi.
        const float excess = std::max(s.mean_nodes - (float)lo, 0.0f);
        const float p = 1.0f / (excess + 1.0f);
        uint32_t k = 0;
        while (k < hi - lo && r.unit() >= p) k++;
        return lo + k;
    }
    return r.between(lo, hi);
}

// The muscle gene between bones ba and bb anchored at aa and ab, with the
// rhythm and lengths drawn from the stream.
void add_muscle(Body& b, Stream& r, uint32_t ba, uint32_t bb, float aa, float ab) {
    auto point = [&](uint32_t bone, float t, float out[2]) {
        const ce_node_gene& p = b.nodes[b.bones[bone].a];
        const ce_node_gene& q = b.nodes[b.bones[bone].b];
        out[0] = p.x + (q.x - p.x) * t;
        out[1] = p.y + (q.y - p.y) * t;
    };
    float p[2], q[2];
    point(ba, aa, p);
    point(bb, ab, q);
    const float d = std::max(std::hypot(p[0] - q[0], p[1] - q[1]), 0.01f);
    ce_muscle_gene m{};
    m.bone_a = ba;
    m.bone_b = bb;
    m.anchor_a = aa;
    m.anchor_b = ab;
    m.short_len = r.range(0.8f, 1.0f) * d;
    m.long_len = r.range(1.0f, 1.3f) * d;
    m.period = r.range(0.5f, 1.5f);
    const float t_on = r.unit() * m.period;
    const float t_off = r.unit() * m.period;
    m.phase = frac(-t_on / m.period);
    m.duty = std::min(std::max(frac((t_off - t_on) / m.period), 0.05f), 0.95f);
    m.stiffness = 90.0f;
    m.sensor = CE_NO_SENSOR;
    m.reset = 0.0f;
    m.tendon = 0.0f;
    b.muscles.push_back(m);
    b.strength.push_back(r.range(0.5f, 1.5f));
}

Body make_body(const ce_gen_spec& s, uint64_t index) {
    Stream r(s.seed, index);
    Body b;
    const uint32_t n = draw_nodes(s, r);
    b.nodes.resize(n);
    for (auto& g : b.nodes) {
        g.x = r.range(-0.5f, 0.5f);
        g.y = r.range(0.0f, 1.0f);
        g.diameter = r.range(0.06f, 0.12f);
        g.friction = r.range(s.friction_lo, s.friction_hi);
    }
    // The highest node becomes the head.
    uint32_t top = 0;
    for (uint32_t i = 1; i < n; i++) {
        if (b.nodes[i].y > b.nodes[top].y) top = i;
    }
    std::swap(b.nodes[0], b.nodes[top]);
    b.nodes[0].diameter = 0.12f;
    // A random tree: node 1 hangs from the head (the neck), node i >= 2 from
    // a node in 1 .. i-1, so bone j = i - 1 joins parent(i) to i.
    const float lo_deg = s.joint_lo_deg, hi_deg = s.joint_hi_deg;
    for (uint32_t i = 1; i < n; i++) {
        const uint32_t parent = i == 1 ? 0u : 1u + r.below(i - 1);
        const ce_node_gene& p = b.nodes[parent];
        const ce_node_gene& q = b.nodes[i];
        ce_bone_gene bone{};
        bone.a = parent;
        bone.b = i;
        bone.rest_length = std::min(std::max(std::hypot(q.x - p.x, q.y - p.y), 0.03f), 2.0f);
        const float half = (hi_deg > lo_deg ? r.range(lo_deg, hi_deg) : lo_deg) * (3.14159265358979f / 180.0f);
        bone.min_angle = -half;
        bone.max_angle = half;
        bone.organ_mass = 0.0f;
        bone.organ_at = 0.5f;
        b.bones.push_back(bone);
    }
    // The spanning muscles, one per joint (every bone but the neck turns
    // against the bone that ends at its pivot).
    std::vector<uint32_t> span_a, span_b;
    std::vector<float> span_aa;
    for (uint32_t j = 1; j + 1 < n; j++) {
        const uint32_t hub = b.bones[j].a;
        const uint32_t p = hub - 1;  // the bone that ends at `hub`
        span_a.push_back(p);
        span_b.push_back(j);
        span_aa.push_back(b.bones[p].a == hub ? 1.0f : 0.0f);
    }
    uint32_t spanning = (uint32_t)span_a.size();
    uint32_t extras;
    if (s.muscle_rule == 1) {
        const uint32_t target = r.between(std::max(s.min_muscles, 1u), std::max(s.max_muscles, s.min_muscles));
        spanning = std::min(spanning, target);
        extras = target - spanning;
    } else {
        extras = r.between(0, s.max_extra);
    }
    for (uint32_t k = 0; k < spanning; k++) add_muscle(b, r, span_a[k], span_b[k], span_aa[k], 1.0f);
    // Extra muscles between bones at two distinct random nodes.
    std::vector<std::vector<uint32_t>> incident(n);
    for (uint32_t j = 0; j + 1 < n; j++) {
        incident[b.bones[j].a].push_back(j);
        incident[b.bones[j].b].push_back(j);
    }
    for (uint32_t e = 0; e < extras; e++) {
        bool placed = false;
        for (int attempt = 0; attempt < 16 && !placed; attempt++) {
            const uint32_t u = r.below(n);
            uint32_t v = r.below(n - 1);
            if (v >= u) v++;
            const uint32_t ba = incident[u][r.below((uint32_t)incident[u].size())];
            const uint32_t bb = incident[v][r.below((uint32_t)incident[v].size())];
            if (ba == bb) continue;
            add_muscle(b, r, ba, bb, b.bones[ba].a == u ? 0.0f : 1.0f, b.bones[bb].a == v ? 0.0f : 1.0f);
            placed = true;
        }
        if (!placed) {
            // A body of three nodes always has two bones at node 1.
            add_muscle(b, r, 0, 1, 0.0f, 1.0f);
        }
    }
    if (b.muscles.size() > CE_MAX_MUSCLES) {
        b.muscles.resize(CE_MAX_MUSCLES);
        b.strength.resize(CE_MAX_MUSCLES);
    }
    return b;
}

}  // namespace

extern "C" ce_status ce_generate_size(const ce_gen_spec* spec, size_t first, size_t count, size_t* nodes,
                                      size_t* bones, size_t* muscles) {
    if (!spec || !nodes || !bones || !muscles) {
        ce::set_error("ce_generate_size: null argument");
        return CE_ERR_INVALID;
    }
    size_t nn = 0, nb = 0, nm = 0;
#pragma omp parallel for reduction(+ : nn, nb, nm) schedule(dynamic, 1024)
    for (long long i = 0; i < (long long)count; i++) {
        const Body b = make_body(*spec, first + (uint64_t)i);
        nn += b.nodes.size();
        nb += b.bones.size();
        nm += b.muscles.size();
    }
    *nodes = nn;
    *bones = nb;
    *muscles = nm;
    return CE_OK;
}

extern "C" ce_status ce_generate(const ce_gen_spec* spec, size_t first, size_t count, ce_node_gene* nodes,
                                 ce_bone_gene* bones, ce_muscle_gene* muscles, float* strength_scale,
                                 ce_genome* genomes) {
    if (!spec || !nodes || !bones || !muscles || !genomes) {
        ce::set_error("ce_generate: null argument");
        return CE_ERR_INVALID;
    }
    std::vector<Body> all(count);
#pragma omp parallel for schedule(dynamic, 1024)
    for (long long i = 0; i < (long long)count; i++) all[i] = make_body(*spec, first + (uint64_t)i);
    size_t an = 0, ab = 0, am = 0;
    for (size_t i = 0; i < count; i++) {
        const Body& b = all[i];
        ce_genome g{};
        g.node_start = (uint32_t)an;
        g.node_count = (uint32_t)b.nodes.size();
        g.bone_start = (uint32_t)ab;
        g.bone_count = (uint32_t)b.bones.size();
        g.muscle_start = (uint32_t)am;
        g.muscle_count = (uint32_t)b.muscles.size();
        g.id = spec->first_id + first + i;
        g.flags = 0;
        genomes[i] = g;
        std::copy(b.nodes.begin(), b.nodes.end(), nodes + an);
        std::copy(b.bones.begin(), b.bones.end(), bones + ab);
        std::copy(b.muscles.begin(), b.muscles.end(), muscles + am);
        if (strength_scale) std::copy(b.strength.begin(), b.strength.end(), strength_scale + am);
        an += b.nodes.size();
        ab += b.bones.size();
        am += b.muscles.size();
    }
    return CE_OK;
}
