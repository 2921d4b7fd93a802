/*
 * creature_engine.h -- C ABI of the B200 creature-evaluation engine.
 *
 * The engine runs whole creature trials (the position-based-dynamics substep
 * loop, its per-step tallies, the early rungs and the screen) on an sm_100a
 * GPU and returns one result record per creature. It replaces the CUDA
 * backend and engine thread of the evolution simulator:
 *
 *   reference (Rust)                                   this header
 *   ----------------------------------------------------------------------
 *   shaders/creature.cu:1266-1277  advance(...)        ce_advance_device
 *   src/cuda_engine.rs:2106-2316   CudaEngine::launch  ce_submit
 *   src/cuda_engine.rs:2319-2393   CudaEngine::poll    ce_poll
 *   src/cuda_engine.rs:2054-2100   CudaEngine::record  ce_record
 *   src/engine.rs:163-199          trait Engine        ce_open/ce_submit/
 *                                                      ce_poll/ce_wait/
 *                                                      ce_free_slots/
 *                                                      ce_allocated_bytes
 *   src/engine.rs:430-469          trait Device        ce_release_idle
 *   src/kernel.rs:471-593          pack_reusing        ce_pack
 *   src/kernel.rs:212-251          params              ce_make_params
 *   src/kernel.rs:82-106           world_flags         ce_world_flags
 *   src/scheduler.rs:859-923       trial_steps/to_metrics  ce_to_metrics
 *   src/qd.rs:762-846, 988-999     descriptor/niche_in/cell_index ce_niche
 *
 * Every struct below that the reference also defines has the reference's
 * field order and size, so the reference's #[repr(C)] buffers (WavePack
 * words, Params, GpuResult, NodeGene, Bone, Muscle) pass through unchanged.
 *
 * Errors: every entry point returns a ce_status. CE_ERR_OOM is the
 * out-of-memory case the reference's MemoryBackoff retries
 * (src/cuda_engine.rs:425-448, src/engine.rs:534-650); CE_ERR_DEVICE means
 * the engine must be closed and opened again (src/scheduler.rs:742-806).
 * ce_last_error() gives a thread-local message for the last failure.
 *
 * Threading: one handle per GPU, used from one thread at a time, like the
 * reference's engine thread (src/engine.rs:656-719).
 */
#ifndef CREATURE_ENGINE_H
#define CREATURE_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum ce_status {
    CE_OK = 0,
    CE_ERR_INVALID = 1,     /* bad argument, unsupported body or size      */
    CE_ERR_OOM = 2,         /* device or pinned memory exhausted           */
    CE_ERR_TIMEOUT = 3,     /* nothing finished within the timeout         */
    CE_ERR_DEVICE = 4,      /* CUDA failure: close and reopen the engine   */
    CE_ERR_UNSUPPORTED = 5, /* no kernel for this request                  */
    CE_ERR_BUSY = 6         /* no free slot for another submission         */
} ce_status;

/* ---- layout constants (src/kernel.rs:24-51) ---------------------------- */
#define CE_MAX_NODES 32
#define CE_MAX_MUSCLES 96
#define CE_NODE_WORDS 6
#define CE_BONE_WORDS 6
#define CE_MUSCLE_FIELDS 20
#define CE_SUBSTEPS 16
#define CE_WAVE 262144
#define CE_NO_SENSOR 255u   /* src/evolution.rs:247 */
#define CE_NONE 0xffffffffu /* no parent bone / no sensor in the records */

/* World effect bits of ce_world_flags (src/kernel.rs:82-113). */
#define CE_FLAG_GROUND (1u << 0)
#define CE_FLAG_TERRAIN (1u << 1)
#define CE_FLAG_SLOPE (1u << 2)
#define CE_FLAG_GAPS (1u << 3)
#define CE_FLAG_HURDLES (1u << 4)
#define CE_FLAG_QUAKE (1u << 5)
#define CE_FLAG_MUD (1u << 6)
#define CE_FLAG_WATER (1u << 7)
#define CE_FLAG_ICE (1u << 8)
#define CE_FLAG_WIND (1u << 9)
#define CE_FLAG_AIR (1u << 10)
#define CE_FLAG_BRAMBLES (1u << 11)

/* ---- genes (src/evolution.rs:41-50, 58-80, 209-243) -------------------- */
typedef struct ce_node_gene {
    float x, y, diameter, friction;
} ce_node_gene;

typedef struct ce_bone_gene {
    uint32_t a, b;
    float rest_length, min_angle, max_angle, organ_mass, organ_at;
} ce_bone_gene;

typedef struct ce_muscle_gene {
    uint32_t bone_a, bone_b;
    float anchor_a, anchor_b;
    float short_len, long_len; /* `short` and `long` in the reference */
    float period, phase, duty, stiffness;
    uint32_t sensor;
    float reset, tendon;
} ce_muscle_gene;

/* One creature of an arena-packed population (src/evolution.rs:254-269,
 * 440-453): the ranges of its genes in the three gene arrays and its id. */
typedef struct ce_genome {
    uint32_t node_start, node_count;
    uint32_t bone_start, bone_count;
    uint32_t muscle_start, muscle_count;
    uint64_t id;
    uint32_t flags; /* rungs::AUDIT and the others (src/rungs.rs:18-35) */
    uint32_t reserved;
} ce_genome;

typedef struct ce_population {
    const ce_node_gene* nodes;
    const ce_bone_gene* bones;
    const ce_muscle_gene* muscles;
    const ce_genome* genomes;
    size_t count;
    /* Optional factor on each muscle's strength (one per muscle gene, NULL
     * for 1): it multiplies the force cap and the energy store, as the
     * reference's `muscle_scale` does (src/kernel.rs:376, 390-391). */
    const float* strength_scale;
} ce_population;

/* ---- world (the physics subset of src/config.rs:119-161) --------------- */
typedef struct ce_rung {
    float w[6];
    float bias;
    uint32_t off;
} ce_rung; /* rungs::Rung, shaders/creature.cu:66-70 */

typedef struct ce_world {
    uint32_t ground;    /* bool */
    uint32_t terrain;   /* roughness level, 0..4 (physics.rs:523-527) */
    float gravity, air_retention, ground_friction;
    float muscle_energy, muscle_recovery;
    float slope, wind, mud, brambles, water, patches, gaps, hurdles, quake;
    float duration;     /* seconds */
    uint32_t rate;      /* steps per second: 60 standard, 120 fine */
    uint32_t has_screen;
    float screen_seconds, screen_bar, screen_bar_young, screen_bar_reshaped;
    uint32_t has_rungs;
    ce_rung rungs[2];
} ce_world;

/* ---- kernel ABI (shaders/creature.cu:75-128) --------------------------- */
typedef struct ce_params {
    uint32_t count, base, steps, screen_step, stride;
    float gravity, air, friction, terrain, muscle_energy, muscle_recovery;
    float slope, wind, mud, gaps, hurdles, quake;
    float screen_bar, screen_bar_young, screen_bar_reshaped;
    float water, patches, air_sub, inv_muscle_energy, brambles;
    ce_rung r1, r2;
} ce_params;

typedef struct ce_result {
    float fitness, ground_contact, vertical_oscillation, gait_frequency;
    float previous_center_y, vertical_extremum, vertical_trend, gait_turns;
    float height_sum, contact_lo, contact_hi, lift_lo, lift_hi;
    float ground_lo, ground_hi, fall_time, head_shake, screen_x, screened;
} ce_result;

/* The packed records of a batch (src/kernel.rs:56-72): node and bone words,
 * muscle records and two head words (uint32_t[4] each) per creature, in
 * packed order, which is sorted by (muscles, nodes, population index). */
typedef struct ce_wave_pack {
    const uint32_t* lanes;
    size_t lanes_len; /* words */
    const float* muscles;
    size_t muscles_len; /* floats */
    const uint32_t* heads; /* 8 words per creature */
    size_t count;          /* creatures */
} ce_wave_pack;

/* ---- packing (host) ---------------------------------------------------- */
/* The world's effect bits (src/kernel.rs:82-106). */
uint32_t ce_world_flags(const ce_world* world);

/* The launch parameters of a wave (src/kernel.rs:212-251). */
ce_status ce_make_params(const ce_world* world, uint32_t base, uint32_t count, uint32_t stride,
                         ce_params* out);

/* Sizes of the packed records of `indices` (NULL: every creature). */
ce_status ce_pack_size(const ce_population* pop, const uint32_t* indices, size_t n,
                       size_t* lanes_len, size_t* muscles_len);

/* Packs creatures into caller buffers sized by ce_pack_size
 * (src/kernel.rs:336-411, 471-593). `slots` receives, for each packed
 * creature, its position in `indices`. `info` (optional, 4 words per
 * creature) receives node, bone, muscle count and quake hash. */
ce_status ce_pack(const ce_population* pop, const uint32_t* indices, size_t n, const ce_world* world,
                  uint32_t* lanes, float* muscles, uint32_t* heads, uint32_t* slots, uint32_t* info);

/* The host half of packing on the device (the same records as ce_pack,
 * src/kernel.rs:336-411, 471-593). For the `n` creatures of `indices`
 * (NULL: every creature) it writes the packed order (`order[c]`: the
 * population index of packed creature c), each packed creature's record
 * and muscle offsets (`record_at`, `muscle_at`, n each), and, for every
 * bone gene of those creatures, three floats at 3 * (bone_start + j): the
 * bone's gene-pose direction and the sine and cosine of its start-pose
 * angle, from the C library's single-precision functions as the reference's
 * Rust host calls them (physics2::Model::new / start, src/physics2.rs:190-399).
 * `trig` holds 3 * bones_len floats. The plan depends on node and bone genes
 * only: a batch whose muscle genes or frictions change keeps its plan. */
ce_status ce_pack_plan(const ce_population* pop, const uint32_t* indices, size_t n, const ce_world* world,
                       size_t bones_len, uint32_t* order, uint32_t* record_at, uint32_t* muscle_at, float* trig);

/* Packs on the device, one creature a thread, from a plan of ce_pack_plan:
 * `pop` holds device pointers (genes, optional strength scale), `trig`,
 * `order`, `record_at`, `muscle_at` are device copies of the plan, and
 * `lanes`, `muscles`, `heads` (sized as ce_pack_size gives) receive the
 * records, equal to ce_pack's byte for byte. Asynchronous on `stream`.
 * Replaces kernel::pack_reusing's fill (src/kernel.rs:529-567), which the
 * reference runs on host threads. */
ce_status ce_pack_device(const ce_population* pop, const float* trig, const uint32_t* order,
                         const uint32_t* record_at, const uint32_t* muscle_at, size_t n, const ce_world* world,
                         uint32_t* lanes, float* muscles, uint32_t* heads, void* stream);

/* The ground's height and slope under x for bump height `amplitude`, slope
 * `tilt`, pit width `width`, hurdle height `hurdle` and quake phase `phase`
 * (physics::ground, src/physics.rs:668-683), as the packer places creatures
 * on it. */
void ce_ground(float x, float amplitude, float tilt, float width, float hurdle, float phase,
               float* height, float* slope);
/* The quake hash of a creature id (physics::quake_hash, src/physics.rs:640-648). */
uint32_t ce_quake_hash(uint64_t id);

/* One recorded creature's frames (count frames of `stride` float2 slots, as
 * ce_record writes them) in the creature's own node numbering
 * (engine::recorded, src/engine.rs:1062-1127): positions[count][nodes][2];
 * with forces in the frames, energy[count][muscles], pull[count][muscles],
 * ground[count][nodes], friction[count][nodes] and broken[count] (each NULL
 * to skip). `bones` are the creature's bone genes in canonical order. */
ce_status ce_replay_decode(const ce_bone_gene* bones, uint32_t node_count, uint32_t muscles,
                           const float* frames, uint32_t count, uint32_t stride, float* positions,
                           float* energy, float* pull, float* ground, float* friction, uint64_t* broken);

/* Frame slots of a recording (src/creature_kernel.rs:312-326). */
uint32_t ce_frame_stride(uint32_t max_muscles);

/* ---- synthetic population generator ------------------------------------ */
typedef struct ce_gen_spec {
    uint64_t seed;
    uint32_t min_nodes, max_nodes;
    uint32_t node_dist;      /* 0 uniform, 1 geometric with mean `mean_nodes` */
    float mean_nodes;
    uint32_t min_muscles, max_muscles;
    uint32_t muscle_rule;    /* 0 spanning + up to `max_extra` extras,
                                1 muscle count uniform in [min, max]        */
    uint32_t max_extra;
    float joint_lo_deg, joint_hi_deg; /* joint half-range drawn uniformly */
    float friction_lo, friction_hi;
    uint64_t first_id;
} ce_gen_spec;

/* Counts of the genes that ce_generate writes for creatures
 * [first, first + count). */
ce_status ce_generate_size(const ce_gen_spec* spec, size_t first, size_t count, size_t* nodes,
                           size_t* bones, size_t* muscles);
/* Writes `count` creatures: creature i is a function of (seed, first + i). */
ce_status ce_generate(const ce_gen_spec* spec, size_t first, size_t count, ce_node_gene* nodes,
                      ce_bone_gene* bones, ce_muscle_gene* muscles, float* strength_scale,
                      ce_genome* genomes);

/* ---- metrics (host) ---------------------------------------------------- */
typedef struct ce_metrics {
    float fitness, ground_contact, vertical_oscillation, gait_frequency, mean_height, feet;
    float screen_x;
    uint32_t screened, steps;
} ce_metrics;

/* The metrics epilogue on the device: ce_to_metrics and the dense cell of
 * ce_niche for `count` results (device pointers: results, heads of the
 * packed batch, shape classes from ce_shape_classes; `metrics` may be NULL),
 * equal to the host's to the bit; asynchronous on `stream` (a cudaStream_t).
 * No counterpart in the reference, which does this on the host
 * (src/scheduler.rs:890-923, src/qd.rs:762-999). */
ce_status ce_metrics_device(const ce_result* results, const uint32_t* heads, const uint8_t* shape_classes,
                            size_t count, const ce_world* world, int global_layout, ce_metrics* metrics,
                            int64_t* cells, void* stream);
/* ---- generation dump rows (src/storage/dump.rs) ---- */
/* One row a creature, 64 bytes little endian, in the layout of
 * storage/dump.rs:76-113 (ROW_BYTES): the breeding fields the caller knows
 * (ce_dump_head), the behaviour cell of the result
 * (((contact * 8 + cadence) * 6 + height) * 5 + feet, dump::cell), the
 * standard fitness, the archive fitness and the seven rung trace words of
 * the result (GpuResult::rung_trace). The row's flags byte is the head's
 * with CE_DUMP_SCREENED added when the screen stopped the trial
 * (write_rows, storage/dump.rs:409-455). */
#define CE_DUMP_ROW_BYTES 64u
#define CE_DUMP_FINE 4u
#define CE_DUMP_RERUN 8u
#define CE_DUMP_SCREENED 16u
#define CE_DUMP_EXCLUDED 32u
#define CE_DUMP_PARENT_RESERVE 64u
typedef struct ce_dump_head {
    uint64_t parent;         /* parent id, UINT64_MAX for none */
    uint32_t slot;           /* ring slot */
    uint16_t op;             /* structural operator index (12 bits), 0xFFF for none */
    uint16_t parent_cell;    /* parent's cell, UINT16_MAX for none */
    uint16_t cma;            /* CMA emitter that sampled it, UINT16_MAX for none */
    uint16_t period;         /* rhythm period of its first muscle, f16 bits */
    uint8_t emitter;         /* Emitter::index */
    uint8_t flags;           /* bred flags, with FINE, RERUN, EXCLUDED as the caller's metrics say */
    uint8_t kind;            /* where the result entered (low four bits) */
    uint8_t nodes, muscles, parent_nodes, parent_muscles;
    uint8_t reserved;
} ce_dump_head;
/* Host rows of `count` results (packed order; `heads` the packed batch's
 * heads for the node counts; `archive_fitness` NULL for the results'). */
ce_status ce_dump_rows(const ce_result* results, const uint32_t* heads, const ce_dump_head* dump,
                       const float* archive_fitness, size_t count, const ce_world* world, uint8_t* rows);
/* The same on the device (device pointers, `rows` 16-byte aligned),
 * asynchronous on `stream`; equal to ce_dump_rows to the byte. No
 * counterpart in the reference, which writes the rows on the host. */
ce_status ce_dump_rows_device(const ce_result* results, const uint32_t* heads, const ce_dump_head* dump,
                              const float* archive_fitness, size_t count, const ce_world* world, uint8_t* rows,
                              void* stream);

/* ---- samples of parent genomes (the refined search's ask step) ---- */
/* Sample g is a child of parent g mod P with every coordinate of the
 * optimizer's parameter vector of its body (src/qd.rs:2700-2770) moved by
 * sigma x N(0, 1) and put back with apply_parameters' clamps
 * (src/qd.rs:2773-2811), diameter and friction held to the workloads'
 * ranges; its id is first_id + g, its strength factors its parent's. The
 * deviates come from a counter-based hash of (seed, g, gene, field), so a
 * sample does not depend on the range a call draws. No counterpart in the
 * reference, which samples on the host. ce_sample_rows gives the rows of
 * samples [first, first + count) from the parents' (host) genomes (at most
 * 2^32 - 1 rows of a kind a call: the samples' gene starts are 32-bit);
 * ce_sample_device writes them (device pointers; the parents' genes packed
 * in order from row 0; `strength` may be NULL), asynchronous on `stream`
 * after a small synchronous read of the parents' genomes. */
ce_status ce_sample_rows(const ce_genome* parent_genomes, size_t parents, uint64_t first, size_t count,
                         size_t* nodes, size_t* bones, size_t* muscles);
ce_status ce_sample_device(const ce_population* parents, uint64_t first, size_t count, float sigma, uint64_t seed,
                           uint64_t first_id, ce_node_gene* nodes, ce_bone_gene* bones, ce_muscle_gene* muscles,
                           float* strength, ce_genome* genomes, void* stream);

/* Shape classes (the niche's aspect axis, from the genes) of a batch packed
 * by ce_pack(pop, indices, n, ..., slots, ...), in packed order. */
ce_status ce_shape_classes(const ce_population* pop, const uint32_t* indices, size_t n, const uint32_t* slots,
                           int global_layout, uint8_t* out);
/* The five mean heights where the niche's height bin steps up. */
void ce_height_bin_edges(float out[5]);

/* scheduler::to_metrics for one result (src/scheduler.rs:859-923). */
ce_status ce_to_metrics(const ce_result* r, uint32_t node_count, const ce_world* world,
                        ce_metrics* out);
/* ce_to_metrics for n results; node_counts[i] is result i's node count. */
ce_status ce_to_metrics_batch(const ce_result* r, const uint32_t* node_counts, size_t n,
                              const ce_world* world, ce_metrics* out);
/* ce_niche for creature indices[i] of `pop` with metrics m[i] (indices NULL:
 * creature i); cells[i] receives the dense cell or -1. */
ce_status ce_niche_batch(const ce_population* pop, const uint32_t* indices, size_t n,
                         const ce_metrics* m, int global_layout, int64_t* cells);
/* qd::descriptor + Descriptor::niche_in + cell_index (src/qd.rs:762-846,
 * 988-999): the dense cell of a creature in the global (global != 0) or
 * island layout, -1 outside the grid. */
int64_t ce_niche(const ce_node_gene* nodes, uint32_t node_count, uint32_t muscle_count,
                 const ce_metrics* m, int global_layout, uint8_t niche_out[6]);

/* ---- CMA-ES emitters on the device ---- */
/* One emitter per template body: the reference's CmaEmitter (src/qd.rs:
 * 2130-2188), which the reference keeps on the host, in either of its modes:
 * a separable CMA-ES optimizer (CmaEmitter::optimizer: the parameter vector
 * of write_parameters, src/qd.rs:2734-2770, in physical units) or a CMA-ME
 * emitter (CmaEmitter::new: exploring_parameters, src/qd.rs:2504-2538,
 * normalised to about 0-1). Every pointer is a device address. `templates`
 * holds one template body an emitter (count = emitters, genes packed in
 * order from row 0); emitter e's coordinates are [offsets[e], offsets[e + 1])
 * of mean, covariance, path_c and path_sigma, and sigma[e] is its step
 * size. */
typedef struct ce_cma {
    ce_population templates;
    const uint8_t* exploring; /* 1 a CMA-ME emitter, 0 an optimizer, one an emitter; NULL: all optimizers */
    const uint64_t* offsets;  /* emitters + 1 entries (ce_cma_offsets) */
    float* mean;
    float* covariance;
    float* path_c;
    float* path_sigma;
    float* sigma;             /* one an emitter */
} ce_cma;
/* What a batch of samples is drawn with. Sample g draws from the breeding
 * stream Rng::stream(seed, generation, round, slot g) (src/evolution.rs:
 * 455-600): the reference's counter-based generator, restated, so a sample
 * is the reference's child for that ring slot given the same emitter state. */
typedef struct ce_cma_draw {
    uint64_t seed;                    /* Config::seed */
    uint32_t generation;
    uint32_t reserved;                /* 0 */
    uint64_t round;                   /* the breeding round */
    uint64_t first_id;                /* sample g gets id first_id + g */
    float strength;                   /* Config::mutation (1 by default) */
    float min_size, max_size;         /* repair's diameter range (0.06, 0.12 m by default) */
    float min_friction, max_friction; /* repair's friction range (0.65, 1 by default) */
} ce_cma_draw;
/* The coordinate offsets of emitters with these template genomes and modes
 * (host arrays; `exploring` may be NULL; `offsets` gets emitters + 1
 * entries, the last the total). */
ce_status ce_cma_offsets(const ce_genome* templates, const uint8_t* exploring, size_t emitters,
                         uint64_t* offsets);
/* CmaEmitter::optimizer and CmaEmitter::new: the means at the templates'
 * coordinates, unit covariances, zero paths, step size 0.5 for an optimizer
 * and 0.12 for a CMA-ME emitter. Checks (reading the template genomes back,
 * synchronising `stream`) that their genes are packed in order from row 0,
 * which ask relies on; ask and tell only launch. */
ce_status ce_cma_init(const ce_cma* cma, void* stream);
/* sample_optimizing / sample_exploring (src/qd.rs:2244-2289, 2377-2402) for
 * samples [first, first + count): sample g belongs to emitter g mod emitters,
 * goes back to genes with apply_parameters / apply_exploring_parameters
 * (src/qd.rs:2579-2606, 2773-2811) and repair's diameter and friction
 * ranges (src/evolution.rs:1230-1234), id draw->first_id + g. The rows are
 * laid out as ce_sample_device lays them (ce_sample_rows with the templates
 * as parents sizes them); `strength_out` (or NULL) gets the templates'
 * strength factors, `values` (or NULL) the drawn coordinates, `stride`
 * floats a sample (the largest emitter's coordinates; any past `stride`
 * are not written). */
ce_status ce_cma_ask(const ce_cma* cma, const ce_cma_draw* draw, uint64_t first, size_t count,
                     ce_node_gene* nodes, ce_bone_gene* bones, ce_muscle_gene* muscles, float* strength_out,
                     ce_genome* genomes, float* values, size_t stride, void* stream);
/* tell, tell_optimizing and tell_exploring (src/qd.rs:2213-2243,
 * 2290-2376, 2405-2474) from the samples [first, first + count) of one
 * ce_cma_ask (their genes and one key a sample, in that order: fitness for
 * an optimizer, the archive's improvement key for a CMA-ME emitter): each
 * emitter keeps its finite samples above the failure score whose body plan
 * is the template's (counts and bone and muscle connections, gene by gene),
 * the best 1024 best first (ties by sample index), and updates its mean,
 * paths, covariance and step size. At most 4096 samples an emitter a call. */
ce_status ce_cma_tell(const ce_cma* cma, const ce_population* samples, const float* keys, uint64_t first,
                      size_t count, void* stream);
/* CmaEmitter::recentered (src/qd.rs:2166-2177) for emitters which[0..n)
 * (device array, distinct emitters): emitter which[i] restarts from body i of `bodies`, which
 * must have its template's node, bone and muscle counts (else it is left as
 * it was and rejected[i], a device array or NULL, is set to 1; an index
 * past the last emitter is rejected too). The body's
 * genes overwrite the template's (the templates' memory must be writable),
 * the mean moves to the body's coordinates, and the covariance, paths and
 * step size are kept when the body's plan (bone and muscle connections) is
 * the template's, else restart as the mode's constructor sets them. */
ce_status ce_cma_recenter(const ce_cma* cma, const ce_population* bodies, const uint32_t* which, size_t n,
                          uint32_t* rejected, void* stream);

/* ---- rung audit on the device ---- */
/* Sums::add's sums of one class of feature vectors (src/rungs.rs:286-299):
 * the count, the sum of each feature and of each product, float64. */
typedef struct ce_audit_sums {
    uint64_t n;
    double sum[6];
    double xx[6][6];
} ce_audit_sums;
/* One batch's rung audit: Audit::note over every trial (src/rungs.rs:
 * 510-525) and GenAudit::of over its audit rows (src/rungs.rs:319-345). */
typedef struct ce_audit {
    uint64_t creatures, steps;
    uint64_t stops[3];       /* stopped by R1, R2 and the 5 s screen */
    uint32_t rows, reserved; /* audit rows (GenAudit::rows) */
    ce_audit_sums a[2], b[2]; /* per rung: class A (reached the 5 s bar), class B */
} ce_audit;
/* Scratch ce_audit_device needs for `count` trials. */
size_t ce_audit_scratch_bytes(size_t count);
/* The rung audit of `count` trials from resident results, in batch order
 * (record_rungs, src/storage.rs:672-708): creature i's result, genome (its
 * flags: rungs::AUDIT and EXEMPT; its first muscle's period, from `muscles`)
 * and its block's screen bar bars[i] (not finite: no bar). Audit rows are
 * the trials of AUDIT creatures whose trace is not empty; every float64 sum
 * is added in row order, as the reference adds it. a_words (or NULL) gets,
 * per rung r, class A's feature words (6 halves a row) at
 * [(r a_cap + i) 6], the first a_cap rows. All pointers are device
 * addresses; scratch holds ce_audit_scratch_bytes(count) bytes. */
ce_status ce_audit_device(const ce_result* results, const ce_genome* genomes, const ce_muscle_gene* muscles,
                          const float* bars, size_t count, void* scratch, size_t scratch_bytes, ce_audit* out,
                          uint16_t* a_words, size_t a_cap, void* stream);

/* ---- engine ------------------------------------------------------------ */
typedef struct ce_engine ce_engine;

typedef struct ce_options {
    uint32_t slots;          /* concurrent submissions, 0 = default (4) */
    uint32_t ctas_per_sm;    /* resident blocks an SM, 0 = as many as fit */
    uint32_t warps_per_cta;  /* reserved, 0 (blocks are 4 warps) */
    uint32_t chunk_k;        /* claims shrink to 1/chunk_k of a queue's rest a warp, 0 = 64 */
    uint32_t small_body;     /* most nodes of the first size class, 0 = 12 */
    uint32_t reserved[3];
} ce_options;

ce_status ce_open(int device, const ce_options* options, ce_engine** out);
/* Times `sample` (a packed batch like the ones to come) in `world` under a
 * grid of launch settings (blocks an SM, claim chunk divisor, size-class
 * split) and keeps the fastest for the engine's later submissions; `best`
 * (optional) receives it and `seconds` (optional) its GPU time. No
 * counterpart in the reference, whose launch shape is fixed. */
ce_status ce_autotune(ce_engine* engine, const ce_wave_pack* sample, const ce_world* world, ce_options* best,
                      double* seconds);
ce_status ce_close(ce_engine* engine);
const char* ce_last_error(void);

/* Queues the batch `pack` in world `world` (host memory; copied before the
 * call returns). Results come back in packed order through ce_poll. */
ce_status ce_submit(ce_engine* engine, const ce_wave_pack* pack, const ce_world* world,
                    uint64_t* ticket);
/* Takes the oldest finished submission. `n` receives its result count;
 * `cap` must be at least that. CE_ERR_TIMEOUT when none finishes in time. */
ce_status ce_poll(ce_engine* engine, int64_t timeout_us, uint64_t* ticket, ce_result* out,
                  size_t cap, size_t* n, double* busy_seconds);
/* Waits until a submission has finished or `timeout_us` passed. */
ce_status ce_wait(ce_engine* engine, int64_t timeout_us);
int ce_free_slots(ce_engine* engine);
size_t ce_allocated_bytes(ce_engine* engine);
ce_status ce_release_idle(ce_engine* engine);

/* Records K creatures of `pack` (K = pack->count <= CE_RECORD_MAX_CREATURES):
 * every frame of each trial, creature-major then frame-major, `stride`
 * float2 slots per creature and frame (src/creature_kernel.rs:312-326);
 * frames = SETTLE + steps + 1 a creature. The reference records one creature
 * a call; many-creature recordings run as one launch over the GPU. The
 * frames take K x frames x stride x 8 bytes on the device as well.
 * Synchronous. */
#define CE_RECORD_MAX_CREATURES 65536u
ce_status ce_record(ce_engine* engine, const ce_wave_pack* pack, const ce_world* world,
                    float* frames, size_t frames_cap_floats, ce_result* results);

/* Device-level entry, the kernel ABI of shaders/creature.cu:1266-1277: runs
 * `params->count` creatures from `params->base` of device-resident records
 * on `stream` (a cudaStream_t, NULL for the legacy stream). `rate` is the
 * step rate the reference compiles into its kernel (60 or 120). Bodies must
 * have at most `max_nodes` nodes and `max_muscles` muscles. `scratch` is a
 * device buffer of at least ce_advance_scratch_bytes(..., params->count)
 * bytes: the lane slots, and the claim queues that the call first builds
 * by bucketing the creatures by node count (with their claim counters,
 * zeroed by the call). `counter` is kept from the reference's kernel
 * arguments; this entry neither reads nor writes it. Asynchronous. */
size_t ce_advance_scratch_bytes(ce_engine* engine, uint32_t world_flags, uint32_t rate,
                                uint32_t max_nodes, uint32_t max_muscles, uint32_t count);
ce_status ce_advance_device(ce_engine* engine, const uint32_t* records, const float* muscles,
                            const uint32_t* heads, ce_result* results, uint32_t* counter,
                            void* scratch, const ce_params* params, uint32_t world_flags,
                            uint32_t rate, uint32_t max_nodes, uint32_t max_muscles,
                            void* stream);

/* ce_advance_device with the niche epilogue fused into the creature
 * kernel: when a creature's trial ends, the kernel stores its result and
 * also its metrics row (`metrics`, may be NULL) and its dense niche cell
 * (`cells`, int64, -1 for a shape outside the layout), equal to the host's
 * ce_to_metrics and ce_niche to the bit, so no pass over the results
 * follows. `shape_classes` (packed order, from ce_shape_classes) gives each
 * body's shape class; `world` gives the flags, rate and trial length.
 * Replaces the host's scheduler::to_metrics and Descriptor::niche_in
 * (src/scheduler.rs:890-923, src/qd.rs:762-846, 988-999) run after
 * CudaEngine::poll; the reference kernel itself stores results only. */
ce_status ce_advance_device_cells(ce_engine* engine, const uint32_t* records, const float* muscles,
                                  const uint32_t* heads, ce_result* results, uint32_t* counter, void* scratch,
                                  const ce_params* params, const ce_world* world, uint32_t max_nodes,
                                  uint32_t max_muscles, const uint8_t* shape_classes, int global_layout,
                                  ce_metrics* metrics, int64_t* cells, void* stream);

/* Several generations as one CUDA graph (no counterpart in the reference,
 * which launches each wave): the packed batches are copied to the device
 * once; ce_graph_launch runs every generation (node-count bucketing and the
 * size classes' launches, generation after generation) as one graph launch
 * and gives its GPU seconds; ce_graph_results reads a generation's results in
 * packed order. Kernel attributes are set while opening, so the capture holds
 * stream work only. */
typedef struct ce_graph ce_graph;
ce_status ce_graph_open(ce_engine* engine, const ce_wave_pack* packs, uint32_t generations,
                        const ce_world* world, ce_graph** graph);
ce_status ce_graph_launch(ce_graph* graph, double* seconds);
ce_status ce_graph_results(ce_graph* graph, uint32_t generation, ce_result* out, size_t cap);
ce_status ce_graph_close(ce_graph* graph);

/* Gradients of fitness (no counterpart in the reference, which has no
 * derivatives): a forward/backward pair shaped like an autograd function.
 * ce_forward runs the batch in the calm world (flat ground, no effects) or
 * in an effects world (rough, sloped ground with hurdles, tremors, water,
 * ice, wind, thick air: the flag sets of the effects workloads;
 * CE_ERR_UNSUPPORTED for other flag sets, with mud, brambles or gaps, or for
 * muscles with touch sensors) with a
 * checkpoint of each creature's state every `checkpoint_every` substeps
 * (256 only) and keeps what the backward pass needs in the tape; its results
 * equal ce_submit's to the bit. ce_backward returns, for every creature in
 * packed order, d(sum_c dl_dfitness[c] * fitness_c) with respect to the
 * creature's record fields: ce_tape_grad_floats(tape) floats a creature,
 * first 9 a muscle slot (stroke amplitude, hill factor, force cap,
 * 1 / energy capacity, phase, duty, 1 / duty, 1 / (1 - duty), stiffness;
 * muscle slots up to the batch's largest muscle count), then per node row
 * (rows up to the largest node count) its friction, then its mass, then its
 * start position as (x, y) pairs. `dl_dfitness` NULL means 1
 * for every creature. Both are synchronous; ce_tape_seconds gives their
 * GPU time. ce_gene_gradients maps the record gradients to genes. */
typedef struct ce_tape ce_tape;
ce_status ce_forward(ce_engine* engine, const ce_wave_pack* pack, const ce_world* world,
                     uint32_t checkpoint_every, ce_tape** tape);
ce_status ce_tape_results(ce_tape* tape, ce_result* out, size_t cap);
uint32_t ce_tape_grad_floats(ce_tape* tape);
ce_status ce_tape_seconds(ce_tape* tape, double* forward_seconds, double* backward_seconds);
ce_status ce_backward(ce_tape* tape, const float* dl_dfitness, float* grads, size_t cap_floats);
/* ce_backward that also checks its reruns against the forward run, to the
 * bit: per creature (packed order) `mismatches` gets bit 0 when a
 * segment's rerun from its checkpoint does not end on the next checkpoint
 * and bit 1 when a substep's kept rerun does not end on the next tape state;
 * 0 everywhere means every gradient was taken along the forward run's own
 * trajectory. Slower than ce_backward (one more read of the state a
 * substep). */
ce_status ce_backward_checked(ce_tape* tape, const float* dl_dfitness, float* grads, size_t cap_floats,
                              uint32_t* mismatches);
ce_status ce_tape_free(ce_tape* tape);
/* The tangent-linear run of the tape's batch (the worlds ce_forward takes): for each
 * creature, the derivative of its fitness along a direction of its record
 * fields, on the same FP32 trajectory and contact, slip and joint-limit
 * modes as the forward run. Directions in packed order, laid out as
 * ce_backward's gradient (ce_tape_shape's rows and muscle slots), each NULL
 * for zero but not all four: `dstart` rows x 2 floats a creature (start
 * positions), `dmuscle` 9 x muscle slots (amplitude, hill, cap,
 * 1/capacity, phase, duty, 1/duty, 1/(1-duty), stiffness), `dfriction` rows,
 * `dmass` rows (node masses, with their inverses).
 * <ce_backward's gradient, direction> equals `dfitness` up to the rounding
 * of the two derivative computations: the adjoint's check. No counterpart
 * in the reference. */
ce_status ce_tangent(ce_tape* tape, const float* dstart, const float* dmuscle, const float* dfriction,
                     const float* dmass, float* dfitness);
/* The forward run's checkpoints, for checking: per creature (packed order)
 * ceil(steps / 16) checkpoints of rows x 4 + muscle slots floats (positions
 * and velocities of each node row as (x, y) pairs, then the muscles' energy
 * stores), `per_creature` receiving the checkpoint count. */
ce_status ce_tape_checkpoints(ce_tape* tape, float* out, size_t cap_floats, uint32_t* per_creature);
/* Node rows and muscle slots of the tape's gradient records. */
ce_status ce_tape_shape(ce_tape* tape, uint32_t* rows, uint32_t* muscle_slots);
/* Gene gradients of the creatures of a batch packed by ce_pack(pop,
 * indices, n, world, ..., slots, ...), from its record gradients `grads`
 * (rows and muscle slots as ce_tape_shape gives): for each muscle gene 5
 * doubles at muscle_grads[5 * muscle index] (d/d short length, long length,
 * strength scale, on time, off time, the period held fixed; on time and off
 * time give phase = frac(-on / period) and duty = frac((off - on) / period)
 * clamped to [0.05, 0.95]), and d/d friction at node_grads[node index]. */
ce_status ce_gene_gradients(const ce_population* pop, const uint32_t* indices, size_t n,
                            const ce_world* world, const uint32_t* slots, const float* grads,
                            uint32_t rows, uint32_t muscle_slots, double* muscle_grads,
                            double* node_grads);

/* The device-level entry above for a caller that cannot allocate GPU memory:
 * no counterpart in the reference. It allocates nothing: the kernel's
 * scratch (claim counter and lane slots) is a fixed array of
 * ce_noalloc_scratch_bytes() (32 MiB) in the library's device memory, held
 * on every GPU that loads the library until exit. It runs on the current
 * device, as many warps as the array holds at this body size (so it can be
 * slower than ce_advance_device), and rejects a body size whose single block
 * does not fit. Calls share the array: calls that overlap on the GPU race.
 * A call outside a stream capture looks the array's address up on the
 * current device each time (so a primary context that was torn down and
 * created again is followed); a call inside a capture reuses the address
 * the last call outside one found, so the first call on a device must come
 * before any stream capture. Inputs and outputs are the caller's. */
ce_status ce_advance_device_noalloc(const uint32_t* records, const float* muscles,
                                    const uint32_t* heads, ce_result* results,
                                    const ce_params* params, uint32_t world_flags, uint32_t rate,
                                    uint32_t max_nodes, uint32_t max_muscles, void* stream);
size_t ce_noalloc_scratch_bytes(void);

/* The FP32 multiply-add rate of `device` in TFLOP/s (two operations per
 * multiply-add), from a calibration kernel of independent chains on every
 * multiprocessor; the denominator of the creature kernel's FP32 roofline. */
ce_status ce_measure_fp32(int device, double* tflops, double* seconds);

/* Host-side fault injection for the recovery paths (src/scheduler.rs:725):
 * the `after`-th next submit fails with `status`. 0 turns it off. */
ce_status ce_inject_fault(ce_engine* engine, uint32_t after, ce_status status);

/* A batch's gradient ascent kept on the device, as one CUDA graph (no
 * counterpart in the reference, which refines only by CMA-ES). Opening packs
 * the `pop->count` creatures once on the host (the plan of ce_pack_plan),
 * uploads their genes (arrays of nodes_len, bones_len, muscles_len genes;
 * the strength scale if given) and captures `steps` ascent steps and a last
 * scoring: per step the checkpointed forward run (scoring the step's
 * genes), the backward run of d(sum of fitness), the gene gradients (as
 * ce_gene_gradients), one clipped ascent step of `step_size` on each muscle's
 * short, long, strength scale, phase and duty and each node's friction
 * (each move clipped to the coordinate's unit: 0.02 x the body's mean bone
 * length, 0.05, 0.03 for friction; then the genes' clamps) and the
 * repacking of the records on the device (ce_pack_device). The calm and
 * effects worlds, no touch sensors. ce_ascent_launch runs the graph;
 * ce_ascent_fitness gives step k's fitness in population order (k = steps:
 * the last genes); ce_ascent_genes copies the genes back. */
typedef struct ce_ascent ce_ascent;
ce_status ce_ascent_open(ce_engine* engine, const ce_population* pop, const ce_world* world, uint32_t steps,
                         double step_size, size_t nodes_len, size_t bones_len, size_t muscles_len, ce_ascent** out);
ce_status ce_ascent_launch(ce_ascent* ascent, double* seconds);
ce_status ce_ascent_fitness(ce_ascent* ascent, uint32_t step, float* fitness, size_t cap);
ce_status ce_ascent_genes(ce_ascent* ascent, ce_node_gene* nodes, ce_muscle_gene* muscles, float* strength);
ce_status ce_ascent_close(ce_ascent* ascent);

#ifdef __cplusplus
}
#endif
#endif /* CREATURE_ENGINE_H */
