// Launch interface of the creature kernel family, shared by the kernels and
// the host engine.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/creature_engine.h"
#include "niche.cuh"

namespace cek {

// Threads per block and the blocks per multiprocessor the register budget
// is sized for (128 registers a thread at most).
constexpr unsigned kBlock = 128;
constexpr unsigned kMinBlocks = 4;

// Worlds compiled with their effects fixed: the calm world, the effects
// world (rough ground, slope, hurdles, water, ice, wind, thick air), the
// same with earthquakes, and every effect on. Other worlds run on the kernel
// that reads the switches at run time.
constexpr uint32_t kWorldCalm = CE_FLAG_GROUND;
constexpr uint32_t kWorldEffects = CE_FLAG_GROUND | CE_FLAG_TERRAIN | CE_FLAG_SLOPE | CE_FLAG_HURDLES |
                                   CE_FLAG_WATER | CE_FLAG_ICE | CE_FLAG_WIND | CE_FLAG_AIR;
constexpr uint32_t kWorldEffectsQuake = kWorldEffects | CE_FLAG_QUAKE;
constexpr uint32_t kWorldAll = 0xfffu;

// Shared memory of a block: the position, velocity and force tables (8 bytes
// each) for `rows` node rows of every thread, and the (energy store, demand)
// pair of `mm` muscles of every thread.
inline size_t smem_bytes(unsigned rows, unsigned mm, unsigned block) {
    return (size_t)block * (rows * 24u + (mm > 0 ? mm : 1u) * 8u);
}

// Claim queues. A launch with queues takes its creatures from one queue per
// node count: queue q holds order[bounds[q] .. bounds[q + 1]), claimed
// through counter[q], and work[q] is the estimated work of the queues below
// q. Inside a queue the creatures keep the packed order, whose muscle count
// ascends, so the lanes of a warp hold bodies of the same node count and
// nearly the same muscle count and its loops run to nearly the same length.
constexpr unsigned kQueues = CE_MAX_NODES + 1u;  // node counts 0..32
constexpr unsigned kBucketTile = 4096u;          // creatures a block buckets

struct KernelArgs {
    const uint32_t* records;
    const float* muscles;
    const uint4* heads;
    ce_result* results;
    uint32_t* counter;             // one claim counter a queue (one for no queues), zeroed
    float4* scratch;               // slots: warps of the grid x lines x 32 lanes
    float2* frames;                // RECORD: frames of each recorded creature
    const uint32_t* order;         // packed positions of this launch's creatures
    const uint32_t* bounds;        // queues + 1 positions of the order list
    const unsigned long long* work;  // queues + 1 prefix sums of estimated work
    uint32_t queues;               // 0: one queue, positions 0 .. count - 1
    uint32_t count;                // creatures of this launch
    uint32_t rows;                 // node rows: most nodes of a body of this launch
    uint32_t mm;                   // most muscles of a body of this launch
    uint32_t frames_per_creature;  // RECORD: frames of one recording
    uint32_t chunk_k;              // claims shrink to 1 / chunk_k of the rest per warp
    float* ckpt;                   // CKPT: checkpoints, creature-minor: float f of checkpoint k of
                                   // creature c (packed index) at (k * checkpoint_floats + f) * count + c
    uint32_t* ends;                // CKPT: steps each creature's trial ran (packed index)
    // Niche epilogue at the result store (plain kernel; `cells` NULL: none):
    // each creature's metrics row (`metrics` may be NULL) and dense cell,
    // from its result, node count and shape class (packed index).
    const uint8_t* shapes;
    ce_metrics* metrics;
    int64_t* cells;
    MetricsArgs niche;
};

// Metrics arguments of a world in the global (1) or an island's (0) layout.
MetricsArgs metrics_args(const ce_world* world, int global_layout);

// Floats of one checkpoint: positions and velocities of `rows` nodes, then
// the energy stores of `mm` muscles.
__host__ __device__ inline unsigned checkpoint_floats(unsigned rows, unsigned mm) { return 4u * rows + mm; }

// Gradient of one creature's fitness per record field: for each of `mm`
// muscles the stroke amplitude, hill factor, force cap, inverse energy
// capacity, phase, duty, 1 / duty, 1 / (1 - duty) and stiffness, then the
// friction of each of `rows` nodes, then each node's mass (through every
// place the kernel uses a mass or an inverse mass and the fitness's mass
// weighting), then each node's start position (x, y).
constexpr unsigned kGradMuscle = 9u;
__host__ __device__ inline unsigned grad_floats(unsigned rows, unsigned mm) { return kGradMuscle * mm + 4u * rows; }

// Gradient kernels (calm world): the creature kernel with checkpoints every
// 256 substeps (KernelArgs::ckpt, ends), and the backward kernel.
size_t adjoint_smem_bytes(unsigned rows, unsigned mm, unsigned block);
size_t adjoint_slot_bytes(unsigned grid, unsigned rows, unsigned mm);   // lane slots of the backward grid
size_t adjoint_tape_bytes(unsigned grid, unsigned rows, unsigned mm);   // segment tapes of the backward grid
// Worlds the gradient kernels are built for: calm, effects, effects + tremors.
bool gradient_world(uint32_t flags);
cudaError_t adjoint_occupancy(unsigned rows, unsigned mm, uint32_t flags, int rate, int* blocks);
struct LaunchSpec;
cudaError_t launch_forward_ckpt(const LaunchSpec& s, const KernelArgs& a, const ce_params& p);
// The tangent-linear run (the adjoint's check; the gradients' worlds): d fitness
// of each creature along directions of its start positions (dstart, 2 x
// rows floats a creature), muscle record fields (dmuscle, kGradMuscle x mm),
// node frictions (dfriction, rows) and node masses (dmass, rows), packed
// index, each null for 0, into
// dfitness, on the lane slots of adjoint_slot_bytes and the checkpointed
// forward run's ends and results.
size_t tangent_smem_bytes(unsigned rows, unsigned mm, unsigned block);
bool tangent_world(uint32_t flags);
cudaError_t launch_tangent(const LaunchSpec& s, const KernelArgs& a, const ce_params& p, const float* dstart,
                           const float* dmuscle, const float* dfriction, const float* dmass, float* dfitness);
// `mismatch` (NULL: no check): per creature, bits of reruns that did not
// reproduce the forward run to the bit (bit 0 a segment's rerun against the
// next checkpoint, bit 1 a substep's kept rerun against the next tape state).
cudaError_t launch_adjoint(const LaunchSpec& s, const KernelArgs& a, const ce_params& p, float4* tape, float* grads,
                           const float* weights, uint32_t* mismatch);

// The device arrays that bucketing writes for `count` creatures, carved from
// one area of bucket_bytes(count) bytes.
struct Buckets {
    uint32_t* order;            // count packed positions, node count by node count
    uint32_t* hist;             // kQueues x tiles: creatures of each node count per tile
    uint32_t* bounds;           // kQueues + 1
    unsigned long long* work;   // kQueues + 1
    unsigned long long* bins;   // kQueues: estimated work of each node count
    uint32_t* counters;         // kQueues, zeroed by the bucketing
    uint32_t tiles;
};
size_t bucket_bytes(size_t count);
Buckets bucket_layout(void* area, size_t count);
// Buckets creatures base .. base + count - 1 of a packed batch by node count
// (three kernels on `stream`); the heads give the node and muscle counts.
cudaError_t launch_bucket(const uint4* heads, uint32_t base, uint32_t count, const Buckets& b, cudaStream_t stream);

struct LaunchSpec {
    unsigned rows;   // node rows of the tables (most nodes of a body)
    unsigned mm;     // most muscles of a body
    uint32_t flags;  // world effect bits
    bool record;
    int rate;        // steps per second: 60 or 120
    unsigned grid, block;
    cudaStream_t stream;
};

// 16-byte lines of one lane's slot.
unsigned slot_lines(unsigned rows, unsigned mm, bool record);

cudaError_t launch_advance(const LaunchSpec& s, const KernelArgs& a, const ce_params& p);
// The device packer and the refinement's ascent (csrc/pack.cu).
cudaError_t launch_pack(const ce_population& pop, const float* trig, const uint32_t* order, const uint32_t* record_at,
                        const uint32_t* muscle_at, size_t n, const ce_world& w, uint32_t* lanes, float* muscles,
                        uint32_t* heads, cudaStream_t stream);
cudaError_t launch_gene_grads(const ce_population& pop, const float* trig, const uint32_t* order, size_t n,
                              const ce_world& w, const float* grads, uint32_t rows, uint32_t mm, double* muscle_grads,
                              double* node_grads, cudaStream_t stream);
cudaError_t launch_ascend(const ce_population& pop, ce_node_gene* nodes, ce_muscle_gene* muscles, float* strength,
                          const double* muscle_grads, const double* node_grads, double step, cudaStream_t stream);
// A recording's frames from the kernel's frame-major, creature-minor layout
// (`rows` = frames x slots rows of `creatures` entries) to the reference's
// creature-major one (`creatures` rows of `rows` entries).
cudaError_t launch_frames_to_creature_major(const float2* src, float2* dst, size_t rows, uint32_t creatures,
                                            cudaStream_t stream);
cudaError_t advance_occupancy(unsigned rows, unsigned mm, uint32_t flags, bool record, int rate, unsigned block,
                              int* blocks);
// Sets the kernel's dynamic shared-memory limit for `rows` x `mm` tables: a
// CUDA graph's launches are checked against the limit in force when it runs.
cudaError_t advance_reserve_smem(unsigned rows, unsigned mm, uint32_t flags, bool record, int rate, unsigned block);

}  // namespace cek
