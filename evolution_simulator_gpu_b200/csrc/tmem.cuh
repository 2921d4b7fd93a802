// Tensor Memory (TMEM) as per-lane storage for a creature's constants.
//
// Each multiprocessor has 128 TMEM lanes of 512 32-bit columns. With the
// 32x32b access shape a warp reads or writes 32 lanes, thread t its own lane,
// and warp w of a block may touch only lanes 32 (w mod 4) .. 32 (w mod 4) + 31;
// a 128-thread block therefore owns one lane per thread and every column it
// allocates. The creature kernel keeps there, per thread, the constants that
// its node, bone and joint passes read every substep (TmLayout), so those
// passes no longer wait on L2 for them. TMEM addresses are warp-uniform
// (one column for the whole warp), so every access sits in a loop whose trip
// count is the same for all 32 lanes of the warp.
//
// The accesses are the tcgen05 instructions of sm_100a written as inline PTX:
// alloc / relinquish_alloc_permit / dealloc by one warp of the block, ld and
// st of the 32x32b shape, wait::ld and wait::st. A load's registers are
// defined only after wait::ld, so `wait` takes the loaded values as in-out
// operands: nothing that reads them can be scheduled before it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cek {

// Where each kind of constant lives in a lane's TMEM columns, for a class of
// `ns` node rows. Quads are 4 columns starting at a multiple of 4; scalars
// are 1 column.
//   node i quad:   m, 1/m, radius, friction
//   bone j quad:   pivot node (bits), rest length, 1/m of the pivot, air drag factor
//   joint j quad (j = 1 .. ns - 2): topology word, lo, hi, 1/m of the far node
//   bone j limit:  drag limit (0.5 m_bone / h)
//   joint j hub:   1/m of the hub node
//   bone j pivot radius (worlds with water only)
// What the passes derive from these (1/m of a bone's child node, the drag
// scales 0.5 h / m, a joint's middle angle) is recomputed with the same
// operations as the kernel's set-up, so the values are the same to the bit.
struct TmLayout {
    unsigned node, bone, joint, limit, hub, radius, total;
    __host__ __device__ static TmLayout make(unsigned ns, bool water) {
        TmLayout t;
        const unsigned bones = ns - 1u, joints = ns > 2u ? ns - 2u : 0u;
        t.node = 0u;
        t.bone = 4u * ns;
        t.joint = t.bone + 4u * bones;
        t.limit = t.joint + 4u * joints;
        t.hub = t.limit + bones;
        t.radius = t.hub + joints;
        t.total = t.radius + (water ? bones : 0u);
        return t;
    }
};

// Columns a block allocates: a power of two from 32 to 512, at most an even
// share of the 512 among `blocks` resident blocks, and no more than the
// layout needs.
__host__ __device__ inline unsigned tmem_columns(unsigned layout_total, unsigned blocks) {
    unsigned share = 512u;
    while (share > 32u && share * (blocks > 0u ? blocks : 1u) > 512u) share >>= 1u;
    unsigned need = 32u;
    while (need < layout_total && need < 512u) need <<= 1u;
    return need < share ? need : share;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// One warp of the block allocates `cols` columns and writes their address to
// `slot` (shared memory); the permit is given back at once, since the block
// allocates nothing else.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols));
}
__device__ __forceinline__ void tmem_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;"); }
__device__ __forceinline__ void tmem_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;"); }

// This warp's view of the block's TMEM: its 32 lanes, all allocated columns.
struct Tmem {
    uint32_t addr;  // lane field: this warp's lane quarter; column field: 0
    uint32_t cols;  // columns allocated by the block

    __device__ __forceinline__ float4 ld4(uint32_t col) const {
        uint32_t a, b, c, d;
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
                     : "r"(addr + col));
        return make_float4(__uint_as_float(a), __uint_as_float(b), __uint_as_float(c), __uint_as_float(d));
    }
    __device__ __forceinline__ float ld1(uint32_t col) const {
        uint32_t a;
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(a) : "r"(addr + col));
        return __uint_as_float(a);
    }
    __device__ __forceinline__ void st4(uint32_t col, const float4& v) const {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr + col),
                     "r"(__float_as_uint(v.x)), "r"(__float_as_uint(v.y)), "r"(__float_as_uint(v.z)),
                     "r"(__float_as_uint(v.w)));
    }
    // Waits for this thread's loads; the values given become usable.
    __device__ __forceinline__ static void wait(float4& a) {
        asm volatile("tcgen05.wait::ld.sync.aligned;" : "+f"(a.x), "+f"(a.y), "+f"(a.z), "+f"(a.w));
    }
    __device__ __forceinline__ static void wait(float4& a, float& b, float& c) {
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+f"(a.x), "+f"(a.y), "+f"(a.z), "+f"(a.w), "+f"(b), "+f"(c));
    }
    __device__ __forceinline__ static void wait(float4& a, float& b, float& c, float& d) {
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+f"(a.x), "+f"(a.y), "+f"(a.z), "+f"(a.w), "+f"(b), "+f"(c), "+f"(d));
    }
    __device__ __forceinline__ static void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
};

}  // namespace cek
