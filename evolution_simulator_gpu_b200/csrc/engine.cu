// The engine behind the C ABI: one handle per GPU, a few submission slots,
// each with its stream, events, pinned staging and device buffers.
//
// A submission (the reference's CudaEngine::launch, src/cuda_engine.rs:
// 2106-2316) uploads the packed batch, buckets it by node count on the
// device into claim queues, splits it into two size classes by node count
// (bodies of at most 16 nodes, and larger ones), runs one persistent launch
// per class, the two side by side on two streams so that the tail of one
// overlaps the other, and reads the results back. ce_poll hands back
// the oldest finished submission with its GPU-busy seconds, as the
// reference's poll does (src/cuda_engine.rs:2319-2393).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "../../include/creature_engine.h"
#include "host_model.h"
#include "kernels.h"

using ce::set_error;

namespace {

// Bodies of up to this many nodes form the first size class (default).
constexpr unsigned kSmallBody = 12u;

ce_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CE_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return CE_ERR_OOM;
    }
    return CE_ERR_DEVICE;
}
#define CE_TRY(expr, what)                                   \
    do {                                                     \
        ce_status _s = cuda_status((expr), (what));          \
        if (_s != CE_OK) return _s;                          \
    } while (0)

// A device buffer that grows and keeps its memory for later submissions.
struct DeviceBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    ce_status ensure(size_t need) {
        if (need <= bytes) return CE_OK;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        const size_t grown = std::max(need, (size_t)1 << 20);
        CE_TRY(cudaMalloc(&ptr, grown), "cudaMalloc");
        bytes = grown;
        return CE_OK;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};
struct PinnedBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    ce_status ensure(size_t need) {
        if (need <= bytes) return CE_OK;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        const size_t grown = std::max(need, (size_t)1 << 20);
        CE_TRY(cudaMallocHost(&ptr, grown), "cudaMallocHost");
        bytes = grown;
        return CE_OK;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct ClassPlan {
    uint32_t first_n, last_n;  // node counts of the class: its claim queues
    uint32_t count;            // creatures of the class
    uint32_t rows;             // most nodes in the class
    uint32_t mm;               // most muscles in the class
    double work;               // estimated arithmetic of a substep of all its creatures
};

struct Slot {
    bool busy = false;
    uint64_t ticket = 0;
    size_t count = 0;
    cudaStream_t stream = nullptr, side = nullptr;  // side: the second class
    cudaEvent_t start = nullptr, stop = nullptr, done = nullptr, joined = nullptr, bucketed = nullptr;
    DeviceBuf d_lanes, d_muscles, d_heads, d_results, d_buckets, d_scratch;
    PinnedBuf h_upload, h_results;
    std::chrono::steady_clock::time_point submitted;
};

}  // namespace

struct ce_engine {
    int device = 0;
    int sms = 0;
    unsigned ctas_per_sm = 0;  // 0: from the occupancy of each kernel
    unsigned chunk_k = 64;
    size_t smem_optin = 0;  // shared memory a block may use
    size_t smem_sm = 0;     // shared memory of an SM
    size_t smem_reserved = 0;  // shared memory the system keeps a block
    unsigned small_body = kSmallBody;
    std::vector<Slot> slots;
    std::deque<size_t> pending;  // slot indices, oldest first
    uint64_t next_ticket = 1;
    uint32_t fault_after = 0;
    ce_status fault_status = CE_OK;
    // Recording buffers.
    DeviceBuf rec_frames, rec_staging, rec_lanes, rec_muscles, rec_heads, rec_results, rec_counter, rec_scratch;
};

namespace {

ce_status set_device(ce_engine* e) { return cuda_status(cudaSetDevice(e->device), "cudaSetDevice"); }

// The grid of a persistent launch for a class: every block that fits.
unsigned grid_for(ce_engine* e, unsigned rows, unsigned mm, uint32_t flags, bool record, int rate, size_t count) {
    int per_sm = 0;
    if (e->ctas_per_sm) {
        per_sm = (int)e->ctas_per_sm;
    } else if (cek::advance_occupancy(rows, mm, flags, record, rate, cek::kBlock, &per_sm) != cudaSuccess ||
               per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const size_t needed = (count + cek::kBlock - 1) / cek::kBlock;
    const size_t full = (size_t)per_sm * (size_t)e->sms;
    return (unsigned)std::max<size_t>(1, std::min(needed, full));
}

size_t scratch_bytes(unsigned grid, unsigned rows, unsigned mm, bool record) {
    const size_t warps = (size_t)grid * (cek::kBlock / 32u);
    return warps * cek::slot_lines(rows, mm, record) * 32u * 16u;
}

// Grids of a batch's size classes (launched side by side). Each persistent
// launch sized alone fills every SM with its own blocks, so the second class
// would start only as the first one's blocks retire. When the two fit an SM
// together, the large-body class gets one block an SM and the small one as
// many as the shared memory left holds (and one less than it has alone, for
// the registers the large block takes), so both classes run at once. That
// pays while the large bodies carry the lesser part of the work and the
// small ones keep at least half their blocks; measured on the effects
// workload (3M x 20 s) at four class splits: split at 12 nodes (estimated
// work of the large class 0.40 of the small one's, 2 small blocks of 4)
// 2.51 s against 2.77 s one class after the other; at 8 (work 1.12) 4.32 s
// against 2.96 s; at 10 (0.65) 3.91 s against 2.81 s; at 16 (0.17, 1 small
// block of 3) 3.87 s against 2.91 s.
std::vector<unsigned> class_grids(ce_engine* e, const std::vector<ClassPlan>& plans, uint32_t flags, int rate) {
    std::vector<unsigned> grids(plans.size());
    for (size_t c = 0; c < plans.size(); c++) {
        grids[c] = grid_for(e, plans[c].rows, plans[c].mm, flags, false, rate, plans[c].count);
    }
    if (plans.size() != 2 || e->ctas_per_sm != 0 || e->smem_sm == 0) return grids;
    int alone_small = 0, alone_big = 0;
    if (cek::advance_occupancy(plans[0].rows, plans[0].mm, flags, false, rate, cek::kBlock, &alone_small) !=
            cudaSuccess ||
        cek::advance_occupancy(plans[1].rows, plans[1].mm, flags, false, rate, cek::kBlock, &alone_big) !=
            cudaSuccess) {
        cudaGetLastError();
        return grids;
    }
    const size_t small_b = cek::smem_bytes(plans[0].rows, plans[0].mm, cek::kBlock) + e->smem_reserved;
    const size_t big_b = cek::smem_bytes(plans[1].rows, plans[1].mm, cek::kBlock) + e->smem_reserved;
    if (alone_small < 2 || alone_big < 1 || e->smem_sm < big_b + small_b) return grids;
    if (plans[1].work > 0.5 * plans[0].work) return grids;
    const unsigned small_per_sm =
        (unsigned)std::min<size_t>((e->smem_sm - big_b) / small_b, (size_t)alone_small - 1u);
    if (2u * small_per_sm < (unsigned)alone_small) return grids;
    grids[0] = std::min<unsigned>(grids[0], small_per_sm * (unsigned)e->sms);
    grids[1] = std::min<unsigned>(grids[1], (unsigned)e->sms);
    return grids;
}

ce_status check_world(const ce_world* w) {
    if (!w) {
        set_error("null world");
        return CE_ERR_INVALID;
    }
    const uint32_t rate = ce::world_rate(*w);
    if (rate != 60 && rate != 120) {
        set_error("the engine runs 60 or 120 steps per second");
        return CE_ERR_UNSUPPORTED;
    }
    if (ce::world_steps(*w) < 1) {
        set_error("a trial needs at least one step");
        return CE_ERR_INVALID;
    }
    return CE_OK;
}

// Copies `n` bytes from pageable `src` to pinned `dst` on several host
// threads (one thread copies a few GB/s; a generation's records are GBs).
void parallel_copy(char* dst, const char* src, size_t n) {
    const unsigned threads = std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
    if (threads == 1 || n < ((size_t)8 << 20)) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t per = ((n + threads - 1) / threads + 4095) & ~(size_t)4095;
    std::vector<std::thread> pool;
    for (size_t at = per; at < n; at += per) {
        pool.emplace_back([=] { std::memcpy(dst + at, src + at, std::min(per, n - at)); });
    }
    std::memcpy(dst, src, std::min(per, n));
    for (std::thread& t : pool) t.join();
}

// Stages `n` bytes of `src` in the pinned `staging` buffer and copies them to
// `dev` on `stream`, 256 MB at a time, so that the copy of one chunk to the
// GPU runs while the next chunk is staged.
cudaError_t staged_upload(void* dev, char* staging, const void* src, size_t n, cudaStream_t stream) {
    const size_t chunk = (size_t)256 << 20;
    for (size_t at = 0; at < n; at += chunk) {
        const size_t len = std::min(chunk, n - at);
        parallel_copy(staging + at, static_cast<const char*>(src) + at, len);
        const cudaError_t e =
            cudaMemcpyAsync(static_cast<char*>(dev) + at, staging + at, len, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Splits the packed batch into size classes by node count (bodies of at most
// kSmallBody nodes, and larger ones). Each class runs as one launch whose
// claim queues are its node counts (kernels.h); the bucketing kernels build
// the queues on the device.
ce_status plan_classes(const ce_wave_pack* pack, std::vector<ClassPlan>& plans, unsigned small_body = kSmallBody) {
    plans.clear();
    size_t per_n[CE_MAX_NODES + 1] = {};
    uint32_t mm_n[CE_MAX_NODES + 1] = {};
    double work_n[CE_MAX_NODES + 1] = {};
    for (size_t i = 0; i < pack->count; i++) {
        const uint32_t* h = pack->heads + 8 * i;
        const unsigned n = h[0] & 255u, m = h[1];
        if (n < 2 || n > CE_MAX_NODES || m > CE_MAX_MUSCLES) {
            set_error("Unsupported body for the CUDA kernel: " + std::to_string(n) + " nodes, " +
                      std::to_string(m) + " muscles");
            return CE_ERR_INVALID;
        }
        per_n[n]++;
        mm_n[n] = std::max(mm_n[n], m);
        // Operations of a substep: 75 a muscle, 40 a bone, 36 a node, 110 a joint.
        work_n[n] += 75.0 * m + 40.0 * (n - 1) + 36.0 * n + 110.0 * (n >= 2 ? n - 2 : 0);
    }
    for (int big = 0; big < 2; big++) {
        ClassPlan c{0, 0, 0, 2, 0, 0.0};
        for (unsigned n = 2; n <= CE_MAX_NODES; n++) {
            if (per_n[n] == 0 || (n > small_body) != (big != 0)) continue;
            if (c.count == 0) c.first_n = n;
            c.last_n = n;
            c.count += (uint32_t)per_n[n];
            c.rows = n;
            c.mm = std::max(c.mm, mm_n[n]);
            c.work += work_n[n];
        }
        if (c.count) plans.push_back(c);
    }
    return CE_OK;
}

}  // namespace

extern "C" const char* ce_last_error(void) { return ce::g_last_error.c_str(); }

extern "C" ce_status ce_open(int device, const ce_options* options, ce_engine** out) {
    if (!out) {
        set_error("ce_open: null out");
        return CE_ERR_INVALID;
    }
    *out = nullptr;
    int count = 0;
    CE_TRY(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (device < 0 || device >= count) {
        set_error("ce_open: no CUDA device " + std::to_string(device));
        return CE_ERR_INVALID;
    }
    cudaDeviceProp prop;
    CE_TRY(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major != 10) {
        set_error(std::string("ce_open: the kernels are built for sm_100a, device is ") + prop.name);
        return CE_ERR_UNSUPPORTED;
    }
    ce_engine* e = new ce_engine();
    e->device = device;
    e->sms = prop.multiProcessorCount;
    e->smem_optin = prop.sharedMemPerBlockOptin;
    e->smem_sm = prop.sharedMemPerMultiprocessor;
    e->smem_reserved = prop.reservedSharedMemPerBlock;
    unsigned nslots = 4;
    if (options) {
        if (options->slots) nslots = options->slots;
        e->ctas_per_sm = options->ctas_per_sm;
        if (options->chunk_k) e->chunk_k = options->chunk_k;
        if (options->small_body) e->small_body = std::min<unsigned>(options->small_body, CE_MAX_NODES);
    }
    ce_status s = set_device(e);
    if (s != CE_OK) {
        delete e;
        return s;
    }
    e->slots.resize(nslots);
    for (Slot& sl : e->slots) {
        s = cuda_status(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        if (s == CE_OK) s = cuda_status(cudaStreamCreateWithFlags(&sl.side, cudaStreamNonBlocking), "cudaStreamCreate");
        if (s == CE_OK)
            s = cuda_status(cudaEventCreateWithFlags(&sl.joined, cudaEventDisableTiming), "cudaEventCreate");
        if (s == CE_OK)
            s = cuda_status(cudaEventCreateWithFlags(&sl.bucketed, cudaEventDisableTiming), "cudaEventCreate");
        if (s == CE_OK) s = cuda_status(cudaEventCreate(&sl.start), "cudaEventCreate");
        if (s == CE_OK) s = cuda_status(cudaEventCreate(&sl.stop), "cudaEventCreate");
        if (s == CE_OK) s = cuda_status(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "cudaEventCreate");
        if (s != CE_OK) {
            ce_close(e);
            return s;
        }
    }
    *out = e;
    return CE_OK;
}

extern "C" ce_status ce_close(ce_engine* e) {
    if (!e) return CE_OK;
    cudaSetDevice(e->device);
    for (Slot& sl : e->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        sl.d_lanes.release();
        sl.d_muscles.release();
        sl.d_heads.release();
        sl.d_results.release();
        sl.d_buckets.release();
        sl.d_scratch.release();
        sl.h_upload.release();
        sl.h_results.release();
        if (sl.start) cudaEventDestroy(sl.start);
        if (sl.stop) cudaEventDestroy(sl.stop);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.joined) cudaEventDestroy(sl.joined);
        if (sl.bucketed) cudaEventDestroy(sl.bucketed);
        if (sl.side) cudaStreamDestroy(sl.side);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    e->rec_frames.release();
    e->rec_staging.release();
    e->rec_lanes.release();
    e->rec_muscles.release();
    e->rec_heads.release();
    e->rec_results.release();
    e->rec_counter.release();
    e->rec_scratch.release();
    delete e;
    return CE_OK;
}

extern "C" int ce_free_slots(ce_engine* e) {
    if (!e) return 0;
    int n = 0;
    for (const Slot& sl : e->slots) n += sl.busy ? 0 : 1;
    return n;
}

extern "C" size_t ce_allocated_bytes(ce_engine* e) {
    if (!e) return 0;
    size_t b = e->rec_frames.bytes + e->rec_staging.bytes + e->rec_lanes.bytes + e->rec_muscles.bytes + e->rec_heads.bytes +
               e->rec_results.bytes + e->rec_counter.bytes + e->rec_scratch.bytes;
    for (const Slot& sl : e->slots) {
        b += sl.d_lanes.bytes + sl.d_muscles.bytes + sl.d_heads.bytes + sl.d_results.bytes + sl.d_buckets.bytes +
             sl.d_scratch.bytes;
    }
    return b;
}

extern "C" ce_status ce_release_idle(ce_engine* e) {
    if (!e) return CE_ERR_INVALID;
    CE_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    for (Slot& sl : e->slots) {
        if (sl.busy) continue;
        sl.d_lanes.release();
        sl.d_muscles.release();
        sl.d_heads.release();
        sl.d_results.release();
        sl.d_buckets.release();
        sl.d_scratch.release();
        sl.h_upload.release();
        sl.h_results.release();
    }
    return CE_OK;
}

extern "C" ce_status ce_inject_fault(ce_engine* e, uint32_t after, ce_status status) {
    if (!e) return CE_ERR_INVALID;
    e->fault_after = after;
    e->fault_status = status;
    return CE_OK;
}

extern "C" ce_status ce_submit(ce_engine* e, const ce_wave_pack* pack, const ce_world* w, uint64_t* ticket) {
    if (!e || !pack || !ticket || (pack->count && (!pack->lanes || !pack->muscles || !pack->heads))) {
        set_error("ce_submit: null argument");
        return CE_ERR_INVALID;
    }
    ce_status s = check_world(w);
    if (s != CE_OK) return s;
    if (e->fault_after) {
        if (--e->fault_after == 0) {
            set_error("ce_submit: injected fault");
            return e->fault_status;
        }
    }
    size_t si = e->slots.size();
    for (size_t i = 0; i < e->slots.size(); i++) {
        if (!e->slots[i].busy) {
            si = i;
            break;
        }
    }
    if (si == e->slots.size()) {
        set_error("ce_submit: no free slot");
        return CE_ERR_BUSY;
    }
    Slot& sl = e->slots[si];
    CE_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    std::vector<ClassPlan> plans;
    if ((s = plan_classes(pack, plans, e->small_body)) != CE_OK) return s;
    const uint32_t flags = ce_world_flags(w);
    const int rate = (int)ce::world_rate(*w);
    ce_params p;
    ce_make_params(w, 0, (uint32_t)pack->count, 0, &p);
    // Grids and scratch of the classes, which run side by side, each with its
    // own part of the slot's scratch.
    const std::vector<unsigned> grids = class_grids(e, plans, flags, rate);
    std::vector<size_t> scratch_at(plans.size());
    size_t scratch = 0;
    for (size_t c = 0; c < plans.size(); c++) {
        scratch_at[c] = scratch;
        scratch += (scratch_bytes(grids[c], plans[c].rows, plans[c].mm, false) + 255u) & ~(size_t)255u;
    }
    const size_t lanes_b = pack->lanes_len * 4, mus_b = pack->muscles_len * 4, heads_b = pack->count * 32;
    const size_t res_b = pack->count * sizeof(ce_result);
    if ((s = sl.d_lanes.ensure(lanes_b)) || (s = sl.d_muscles.ensure(mus_b)) || (s = sl.d_heads.ensure(heads_b)) ||
        (s = sl.d_buckets.ensure(cek::bucket_bytes(pack->count))) || (s = sl.d_results.ensure(res_b)) ||
        (s = sl.d_scratch.ensure(scratch)) || (s = sl.h_upload.ensure(lanes_b + mus_b + heads_b)) ||
        (s = sl.h_results.ensure(res_b))) {
        return s;
    }
    // Stage the batch in pinned memory and copy it up, chunk by chunk.
    char* up = static_cast<char*>(sl.h_upload.ptr);
    cudaStream_t st = sl.stream;
    CE_TRY(staged_upload(sl.d_lanes.ptr, up, pack->lanes, lanes_b, st), "cudaMemcpyAsync");
    CE_TRY(staged_upload(sl.d_muscles.ptr, up + lanes_b, pack->muscles, mus_b, st), "cudaMemcpyAsync");
    CE_TRY(staged_upload(sl.d_heads.ptr, up + lanes_b + mus_b, pack->heads, heads_b, st), "cudaMemcpyAsync");
    CE_TRY(cudaEventRecord(sl.start, st), "cudaEventRecord");
    const cek::Buckets bk = cek::bucket_layout(sl.d_buckets.ptr, pack->count);
    CE_TRY(cek::launch_bucket(static_cast<const uint4*>(sl.d_heads.ptr), 0u, (uint32_t)pack->count, bk, st),
           "bucketing launch");
    CE_TRY(cudaEventRecord(sl.bucketed, st), "cudaEventRecord");
    CE_TRY(cudaStreamWaitEvent(sl.side, sl.bucketed, 0), "cudaStreamWaitEvent");
    for (size_t c = 0; c < plans.size(); c++) {
        cek::KernelArgs a{};
        a.records = static_cast<const uint32_t*>(sl.d_lanes.ptr);
        a.muscles = static_cast<const float*>(sl.d_muscles.ptr);
        a.heads = static_cast<const uint4*>(sl.d_heads.ptr);
        a.results = static_cast<ce_result*>(sl.d_results.ptr);
        a.counter = bk.counters + plans[c].first_n;
        a.scratch = reinterpret_cast<float4*>(static_cast<char*>(sl.d_scratch.ptr) + scratch_at[c]);
        a.frames = nullptr;
        a.order = bk.order;
        a.bounds = bk.bounds + plans[c].first_n;
        a.work = bk.work + plans[c].first_n;
        a.queues = plans[c].last_n - plans[c].first_n + 1u;
        a.count = plans[c].count;
        a.rows = plans[c].rows;
        a.mm = plans[c].mm;
        a.frames_per_creature = 0;
        a.chunk_k = e->chunk_k;
        cek::LaunchSpec ls{plans[c].rows, plans[c].mm, flags, false, rate, grids[c], cek::kBlock,
                           c == 0 ? st : sl.side};
        CE_TRY(cek::launch_advance(ls, a, p), "advance launch");
    }
    CE_TRY(cudaEventRecord(sl.joined, sl.side), "cudaEventRecord");
    CE_TRY(cudaStreamWaitEvent(st, sl.joined, 0), "cudaStreamWaitEvent");
    CE_TRY(cudaEventRecord(sl.stop, st), "cudaEventRecord");
    CE_TRY(cudaMemcpyAsync(sl.h_results.ptr, sl.d_results.ptr, res_b, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CE_TRY(cudaEventRecord(sl.done, st), "cudaEventRecord");
    sl.busy = true;
    sl.count = pack->count;
    sl.ticket = e->next_ticket++;
    sl.submitted = std::chrono::steady_clock::now();
    e->pending.push_back(si);
    *ticket = sl.ticket;
    return CE_OK;
}

extern "C" ce_status ce_wait(ce_engine* e, int64_t timeout_us) {
    if (!e) return CE_ERR_INVALID;
    if (e->pending.empty()) return CE_ERR_TIMEOUT;
    CE_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(std::max<int64_t>(timeout_us, 0));
    for (;;) {
        for (size_t si : e->pending) {
            const cudaError_t q = cudaEventQuery(e->slots[si].done);
            if (q == cudaSuccess) return CE_OK;
            if (q != cudaErrorNotReady) return cuda_status(q, "cudaEventQuery");
        }
        if (timeout_us >= 0 && std::chrono::steady_clock::now() >= deadline) return CE_ERR_TIMEOUT;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
}

extern "C" ce_status ce_poll(ce_engine* e, int64_t timeout_us, uint64_t* ticket, ce_result* out, size_t cap,
                             size_t* n, double* busy_seconds) {
    if (!e || !ticket || !n) {
        set_error("ce_poll: null argument");
        return CE_ERR_INVALID;
    }
    *n = 0;
    if (e->pending.empty()) {
        set_error("ce_poll: nothing in flight");
        return CE_ERR_TIMEOUT;
    }
    CE_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    const size_t si = e->pending.front();
    Slot& sl = e->slots[si];
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(std::max<int64_t>(timeout_us, 0));
    for (;;) {
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) return cuda_status(q, "cudaEventQuery");
        if (timeout_us >= 0 && std::chrono::steady_clock::now() >= deadline) {
            set_error("ce_poll: timeout");
            return CE_ERR_TIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    if (out && cap < sl.count) {
        set_error("ce_poll: result buffer too small");
        return CE_ERR_INVALID;
    }
    float ms = 0.0f;
    CE_TRY(cudaEventElapsedTime(&ms, sl.start, sl.stop), "cudaEventElapsedTime");
    if (out) {
        parallel_copy(reinterpret_cast<char*>(out), static_cast<const char*>(sl.h_results.ptr),
                      sl.count * sizeof(ce_result));
    }
    *ticket = sl.ticket;
    *n = sl.count;
    if (busy_seconds) *busy_seconds = ms * 1e-3;
    sl.busy = false;
    e->pending.pop_front();
    return CE_OK;
}

extern "C" ce_status ce_record(ce_engine* e, const ce_wave_pack* pack, const ce_world* w, float* frames,
                               size_t frames_cap_floats, ce_result* results) {
    if (!e || !pack || !frames || !results || !pack->count) {
        set_error("ce_record: null argument or empty batch");
        return CE_ERR_INVALID;
    }
    ce_status s = check_world(w);
    if (s != CE_OK) return s;
    if (pack->count > CE_RECORD_MAX_CREATURES) {
        set_error("ce_record: at most " + std::to_string(CE_RECORD_MAX_CREATURES) + " creatures a recording");
        return CE_ERR_INVALID;
    }
    std::vector<ClassPlan> plans;
    if ((s = plan_classes(pack, plans)) != CE_OK) return s;
    unsigned rows = 2, mm = 0;
    for (const ClassPlan& c : plans) {
        rows = std::max(rows, c.rows);
        mm = std::max(mm, c.mm);
    }
    const uint32_t flags = ce_world_flags(w);
    const int rate = (int)ce::world_rate(*w);
    const uint32_t stride = ce_frame_stride(mm);
    ce_params p;
    ce_make_params(w, 0, (uint32_t)pack->count, stride, &p);
    const uint32_t per = ce::world_settle(*w) + p.steps + 1u;
    const size_t frame_floats = (size_t)pack->count * per * stride * 2u;
    if (frames_cap_floats < frame_floats) {
        set_error("ce_record: frame buffer too small, need " + std::to_string(frame_floats) + " floats");
        return CE_ERR_INVALID;
    }
    CE_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    // Frames are indexed by packed creature, so any grid records them; one
    // block of lanes per 128 creatures, up to what the GPU holds at once.
    const unsigned grid = grid_for(e, rows, mm, flags, true, rate, pack->count);
    const size_t lanes_b = pack->lanes_len * 4, mus_b = pack->muscles_len * 4, heads_b = pack->count * 32;
    const size_t res_b = pack->count * sizeof(ce_result);
    if ((s = e->rec_frames.ensure(frame_floats * 4)) || (s = e->rec_staging.ensure(frame_floats * 4)) ||
        (s = e->rec_lanes.ensure(lanes_b)) ||
        (s = e->rec_muscles.ensure(mus_b)) || (s = e->rec_heads.ensure(heads_b)) || (s = e->rec_results.ensure(res_b)) ||
        (s = e->rec_counter.ensure(4)) || (s = e->rec_scratch.ensure(scratch_bytes(grid, rows, mm, true)))) {
        return s;
    }
    CE_TRY(cudaMemcpy(e->rec_lanes.ptr, pack->lanes, lanes_b, cudaMemcpyHostToDevice), "cudaMemcpy");
    CE_TRY(cudaMemcpy(e->rec_muscles.ptr, pack->muscles, mus_b, cudaMemcpyHostToDevice), "cudaMemcpy");
    CE_TRY(cudaMemcpy(e->rec_heads.ptr, pack->heads, heads_b, cudaMemcpyHostToDevice), "cudaMemcpy");
    CE_TRY(cudaMemset(e->rec_counter.ptr, 0, 4), "cudaMemset");
    CE_TRY(cudaMemset(e->rec_staging.ptr, 0, frame_floats * 4), "cudaMemset");
    cek::KernelArgs a{};
    a.records = static_cast<const uint32_t*>(e->rec_lanes.ptr);
    a.muscles = static_cast<const float*>(e->rec_muscles.ptr);
    a.heads = static_cast<const uint4*>(e->rec_heads.ptr);
    a.results = static_cast<ce_result*>(e->rec_results.ptr);
    a.counter = static_cast<uint32_t*>(e->rec_counter.ptr);
    a.scratch = static_cast<float4*>(e->rec_scratch.ptr);
    a.frames = static_cast<float2*>(e->rec_staging.ptr);
    a.order = nullptr;
    a.count = (uint32_t)pack->count;
    a.rows = rows;
    a.mm = mm;
    a.frames_per_creature = per;
    a.chunk_k = 1;
    cek::LaunchSpec ls{rows, mm, flags, true, rate, grid, cek::kBlock, nullptr};
    CE_TRY(cek::launch_advance(ls, a, p), "record launch");
    CE_TRY(cek::launch_frames_to_creature_major(static_cast<const float2*>(e->rec_staging.ptr),
                                                static_cast<float2*>(e->rec_frames.ptr), (size_t)per * stride,
                                                (uint32_t)pack->count, nullptr),
           "frame transpose launch");
    CE_TRY(cudaDeviceSynchronize(), "record kernel");
    CE_TRY(cudaMemcpy(frames, e->rec_frames.ptr, frame_floats * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    CE_TRY(cudaMemcpy(results, e->rec_results.ptr, res_b, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CE_OK;
}

// The device entry's scratch: the lane slots of the grid, then the claim
// queues of `count` creatures.
namespace {
size_t slots_part(ce_engine* e, uint32_t world_flags, uint32_t rate, uint32_t max_nodes, uint32_t max_muscles) {
    const unsigned grid = grid_for(e, max_nodes, max_muscles, world_flags, false, (int)rate, (size_t)1 << 30);
    return (scratch_bytes(grid, max_nodes, max_muscles, false) + 255u) & ~(size_t)255u;
}
}  // namespace

extern "C" size_t ce_advance_scratch_bytes(ce_engine* e, uint32_t world_flags, uint32_t rate, uint32_t max_nodes,
                                           uint32_t max_muscles, uint32_t count) {
    if (!e || max_nodes < 2 || max_nodes > CE_MAX_NODES || max_muscles > CE_MAX_MUSCLES) return 0;
    if (rate != 60 && rate != 120) return 0;
    return slots_part(e, world_flags, rate, max_nodes, max_muscles) + cek::bucket_bytes(count);
}

namespace {
// The device entry, with the niche epilogue when `cells` is given.
ce_status advance_device(ce_engine* e, const uint32_t* records, const float* muscles, const uint32_t* heads,
                         ce_result* results, uint32_t* counter, void* scratch, const ce_params* params,
                         uint32_t world_flags, uint32_t rate, uint32_t max_nodes, uint32_t max_muscles,
                         void* stream, const uint8_t* shapes, const cek::MetricsArgs* niche, ce_metrics* metrics,
                         int64_t* cells, const char* what) {
    if (!e || !records || !muscles || !heads || !results || !counter || !scratch || !params) {
        set_error(std::string(what) + ": null argument");
        return CE_ERR_INVALID;
    }
    if (max_nodes < 2 || max_nodes > CE_MAX_NODES || max_muscles > CE_MAX_MUSCLES || params->steps < 1 ||
        (rate != 60 && rate != 120)) {
        set_error(std::string(what) + ": unsupported sizes");
        return CE_ERR_INVALID;
    }
    CE_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    const unsigned grid = grid_for(e, max_nodes, max_muscles, world_flags, false, (int)rate, params->count);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const cek::Buckets bk = cek::bucket_layout(
        static_cast<char*>(scratch) + slots_part(e, world_flags, rate, max_nodes, max_muscles), params->count);
    CE_TRY(cek::launch_bucket(reinterpret_cast<const uint4*>(heads), params->base, params->count, bk, st),
           "bucketing launch");
    cek::KernelArgs a{};
    a.records = records;
    a.muscles = muscles;
    a.heads = reinterpret_cast<const uint4*>(heads);
    a.results = results;
    a.counter = bk.counters;
    a.scratch = static_cast<float4*>(scratch);
    a.frames = nullptr;
    a.order = bk.order;
    a.bounds = bk.bounds;
    a.work = bk.work;
    a.queues = cek::kQueues;
    a.count = params->count;
    a.rows = max_nodes;
    a.mm = max_muscles;
    a.frames_per_creature = 0;
    a.chunk_k = e->chunk_k;
    if (cells) {
        a.shapes = shapes;
        a.metrics = metrics;
        a.cells = cells;
        a.niche = *niche;
    }
    cek::LaunchSpec ls{max_nodes, max_muscles, world_flags, false, (int)rate, grid, cek::kBlock, st};
    CE_TRY(cek::launch_advance(ls, a, *params), "advance launch");
    return CE_OK;
}
}  // namespace

extern "C" ce_status ce_advance_device(ce_engine* e, const uint32_t* records, const float* muscles,
                                       const uint32_t* heads, ce_result* results, uint32_t* counter, void* scratch,
                                       const ce_params* params, uint32_t world_flags, uint32_t rate,
                                       uint32_t max_nodes, uint32_t max_muscles, void* stream) {
    return advance_device(e, records, muscles, heads, results, counter, scratch, params, world_flags, rate,
                          max_nodes, max_muscles, stream, nullptr, nullptr, nullptr, nullptr, "ce_advance_device");
}

extern "C" ce_status ce_advance_device_cells(ce_engine* e, const uint32_t* records, const float* muscles,
                                             const uint32_t* heads, ce_result* results, uint32_t* counter,
                                             void* scratch, const ce_params* params, const ce_world* world,
                                             uint32_t max_nodes, uint32_t max_muscles, const uint8_t* shape_classes,
                                             int global_layout, ce_metrics* metrics, int64_t* cells, void* stream) {
    if (!world || !shape_classes || !cells) {
        set_error("ce_advance_device_cells: null argument");
        return CE_ERR_INVALID;
    }
    ce_status s = check_world(world);
    if (s != CE_OK) return s;
    const cek::MetricsArgs k = cek::metrics_args(world, global_layout);
    return advance_device(e, records, muscles, heads, results, counter, scratch, params, ce_world_flags(world),
                          ce::world_rate(*world), max_nodes, max_muscles, stream, shape_classes, &k, metrics, cells,
                          "ce_advance_device_cells");
}

// ------------------------------------------------------------- gradients
// A forward run kept for its backward pass (shaped like an autograd
// function: ce_forward saves, ce_backward consumes). It owns its device
// buffers and stream; one forward, then any number of backward passes.
struct ce_tape {
    ce_engine* engine = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    size_t count = 0;
    unsigned rows = 2, mm = 0, ckpts = 0, grid = 1;
    uint32_t flags = 0;
    int rate = 60;
    ce_params params{};
    DeviceBuf d_lanes, d_muscles, d_heads, d_results, d_buckets, d_ckpt, d_ends, d_scratch, d_tape, d_grads,
        d_weights, d_mismatch;
    std::vector<ce_result> results;
    double forward_seconds = 0.0, backward_seconds = 0.0;
};

namespace {

ce_status tape_time(ce_tape* t, double* seconds) {
    CE_TRY(cudaEventSynchronize(t->stop), "gradient kernels");
    float ms = 0.0f;
    CE_TRY(cudaEventElapsedTime(&ms, t->start, t->stop), "cudaEventElapsedTime");
    *seconds = ms * 1e-3;
    return CE_OK;
}

cek::KernelArgs tape_args(ce_tape* t, const cek::Buckets& bk) {
    cek::KernelArgs a{};
    a.records = static_cast<const uint32_t*>(t->d_lanes.ptr);
    a.muscles = static_cast<const float*>(t->d_muscles.ptr);
    a.heads = static_cast<const uint4*>(t->d_heads.ptr);
    a.results = static_cast<ce_result*>(t->d_results.ptr);
    a.counter = bk.counters;
    a.order = bk.order;
    a.bounds = bk.bounds;
    a.work = bk.work;
    a.queues = cek::kQueues;
    a.count = (uint32_t)t->count;
    a.rows = t->rows;
    a.mm = t->mm;
    a.chunk_k = t->engine->chunk_k;
    a.ckpt = static_cast<float*>(t->d_ckpt.ptr);
    a.ends = static_cast<uint32_t*>(t->d_ends.ptr);
    return a;
}

}  // namespace

extern "C" ce_status ce_forward(ce_engine* e, const ce_wave_pack* pack, const ce_world* w, uint32_t checkpoint_every,
                                ce_tape** out) {
    if (!e || !pack || !out || !pack->count) {
        set_error("ce_forward: null argument or empty batch");
        return CE_ERR_INVALID;
    }
    *out = nullptr;
    ce_status s = check_world(w);
    if (s != CE_OK) return s;
    const uint32_t flags = ce_world_flags(w);
    if (!cek::gradient_world(flags)) {
        set_error("ce_forward: gradients are built for the calm world and the effects worlds (without mud, "
                  "brambles or gaps)");
        return CE_ERR_UNSUPPORTED;
    }
    if (checkpoint_every != 256u) {
        set_error("ce_forward: checkpoints come every 256 substeps");
        return CE_ERR_UNSUPPORTED;
    }
    std::vector<ClassPlan> plans;
    if ((s = plan_classes(pack, plans)) != CE_OK) return s;
    for (size_t k = 0; k < pack->muscles_len / CE_MUSCLE_FIELDS; k++) {
        uint32_t sensor;
        std::memcpy(&sensor, pack->muscles + k * CE_MUSCLE_FIELDS + 16, 4);
        if (sensor != CE_NONE) {
            set_error("ce_forward: muscles with touch sensors are not differentiated");
            return CE_ERR_UNSUPPORTED;
        }
    }
    ce_tape* t = new ce_tape;
    t->engine = e;
    t->count = pack->count;
    t->flags = flags;
    for (const ClassPlan& c : plans) {
        t->rows = std::max(t->rows, c.rows);
        t->mm = std::max(t->mm, c.mm);
    }
    t->rate = (int)ce::world_rate(*w);
    if (cek::adjoint_smem_bytes(t->rows, t->mm, cek::kBlock) > e->smem_optin) {
        const std::string why = "ce_forward: bodies of " + std::to_string(t->rows) + " nodes and " +
                                std::to_string(t->mm) + " muscles need more shared memory for the backward pass "
                                "than a block has";
        ce_tape_free(t);
        set_error(why);
        return CE_ERR_UNSUPPORTED;
    }
    ce_make_params(w, 0, (uint32_t)pack->count, 0, &t->params);
    t->ckpts = (t->params.steps + 15u) / 16u;
    auto fail = [&](ce_status st) {
        ce_tape_free(t);
        return st;
    };
    if ((s = set_device(e)) != CE_OK) return fail(s);
    if ((s = cuda_status(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (s = cuda_status(cudaEventCreate(&t->start), "cudaEventCreate")) ||
        (s = cuda_status(cudaEventCreate(&t->stop), "cudaEventCreate"))) {
        return fail(s);
    }
    const size_t lanes_b = pack->lanes_len * 4, mus_b = pack->muscles_len * 4, heads_b = pack->count * 32;
    const size_t res_b = pack->count * sizeof(ce_result);
    const size_t ckpt_b = pack->count * (size_t)t->ckpts * cek::checkpoint_floats(t->rows, t->mm) * 4;
    t->grid = grid_for(e, t->rows, t->mm, flags, false, t->rate, pack->count);
    if ((s = t->d_lanes.ensure(lanes_b)) || (s = t->d_muscles.ensure(std::max<size_t>(mus_b, 4))) ||
        (s = t->d_heads.ensure(heads_b)) || (s = t->d_results.ensure(res_b)) ||
        (s = t->d_buckets.ensure(cek::bucket_bytes(pack->count))) || (s = t->d_ckpt.ensure(ckpt_b)) ||
        (s = t->d_ends.ensure(pack->count * 4)) ||
        (s = t->d_scratch.ensure(scratch_bytes(t->grid, t->rows, t->mm, false)))) {
        return fail(s);
    }
    cudaStream_t st = t->stream;
    if ((s = cuda_status(cudaMemcpyAsync(t->d_lanes.ptr, pack->lanes, lanes_b, cudaMemcpyHostToDevice, st),
                         "cudaMemcpyAsync")) ||
        (s = cuda_status(cudaMemcpyAsync(t->d_muscles.ptr, pack->muscles, mus_b, cudaMemcpyHostToDevice, st),
                         "cudaMemcpyAsync")) ||
        (s = cuda_status(cudaMemcpyAsync(t->d_heads.ptr, pack->heads, heads_b, cudaMemcpyHostToDevice, st),
                         "cudaMemcpyAsync")) ||
        (s = cuda_status(cudaMemsetAsync(t->d_ends.ptr, 0, pack->count * 4, st), "cudaMemsetAsync"))) {
        return fail(s);
    }
    const cek::Buckets bk = cek::bucket_layout(t->d_buckets.ptr, pack->count);
    if ((s = cuda_status(cudaEventRecord(t->start, st), "cudaEventRecord")) ||
        (s = cuda_status(cek::launch_bucket(static_cast<const uint4*>(t->d_heads.ptr), 0u, (uint32_t)pack->count,
                                            bk, st),
                         "bucketing launch"))) {
        return fail(s);
    }
    cek::KernelArgs a = tape_args(t, bk);
    a.scratch = static_cast<float4*>(t->d_scratch.ptr);
    cek::LaunchSpec ls{t->rows, t->mm, flags, false, t->rate, t->grid, cek::kBlock, st};
    if ((s = cuda_status(cek::launch_forward_ckpt(ls, a, t->params), "forward launch")) ||
        (s = cuda_status(cudaEventRecord(t->stop, st), "cudaEventRecord")) ||
        (s = tape_time(t, &t->forward_seconds))) {
        return fail(s);
    }
    t->results.resize(pack->count);
    if ((s = cuda_status(cudaMemcpy(t->results.data(), t->d_results.ptr, res_b, cudaMemcpyDeviceToHost),
                         "cudaMemcpy"))) {
        return fail(s);
    }
    *out = t;
    return CE_OK;
}

extern "C" ce_status ce_tape_results(ce_tape* t, ce_result* out, size_t cap) {
    if (!t || !out || cap < t->count) {
        set_error("ce_tape_results: null argument or buffer too small");
        return CE_ERR_INVALID;
    }
    std::memcpy(out, t->results.data(), t->count * sizeof(ce_result));
    return CE_OK;
}

extern "C" uint32_t ce_tape_grad_floats(ce_tape* t) { return t ? cek::grad_floats(t->rows, t->mm) : 0u; }

extern "C" ce_status ce_tape_seconds(ce_tape* t, double* forward, double* backward) {
    if (!t) return CE_ERR_INVALID;
    if (forward) *forward = t->forward_seconds;
    if (backward) *backward = t->backward_seconds;
    return CE_OK;
}

namespace {

// ce_backward and ce_backward_checked: the backward run, with the reruns'
// check when `mismatches` is not NULL.
ce_status backward(ce_tape* t, const float* dl_dfitness, float* grads, size_t cap_floats, uint32_t* mismatches) {
    if (!t || !grads) {
        set_error("ce_backward: null argument");
        return CE_ERR_INVALID;
    }
    const size_t per = cek::grad_floats(t->rows, t->mm);
    if (cap_floats < t->count * per) {
        set_error("ce_backward: gradient buffer too small, need " + std::to_string(t->count * per) + " floats");
        return CE_ERR_INVALID;
    }
    ce_status s = set_device(t->engine);
    if (s != CE_OK) return s;
    int per_sm = 0;
    if (cek::adjoint_occupancy(t->rows, t->mm, t->flags, t->rate, &per_sm) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const size_t needed = (t->count + cek::kBlock - 1) / cek::kBlock;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min(needed, (size_t)per_sm * t->engine->sms));
    const size_t slot_b = cek::adjoint_slot_bytes(grid, t->rows, t->mm);
    const size_t grads_b = t->count * per * 4;
    if ((s = t->d_scratch.ensure(slot_b)) || (s = t->d_tape.ensure(cek::adjoint_tape_bytes(grid, t->rows, t->mm))) ||
        (s = t->d_grads.ensure(grads_b)) || (s = t->d_weights.ensure(t->count * 4)) ||
        (mismatches && (s = t->d_mismatch.ensure(t->count * 4)))) {
        return s;
    }
    cudaStream_t st = t->stream;
    if (dl_dfitness) {
        CE_TRY(cudaMemcpyAsync(t->d_weights.ptr, dl_dfitness, t->count * 4, cudaMemcpyHostToDevice, st),
               "cudaMemcpyAsync");
    }
    CE_TRY(cudaMemsetAsync(t->d_grads.ptr, 0, grads_b, st), "cudaMemsetAsync");
    if (mismatches) CE_TRY(cudaMemsetAsync(t->d_mismatch.ptr, 0, t->count * 4, st), "cudaMemsetAsync");
    CE_TRY(cudaEventRecord(t->start, st), "cudaEventRecord");
    const cek::Buckets bk = cek::bucket_layout(t->d_buckets.ptr, t->count);
    CE_TRY(cek::launch_bucket(static_cast<const uint4*>(t->d_heads.ptr), 0u, (uint32_t)t->count, bk, st),
           "bucketing launch");
    cek::KernelArgs a = tape_args(t, bk);
    a.scratch = static_cast<float4*>(t->d_scratch.ptr);
    cek::LaunchSpec ls{t->rows, t->mm, t->flags, false, t->rate, grid, cek::kBlock, st};
    CE_TRY(cek::launch_adjoint(ls, a, t->params, static_cast<float4*>(t->d_tape.ptr),
                               static_cast<float*>(t->d_grads.ptr),
                               dl_dfitness ? static_cast<const float*>(t->d_weights.ptr) : nullptr,
                               mismatches ? static_cast<uint32_t*>(t->d_mismatch.ptr) : nullptr),
           "backward launch");
    CE_TRY(cudaEventRecord(t->stop, st), "cudaEventRecord");
    if ((s = tape_time(t, &t->backward_seconds)) != CE_OK) return s;
    CE_TRY(cudaMemcpy(grads, t->d_grads.ptr, grads_b, cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (mismatches) {
        CE_TRY(cudaMemcpy(mismatches, t->d_mismatch.ptr, t->count * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    }
    return CE_OK;
}

}  // namespace

extern "C" ce_status ce_backward(ce_tape* t, const float* dl_dfitness, float* grads, size_t cap_floats) {
    return backward(t, dl_dfitness, grads, cap_floats, nullptr);
}

extern "C" ce_status ce_backward_checked(ce_tape* t, const float* dl_dfitness, float* grads, size_t cap_floats,
                                         uint32_t* mismatches) {
    if (!mismatches) {
        set_error("ce_backward_checked: null mismatches");
        return CE_ERR_INVALID;
    }
    return backward(t, dl_dfitness, grads, cap_floats, mismatches);
}

extern "C" ce_status ce_tangent(ce_tape* t, const float* dstart, const float* dmuscle, const float* dfriction,
                                const float* dmass, float* dfitness) {
    if (!t || !dfitness || (!dstart && !dmuscle && !dfriction && !dmass)) {
        set_error("ce_tangent: null argument (a tape, the output and at least one direction)");
        return CE_ERR_INVALID;
    }
    if (!cek::tangent_world(t->flags)) {
        set_error("ce_tangent: the tangent-linear run is built for the gradients' worlds (calm, effects without "
                  "mud, brambles or gaps)");
        return CE_ERR_UNSUPPORTED;
    }
    if (cek::tangent_smem_bytes(t->rows, t->mm, cek::kBlock) > t->engine->smem_optin) {
        set_error("ce_tangent: bodies too large for the tangent run's shared memory");
        return CE_ERR_UNSUPPORTED;
    }
    ce_status s = set_device(t->engine);
    if (s != CE_OK) return s;
    const size_t n = t->count;
    const size_t start_b = n * 2u * t->rows * 4u, muscle_b = n * (size_t)cek::kGradMuscle * t->mm * 4u,
                 friction_b = n * (size_t)t->rows * 4u, mass_b = friction_b;
    const size_t needed = (n + cek::kBlock - 1) / cek::kBlock;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min(needed, (size_t)t->engine->sms));
    // The directions and the result live only for this call.
    struct Owned {
        DeviceBuf buf;
        ~Owned() { buf.release(); }
    } dir, out;
    const size_t dir_b =
        (dstart ? start_b : 0) + (dmuscle ? muscle_b : 0) + (dfriction ? friction_b : 0) + (dmass ? mass_b : 0);
    if ((s = t->d_scratch.ensure(cek::adjoint_slot_bytes(grid, t->rows, t->mm))) || (s = dir.buf.ensure(dir_b)) ||
        (s = out.buf.ensure(n * 4))) {
        return s;
    }
    cudaStream_t st = t->stream;
    char* at = static_cast<char*>(dir.buf.ptr);
    const float *d_start = nullptr, *d_muscle = nullptr, *d_friction = nullptr, *d_mass = nullptr;
    if (dstart) {
        CE_TRY(cudaMemcpyAsync(at, dstart, start_b, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        d_start = reinterpret_cast<const float*>(at);
        at += start_b;
    }
    if (dmuscle) {
        CE_TRY(cudaMemcpyAsync(at, dmuscle, muscle_b, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        d_muscle = reinterpret_cast<const float*>(at);
        at += muscle_b;
    }
    if (dfriction) {
        CE_TRY(cudaMemcpyAsync(at, dfriction, friction_b, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        d_friction = reinterpret_cast<const float*>(at);
        at += friction_b;
    }
    if (dmass) {
        CE_TRY(cudaMemcpyAsync(at, dmass, mass_b, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        d_mass = reinterpret_cast<const float*>(at);
    }
    CE_TRY(cudaMemsetAsync(out.buf.ptr, 0, n * 4, st), "cudaMemsetAsync");
    const cek::Buckets bk = cek::bucket_layout(t->d_buckets.ptr, n);
    CE_TRY(cek::launch_bucket(static_cast<const uint4*>(t->d_heads.ptr), 0u, (uint32_t)n, bk, st),
           "bucketing launch");
    cek::KernelArgs a = tape_args(t, bk);
    a.scratch = static_cast<float4*>(t->d_scratch.ptr);
    cek::LaunchSpec ls{t->rows, t->mm, t->flags, false, t->rate, grid, cek::kBlock, st};
    CE_TRY(cek::launch_tangent(ls, a, t->params, d_start, d_muscle, d_friction, d_mass,
                               static_cast<float*>(out.buf.ptr)),
           "tangent launch");
    CE_TRY(cudaMemcpyAsync(dfitness, out.buf.ptr, n * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CE_TRY(cudaStreamSynchronize(st), "tangent run");
    return CE_OK;
}

extern "C" ce_status ce_tape_free(ce_tape* t) {
    if (!t) return CE_OK;
    if (t->engine) cudaSetDevice(t->engine->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    for (DeviceBuf* b : {&t->d_lanes, &t->d_muscles, &t->d_heads, &t->d_results, &t->d_buckets, &t->d_ckpt,
                         &t->d_ends, &t->d_scratch, &t->d_tape, &t->d_grads, &t->d_weights, &t->d_mismatch}) {
        b->release();
    }
    if (t->start) cudaEventDestroy(t->start);
    if (t->stop) cudaEventDestroy(t->stop);
    if (t->stream) cudaStreamDestroy(t->stream);
    delete t;
    return CE_OK;
}

extern "C" ce_status ce_tape_shape(ce_tape* t, uint32_t* rows, uint32_t* muscle_slots) {
    if (!t) return CE_ERR_INVALID;
    if (rows) *rows = t->rows;
    if (muscle_slots) *muscle_slots = t->mm;
    return CE_OK;
}

extern "C" ce_status ce_tape_checkpoints(ce_tape* t, float* out, size_t cap_floats, uint32_t* per_creature) {
    if (!t || !out) return CE_ERR_INVALID;
    const size_t per = (size_t)t->ckpts * cek::checkpoint_floats(t->rows, t->mm);
    if (cap_floats < per * t->count) {
        set_error("ce_tape_checkpoints: buffer too small, need " + std::to_string(per * t->count) + " floats");
        return CE_ERR_INVALID;
    }
    ce_status s = set_device(t->engine);
    if (s != CE_OK) return s;
    // The device keeps them creature-minor ([checkpoint][float][creature]);
    // the caller gets [creature][checkpoint][float].
    std::vector<float> stage(per * t->count);
    CE_TRY(cudaMemcpy(stage.data(), t->d_ckpt.ptr, per * t->count * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (size_t c = 0; c < t->count; c++) {
        for (size_t f = 0; f < per; f++) out[c * per + f] = stage[f * t->count + c];
    }
    if (per_creature) *per_creature = t->ckpts;
    return CE_OK;
}

// ------------------------------------------------------ refinement ascent
// A batch's gradient ascent kept on the device and run as one CUDA graph:
// per step the checkpointed forward run (which scores the step's genes),
// the backward run, the gene gradients, the clipped ascent step on the
// genes and the repacking of the records from them; then a plain run scores
// the last genes. The host packs once (its plan: order, offsets and the C
// library's trig values, which the steps never change) and reads the
// fitness of every step and the final genes at the end.
struct ce_ascent {
    ce_engine* engine = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t count = 0, nodes_len = 0, bones_len = 0, muscles_len = 0;
    unsigned rows = 2, mm = 0, ckpts = 0, steps = 0;
    uint32_t flags = 0;
    int rate = 60;
    ce_params params{};
    ce_world world{};
    bool has_strength = false;
    std::vector<uint32_t> order;
    DeviceBuf d_nodes, d_bones, d_muscle_genes, d_genomes, d_strength, d_trig, d_order, d_rat, d_mat;
    DeviceBuf d_lanes, d_muscles, d_heads, d_buckets, d_ckpt, d_ends, d_scratch, d_tape, d_grads, d_mg, d_ng;
    std::vector<DeviceBuf> d_results;  // one a step, then the last genes' run
};

extern "C" ce_status ce_ascent_close(ce_ascent* a) {
    if (!a) return CE_OK;
    if (a->engine) cudaSetDevice(a->engine->device);
    if (a->stream) cudaStreamSynchronize(a->stream);
    if (a->exec) cudaGraphExecDestroy(a->exec);
    if (a->graph) cudaGraphDestroy(a->graph);
    for (DeviceBuf* b : {&a->d_nodes, &a->d_bones, &a->d_muscle_genes, &a->d_genomes, &a->d_strength, &a->d_trig,
                         &a->d_order, &a->d_rat, &a->d_mat, &a->d_lanes, &a->d_muscles, &a->d_heads, &a->d_buckets,
                         &a->d_ckpt, &a->d_ends, &a->d_scratch, &a->d_tape, &a->d_grads, &a->d_mg, &a->d_ng}) {
        b->release();
    }
    for (DeviceBuf& b : a->d_results) b.release();
    if (a->start) cudaEventDestroy(a->start);
    if (a->stop) cudaEventDestroy(a->stop);
    if (a->stream) cudaStreamDestroy(a->stream);
    delete a;
    return CE_OK;
}

extern "C" ce_status ce_ascent_open(ce_engine* e, const ce_population* pop, const ce_world* w, uint32_t steps,
                                    double step_size, size_t nodes_len, size_t bones_len, size_t muscles_len,
                                    ce_ascent** out) {
    if (!e || !pop || !out || !pop->count || steps == 0) {
        set_error("ce_ascent_open: null argument, empty population or no step");
        return CE_ERR_INVALID;
    }
    *out = nullptr;
    ce_status s = check_world(w);
    if (s != CE_OK) return s;
    const uint32_t flags = ce_world_flags(w);
    if (!cek::gradient_world(flags)) {
        set_error("ce_ascent_open: gradients are built for the calm world and the effects worlds (without mud, "
                  "brambles or gaps)");
        return CE_ERR_UNSUPPORTED;
    }
    for (size_t k = 0; k < muscles_len; k++) {
        if (pop->muscles[k].sensor != CE_NO_SENSOR) {
            set_error("ce_ascent_open: muscles with touch sensors are not differentiated");
            return CE_ERR_UNSUPPORTED;
        }
    }
    ce_ascent* a = new ce_ascent;
    auto fail = [&](ce_status st) {
        ce_ascent_close(a);
        return st;
    };
    a->engine = e;
    a->count = pop->count;
    a->nodes_len = nodes_len;
    a->bones_len = bones_len;
    a->muscles_len = muscles_len;
    a->steps = steps;
    a->flags = flags;
    a->world = *w;
    a->rate = (int)ce::world_rate(*w);
    a->has_strength = pop->strength_scale != nullptr;
    // The host plan, and a host packing for the sizes and body checks.
    const size_t n = pop->count;
    size_t lanes_len = 0, mus_len = 0;
    if ((s = ce_pack_size(pop, nullptr, n, &lanes_len, &mus_len)) != CE_OK) return fail(s);
    std::vector<uint32_t> lanes(lanes_len), heads(8 * n), rat(n), mat(n);
    std::vector<float> muscles(mus_len), trig(3 * std::max<size_t>(bones_len, 1));
    a->order.resize(n);
    if ((s = ce_pack_plan(pop, nullptr, n, w, bones_len, a->order.data(), rat.data(), mat.data(), trig.data())) !=
            CE_OK ||
        (s = ce_pack(pop, nullptr, n, w, lanes.data(), muscles.data(), heads.data(), nullptr, nullptr)) != CE_OK) {
        return fail(s);
    }
    ce_wave_pack wp{lanes.data(), lanes_len, muscles.data(), mus_len, heads.data(), n};
    std::vector<ClassPlan> plans;
    if ((s = plan_classes(&wp, plans)) != CE_OK) return fail(s);
    for (const ClassPlan& c : plans) {
        a->rows = std::max(a->rows, c.rows);
        a->mm = std::max(a->mm, c.mm);
    }
    if (cek::adjoint_smem_bytes(a->rows, a->mm, cek::kBlock) > e->smem_optin) {
        set_error("ce_ascent_open: bodies too large for the backward pass's shared memory");
        return fail(CE_ERR_UNSUPPORTED);
    }
    ce_make_params(w, 0, (uint32_t)n, 0, &a->params);
    a->ckpts = (a->params.steps + 15u) / 16u;
    if ((s = set_device(e)) != CE_OK) return fail(s);
    if ((s = cuda_status(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (s = cuda_status(cudaEventCreate(&a->start), "cudaEventCreate")) ||
        (s = cuda_status(cudaEventCreate(&a->stop), "cudaEventCreate"))) {
        return fail(s);
    }
    // Launch shapes: the forward grid as ce_forward's, the backward as ce_backward's.
    const unsigned fgrid = grid_for(e, a->rows, a->mm, flags, false, a->rate, n);
    int per_sm = 0;
    if (cek::adjoint_occupancy(a->rows, a->mm, flags, a->rate, &per_sm) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const unsigned bgrid =
        (unsigned)std::max<size_t>(1, std::min((n + cek::kBlock - 1) / cek::kBlock, (size_t)per_sm * e->sms));
    const size_t per_grad = cek::grad_floats(a->rows, a->mm);
    const size_t res_b = n * sizeof(ce_result);
    auto up = [&](DeviceBuf& d, const void* src, size_t bytes) -> ce_status {
        ce_status st = d.ensure(std::max<size_t>(bytes, 4));
        if (st != CE_OK) return st;
        return bytes ? cuda_status(cudaMemcpy(d.ptr, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") : CE_OK;
    };
    if ((s = up(a->d_nodes, pop->nodes, nodes_len * sizeof(ce_node_gene))) ||
        (s = up(a->d_bones, pop->bones, bones_len * sizeof(ce_bone_gene))) ||
        (s = up(a->d_muscle_genes, pop->muscles, muscles_len * sizeof(ce_muscle_gene))) ||
        (s = up(a->d_genomes, pop->genomes, n * sizeof(ce_genome))) ||
        (s = up(a->d_strength, pop->strength_scale, a->has_strength ? muscles_len * 4 : 0)) ||
        (s = up(a->d_trig, trig.data(), trig.size() * 4)) || (s = up(a->d_order, a->order.data(), n * 4)) ||
        (s = up(a->d_rat, rat.data(), n * 4)) || (s = up(a->d_mat, mat.data(), n * 4)) ||
        (s = up(a->d_lanes, lanes.data(), lanes_len * 4)) || (s = up(a->d_muscles, muscles.data(), mus_len * 4)) ||
        (s = up(a->d_heads, heads.data(), n * 32)) || (s = a->d_buckets.ensure(cek::bucket_bytes(n))) ||
        (s = a->d_ckpt.ensure(n * (size_t)a->ckpts * cek::checkpoint_floats(a->rows, a->mm) * 4)) ||
        (s = a->d_ends.ensure(n * 4)) ||
        (s = a->d_scratch.ensure(std::max(scratch_bytes(fgrid, a->rows, a->mm, false),
                                          cek::adjoint_slot_bytes(bgrid, a->rows, a->mm)))) ||
        (s = a->d_tape.ensure(cek::adjoint_tape_bytes(bgrid, a->rows, a->mm))) ||
        (s = a->d_grads.ensure(n * per_grad * 4)) || (s = a->d_mg.ensure(std::max<size_t>(muscles_len, 1) * 5 * 8)) ||
        (s = a->d_ng.ensure(std::max<size_t>(nodes_len, 1) * 8))) {
        return fail(s);
    }
    a->d_results.resize(steps + 1u);
    for (DeviceBuf& b : a->d_results) {
        if ((s = b.ensure(res_b)) != CE_OK) return fail(s);
    }
    ce_population dpop{static_cast<const ce_node_gene*>(a->d_nodes.ptr), static_cast<const ce_bone_gene*>(a->d_bones.ptr),
                       static_cast<const ce_muscle_gene*>(a->d_muscle_genes.ptr),
                       static_cast<const ce_genome*>(a->d_genomes.ptr), n,
                       a->has_strength ? static_cast<const float*>(a->d_strength.ptr) : nullptr};
    const cek::Buckets bk = cek::bucket_layout(a->d_buckets.ptr, n);
    auto args = [&](size_t result) {
        cek::KernelArgs k{};
        k.records = static_cast<const uint32_t*>(a->d_lanes.ptr);
        k.muscles = static_cast<const float*>(a->d_muscles.ptr);
        k.heads = static_cast<const uint4*>(a->d_heads.ptr);
        k.results = static_cast<ce_result*>(a->d_results[result].ptr);
        k.counter = bk.counters;
        k.scratch = static_cast<float4*>(a->d_scratch.ptr);
        k.order = bk.order;
        k.bounds = bk.bounds;
        k.work = bk.work;
        k.queues = cek::kQueues;
        k.count = (uint32_t)n;
        k.rows = a->rows;
        k.mm = a->mm;
        k.chunk_k = e->chunk_k;
        k.ckpt = static_cast<float*>(a->d_ckpt.ptr);
        k.ends = static_cast<uint32_t*>(a->d_ends.ptr);
        return k;
    };
    const cudaStream_t st = a->stream;
    if ((s = cuda_status(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture")))
        return fail(s);
    cudaError_t ce = cudaSuccess;
    const auto* heads_d = static_cast<const uint4*>(a->d_heads.ptr);
    for (uint32_t k = 0; k < steps && ce == cudaSuccess; k++) {
        const cek::KernelArgs ka = args(k);
        const cek::LaunchSpec fs{a->rows, a->mm, flags, false, a->rate, fgrid, cek::kBlock, st};
        const cek::LaunchSpec bs{a->rows, a->mm, flags, false, a->rate, bgrid, cek::kBlock, st};
        if (ce == cudaSuccess) ce = cek::launch_bucket(heads_d, 0u, (uint32_t)n, bk, st);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(a->d_ends.ptr, 0, n * 4, st);
        if (ce == cudaSuccess) ce = cek::launch_forward_ckpt(fs, ka, a->params);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(a->d_grads.ptr, 0, n * per_grad * 4, st);
        if (ce == cudaSuccess) ce = cek::launch_bucket(heads_d, 0u, (uint32_t)n, bk, st);
        if (ce == cudaSuccess)
            ce = cek::launch_adjoint(bs, ka, a->params, static_cast<float4*>(a->d_tape.ptr),
                                     static_cast<float*>(a->d_grads.ptr), nullptr, nullptr);
        if (ce == cudaSuccess)
            ce = cek::launch_gene_grads(dpop, static_cast<const float*>(a->d_trig.ptr),
                                        static_cast<const uint32_t*>(a->d_order.ptr), n, a->world,
                                        static_cast<const float*>(a->d_grads.ptr), a->rows, a->mm,
                                        static_cast<double*>(a->d_mg.ptr), static_cast<double*>(a->d_ng.ptr), st);
        if (ce == cudaSuccess)
            ce = cek::launch_ascend(dpop, static_cast<ce_node_gene*>(a->d_nodes.ptr),
                                    static_cast<ce_muscle_gene*>(a->d_muscle_genes.ptr),
                                    a->has_strength ? static_cast<float*>(a->d_strength.ptr) : nullptr,
                                    static_cast<const double*>(a->d_mg.ptr), static_cast<const double*>(a->d_ng.ptr),
                                    step_size, st);
        if (ce == cudaSuccess)
            ce = cek::launch_pack(dpop, static_cast<const float*>(a->d_trig.ptr),
                                  static_cast<const uint32_t*>(a->d_order.ptr),
                                  static_cast<const uint32_t*>(a->d_rat.ptr), static_cast<const uint32_t*>(a->d_mat.ptr),
                                  n, a->world, static_cast<uint32_t*>(a->d_lanes.ptr),
                                  static_cast<float*>(a->d_muscles.ptr), static_cast<uint32_t*>(a->d_heads.ptr), st);
    }
    if (ce == cudaSuccess) ce = cek::launch_bucket(heads_d, 0u, (uint32_t)n, bk, st);
    if (ce == cudaSuccess) {
        cek::KernelArgs ka = args(steps);
        ka.ckpt = nullptr;
        ka.ends = nullptr;
        const cek::LaunchSpec ls{a->rows, a->mm, flags, false, a->rate, fgrid, cek::kBlock, st};
        ce = cek::launch_advance(ls, ka, a->params);
    }
    cudaGraph_t graph = nullptr;
    const ce_status end = cuda_status(cudaStreamEndCapture(st, &graph), "cudaStreamEndCapture");
    a->graph = graph;
    if ((s = cuda_status(ce, "ascent capture")) != CE_OK) return fail(s);
    if (end != CE_OK) return fail(end);
    if ((s = cuda_status(cudaGraphInstantiate(&a->exec, a->graph, 0), "cudaGraphInstantiate")) != CE_OK) return fail(s);
    *out = a;
    return CE_OK;
}

extern "C" ce_status ce_ascent_launch(ce_ascent* a, double* seconds) {
    if (!a || !a->exec) return CE_ERR_INVALID;
    ce_status s = set_device(a->engine);
    if (s != CE_OK) return s;
    CE_TRY(cudaEventRecord(a->start, a->stream), "cudaEventRecord");
    CE_TRY(cudaGraphLaunch(a->exec, a->stream), "cudaGraphLaunch");
    CE_TRY(cudaEventRecord(a->stop, a->stream), "cudaEventRecord");
    CE_TRY(cudaEventSynchronize(a->stop), "ascent graph");
    float ms = 0.0f;
    CE_TRY(cudaEventElapsedTime(&ms, a->start, a->stop), "cudaEventElapsedTime");
    if (seconds) *seconds = ms * 1e-3;
    return CE_OK;
}

extern "C" ce_status ce_ascent_fitness(ce_ascent* a, uint32_t step, float* fitness, size_t cap) {
    if (!a || !fitness || step > a->steps || cap < a->count) {
        set_error("ce_ascent_fitness: bad step or buffer too small");
        return CE_ERR_INVALID;
    }
    ce_status s = set_device(a->engine);
    if (s != CE_OK) return s;
    std::vector<ce_result> res(a->count);
    CE_TRY(cudaMemcpy(res.data(), a->d_results[step].ptr, a->count * sizeof(ce_result), cudaMemcpyDeviceToHost),
           "cudaMemcpy");
    for (size_t c = 0; c < a->count; c++) fitness[a->order[c]] = res[c].fitness;
    return CE_OK;
}

extern "C" ce_status ce_ascent_genes(ce_ascent* a, ce_node_gene* nodes, ce_muscle_gene* muscles, float* strength) {
    if (!a || !nodes || !muscles) return CE_ERR_INVALID;
    ce_status s = set_device(a->engine);
    if (s != CE_OK) return s;
    CE_TRY(cudaMemcpy(nodes, a->d_nodes.ptr, a->nodes_len * sizeof(ce_node_gene), cudaMemcpyDeviceToHost),
           "cudaMemcpy");
    CE_TRY(cudaMemcpy(muscles, a->d_muscle_genes.ptr, a->muscles_len * sizeof(ce_muscle_gene),
                      cudaMemcpyDeviceToHost),
           "cudaMemcpy");
    if (strength && a->has_strength) {
        CE_TRY(cudaMemcpy(strength, a->d_strength.ptr, a->muscles_len * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    }
    return CE_OK;
}

// ------------------------------------------------------ generation graphs
// Several packed generations run as one CUDA graph: per generation the
// node-count bucketing and the size classes' launches (two streams joined
// by events), the generations one after another, all captured once and
// replayed by ce_graph_launch. Batches stay resident on the device.
struct ce_graph {
    ce_engine* engine = nullptr;
    cudaStream_t stream = nullptr, side = nullptr;
    std::vector<cudaEvent_t> events;
    cudaEvent_t start = nullptr, stop = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct Gen {
        DeviceBuf lanes, muscles, heads, buckets, results;
        size_t count = 0;
    };
    std::vector<Gen> gens;
    std::vector<DeviceBuf> scratch;  // one a size class, shared by the generations
};

extern "C" ce_status ce_graph_close(ce_graph* g) {
    if (!g) return CE_OK;
    if (g->engine) cudaSetDevice(g->engine->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    for (auto& gen : g->gens) {
        for (DeviceBuf* b : {&gen.lanes, &gen.muscles, &gen.heads, &gen.buckets, &gen.results}) b->release();
    }
    for (auto& b : g->scratch) b.release();
    for (cudaEvent_t ev : g->events) cudaEventDestroy(ev);
    if (g->start) cudaEventDestroy(g->start);
    if (g->stop) cudaEventDestroy(g->stop);
    if (g->side) cudaStreamDestroy(g->side);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return CE_OK;
}

extern "C" ce_status ce_graph_open(ce_engine* e, const ce_wave_pack* packs, uint32_t generations, const ce_world* w,
                                   ce_graph** out) {
    if (!e || !packs || !out || generations == 0) {
        set_error("ce_graph_open: null argument or no generation");
        return CE_ERR_INVALID;
    }
    *out = nullptr;
    ce_status s = check_world(w);
    if (s != CE_OK) return s;
    ce_graph* g = new ce_graph;
    g->engine = e;
    auto fail = [&](ce_status st) {
        ce_graph_close(g);
        return st;
    };
    if ((s = set_device(e)) != CE_OK) return fail(s);
    if ((s = cuda_status(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (s = cuda_status(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (s = cuda_status(cudaEventCreate(&g->start), "cudaEventCreate")) ||
        (s = cuda_status(cudaEventCreate(&g->stop), "cudaEventCreate"))) {
        return fail(s);
    }
    const uint32_t flags = ce_world_flags(w);
    const int rate = (int)ce::world_rate(*w);
    ce_params p;
    // Plans, grids and scratch of every generation; one scratch a class.
    std::vector<std::vector<ClassPlan>> plans(generations);
    std::vector<std::vector<unsigned>> grids(generations);
    size_t scratch_need[2] = {0, 0};
    g->gens.resize(generations);
    for (uint32_t k = 0; k < generations; k++) {
        const ce_wave_pack* pack = packs + k;
        if (!pack->count) {
            set_error("ce_graph_open: empty generation");
            return fail(CE_ERR_INVALID);
        }
        if ((s = plan_classes(pack, plans[k], e->small_body)) != CE_OK) return fail(s);
        const std::vector<unsigned> kg = class_grids(e, plans[k], flags, rate);
        for (size_t ci = 0; ci < plans[k].size(); ci++) {
            const ClassPlan& c = plans[k][ci];
            const unsigned grid = kg[ci];
            grids[k].push_back(grid);
            const size_t at = grids[k].size() - 1;
            scratch_need[at] = std::max(scratch_need[at], scratch_bytes(grid, c.rows, c.mm, false));
        }
        ce_graph::Gen& gen = g->gens[k];
        gen.count = pack->count;
        const size_t lanes_b = pack->lanes_len * 4, mus_b = pack->muscles_len * 4, heads_b = pack->count * 32;
        if ((s = gen.lanes.ensure(lanes_b)) || (s = gen.muscles.ensure(std::max<size_t>(mus_b, 4))) ||
            (s = gen.heads.ensure(heads_b)) || (s = gen.buckets.ensure(cek::bucket_bytes(pack->count))) ||
            (s = gen.results.ensure(pack->count * sizeof(ce_result)))) {
            return fail(s);
        }
        if ((s = cuda_status(cudaMemcpy(gen.lanes.ptr, pack->lanes, lanes_b, cudaMemcpyHostToDevice), "cudaMemcpy")) ||
            (s = cuda_status(cudaMemcpy(gen.muscles.ptr, pack->muscles, mus_b, cudaMemcpyHostToDevice), "cudaMemcpy")) ||
            (s = cuda_status(cudaMemcpy(gen.heads.ptr, pack->heads, heads_b, cudaMemcpyHostToDevice), "cudaMemcpy"))) {
            return fail(s);
        }
    }
    g->scratch.resize(2);
    for (int c = 0; c < 2; c++) {
        if (scratch_need[c] && (s = g->scratch[c].ensure(scratch_need[c])) != CE_OK) return fail(s);
    }
    g->events.resize(2 * generations, nullptr);
    for (auto& ev : g->events) {
        if ((s = cuda_status(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate"))) return fail(s);
    }
    // Kernel attributes are set by the occupancy queries above, before the
    // capture; the capture itself holds only stream work.
    if ((s = cuda_status(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture")))
        return fail(s);
    ce_status cap = CE_OK;
    for (uint32_t k = 0; k < generations && cap == CE_OK; k++) {
        ce_graph::Gen& gen = g->gens[k];
        ce_make_params(w, 0, (uint32_t)gen.count, 0, &p);
        const cek::Buckets bk = cek::bucket_layout(gen.buckets.ptr, gen.count);
        cap = cuda_status(cek::launch_bucket(static_cast<const uint4*>(gen.heads.ptr), 0u, (uint32_t)gen.count, bk,
                                             g->stream),
                          "bucketing launch");
        if (cap == CE_OK) cap = cuda_status(cudaEventRecord(g->events[2 * k], g->stream), "cudaEventRecord");
        if (cap == CE_OK) cap = cuda_status(cudaStreamWaitEvent(g->side, g->events[2 * k], 0), "cudaStreamWaitEvent");
        for (size_t c = 0; c < plans[k].size() && cap == CE_OK; c++) {
            cek::KernelArgs a{};
            a.records = static_cast<const uint32_t*>(gen.lanes.ptr);
            a.muscles = static_cast<const float*>(gen.muscles.ptr);
            a.heads = static_cast<const uint4*>(gen.heads.ptr);
            a.results = static_cast<ce_result*>(gen.results.ptr);
            a.counter = bk.counters + plans[k][c].first_n;
            a.scratch = static_cast<float4*>(g->scratch[c].ptr);
            a.order = bk.order;
            a.bounds = bk.bounds + plans[k][c].first_n;
            a.work = bk.work + plans[k][c].first_n;
            a.queues = plans[k][c].last_n - plans[k][c].first_n + 1u;
            a.count = plans[k][c].count;
            a.rows = plans[k][c].rows;
            a.mm = plans[k][c].mm;
            a.chunk_k = e->chunk_k;
            cek::LaunchSpec ls{plans[k][c].rows, plans[k][c].mm, flags, false, rate, grids[k][c], cek::kBlock,
                               c == 0 ? g->stream : g->side};
            cap = cuda_status(cek::launch_advance(ls, a, p), "advance launch");
        }
        if (cap == CE_OK) cap = cuda_status(cudaEventRecord(g->events[2 * k + 1], g->side), "cudaEventRecord");
        if (cap == CE_OK) cap = cuda_status(cudaStreamWaitEvent(g->stream, g->events[2 * k + 1], 0), "cudaStreamWaitEvent");
    }
    cudaGraph_t graph = nullptr;
    const ce_status end = cuda_status(cudaStreamEndCapture(g->stream, &graph), "cudaStreamEndCapture");
    g->graph = graph;
    if (cap != CE_OK) return fail(cap);
    if (end != CE_OK) return fail(end);
    // The largest tables of any launch in the graph.
    unsigned max_rows = 2, max_mm = 0;
    size_t max_smem = 0;
    for (const auto& ps : plans) {
        for (const ClassPlan& c : ps) {
            const size_t b = cek::smem_bytes(c.rows, c.mm, cek::kBlock);
            if (b > max_smem) {
                max_smem = b;
                max_rows = c.rows;
                max_mm = c.mm;
            }
        }
    }
    if ((s = cuda_status(cek::advance_reserve_smem(max_rows, max_mm, flags, false, rate, cek::kBlock),
                         "cudaFuncSetAttribute")) ||
        (s = cuda_status(cudaGraphInstantiate(&g->exec, g->graph, 0), "cudaGraphInstantiate"))) {
        return fail(s);
    }
    *out = g;
    return CE_OK;
}

extern "C" ce_status ce_graph_launch(ce_graph* g, double* seconds) {
    if (!g || !g->exec) return CE_ERR_INVALID;
    ce_status s = set_device(g->engine);
    if (s != CE_OK) return s;
    CE_TRY(cudaEventRecord(g->start, g->stream), "cudaEventRecord");
    CE_TRY(cudaGraphLaunch(g->exec, g->stream), "cudaGraphLaunch");
    CE_TRY(cudaEventRecord(g->stop, g->stream), "cudaEventRecord");
    CE_TRY(cudaEventSynchronize(g->stop), "generation graph");
    float ms = 0.0f;
    CE_TRY(cudaEventElapsedTime(&ms, g->start, g->stop), "cudaEventElapsedTime");
    if (seconds) *seconds = ms * 1e-3;
    return CE_OK;
}

extern "C" ce_status ce_graph_results(ce_graph* g, uint32_t generation, ce_result* out, size_t cap) {
    if (!g || !out || generation >= g->gens.size() || cap < g->gens[generation].count) {
        set_error("ce_graph_results: bad generation or buffer too small");
        return CE_ERR_INVALID;
    }
    ce_status s = set_device(g->engine);
    if (s != CE_OK) return s;
    CE_TRY(cudaMemcpy(out, g->gens[generation].results.ptr, g->gens[generation].count * sizeof(ce_result),
                      cudaMemcpyDeviceToHost),
           "cudaMemcpy");
    return CE_OK;
}

extern "C" ce_status ce_autotune(ce_engine* e, const ce_wave_pack* sample, const ce_world* w, ce_options* best,
                                 double* seconds) {
    if (!e || !sample || !sample->count) {
        set_error("ce_autotune: null argument or empty sample");
        return CE_ERR_INVALID;
    }
    const unsigned keep_cta = e->ctas_per_sm, keep_chunk = e->chunk_k, keep_small = e->small_body;
    std::vector<ce_result> out(sample->count);
    auto time_one = [&](double* busy) -> ce_status {
        uint64_t ticket = 0, got = 0;
        ce_status s = ce_submit(e, sample, w, &ticket);
        if (s != CE_OK) return s;
        size_t n = 0;
        return ce_poll(e, 600000000, &got, out.data(), out.size(), &n, busy);
    };
    double warm = 0.0;
    ce_status s = time_one(&warm);
    if (s != CE_OK) return s;
    double best_s = 1e300;
    unsigned best_cta = keep_cta, best_chunk = keep_chunk, best_small = keep_small;
    for (unsigned cta : {0u, 3u}) {
        for (unsigned chunk : {16u, 32u, 64u}) {
            for (unsigned small : {10u, 12u, 16u, 24u}) {
                e->ctas_per_sm = cta;
                e->chunk_k = chunk;
                e->small_body = small;
                double busy = 0.0;
                if ((s = time_one(&busy)) != CE_OK) {
                    e->ctas_per_sm = keep_cta;
                    e->chunk_k = keep_chunk;
                    e->small_body = keep_small;
                    return s;
                }
                if (busy < best_s) {
                    best_s = busy;
                    best_cta = cta;
                    best_chunk = chunk;
                    best_small = small;
                }
            }
        }
    }
    e->ctas_per_sm = best_cta;
    e->chunk_k = best_chunk;
    e->small_body = best_small;
    if (best) {
        std::memset(best, 0, sizeof *best);
        best->slots = (uint32_t)e->slots.size();
        best->ctas_per_sm = best_cta;
        best->chunk_k = best_chunk;
        best->small_body = best_small;
    }
    if (seconds) *seconds = best_s;
    return CE_OK;
}
