// engine.cuh -- host-side runtime of the phraya B200 engine: context, device arena,
// extension batch driver. Shared by api.cu (C ABI) and pipeline.cu (align_read).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace phr {

// Bump allocator over one growable device buffer. Reset per call; grown (free +
// cudaMalloc) only between calls, when a call's precomputed need exceeds capacity.
// Grow-only device buffer carved by take(). With a stream set, growth is stream-ordered
// (cudaFreeAsync / cudaMallocAsync on that stream): it never waits for other streams,
// so contexts sharing a device do not stall one another when one of them grows.
struct DeviceArena {
    char* base = nullptr;
    size_t cap = 0;
    size_t used = 0;
    cudaStream_t stream = nullptr;
    cudaError_t reserve(size_t need);
    void reset() { used = 0; }
    void* take(size_t bytes, size_t align = 256);
    ~DeviceArena();
};

// Tunables of one engine; filled from the autotuner cache when present.
struct EngineTune {
    int wfa_group_short = 8;     // lanes per pair for linear WFA pairs with qn+tn < wfa_long_min
    int wfa_affine_group_short = 32;  // the same for gap-affine WFA pairs (32: one pair per warp, wavefronts in registers)
    int wfa_group_long = 32;
    int wfa_long_min = 1024;     // bucket edge: qn+tn from which WFA pairs get wfa_group_long lanes
    int myers_band_base = 64;
    int block_threads = 256;
    int wfa_big_min = 4096;          // linear WFA pairs with qn+tn >= this run one per CTA (0: off)
    int wfa_big_smem = 100 << 10;    // shared memory of that kernel, bytes (two CTAs per SM)
    int max_blocks_per_sm = 4;       // resident blocks per SM of the persistent extension kernels
    int host_chunks = 4;             // chunks a large host batch is copied and aligned in (overlapped)
    int wfa_affine_big_threads = kBigAffineThreads;  // threads per CTA of the gap-affine
                                     // CTA-per-pair kernel (256, 512 or 1024; 1024 / this CTAs per SM)
    int myers_lane_ckpt = 1;         // banded Myers lane kernel: recompute segments from checkpoints (1)
                                     // or store every column's records (0)
};

struct Ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_in = nullptr;    // host -> device copies of pipelined host batches
    cudaStream_t copy_out = nullptr;   // device -> host copies of their results
    DeviceArena arena;       // per-call temporaries
    DeviceArena scratch;     // per-warp slots of the persistent kernels
    DeviceArena io;          // device copies of host inputs / outputs
    DeviceArena pipe;        // align_read pipeline state (kept across its extension calls)
    DeviceArena seeds;       // per-seed arrays of seeding/chaining, sized from the exact seed count
    size_t scratch_budget = 8ull << 30;
    std::string last_error;
    std::atomic<uint64_t> launches{0};
    EngineTune tune;
    std::string tune_file;
    bool tune_file_enable = false;
    std::mutex mu;
    uint32_t* d_counters = nullptr;   // small device scratch for counters (pinned size)
    void* h_pinned = nullptr;         // small pinned host buffer for D2H of counters
    // kernel timing (phr_ctx_set_timing)
    bool timing = false;
    struct Pending {
        std::string name;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::map<std::string, std::pair<uint64_t, double>> timings;
    std::map<std::string, uint64_t> counters;   // work counters (phr_ctx_counter)
    void begin_kernel(const char* name, cudaEvent_t* a);
    void end_kernel(const char* name, cudaEvent_t a);
    void resolve_timings();   // after a stream sync
    // Binds the arenas to `stream` (stream-ordered growth) and keeps freed blocks cached in
    // the device's default memory pool for the next growth.
    void bind_stream();
    ~Ctx();
};

// Brackets one kernel launch with timing events when enabled and counts it.
struct KernelScope {
    Ctx* ctx;
    const char* name;
    cudaEvent_t a = nullptr;
    KernelScope(Ctx* c, const char* n) : ctx(c), name(n) {
        ++ctx->launches;
        if (ctx->timing) ctx->begin_kernel(name, &a);
    }
    ~KernelScope() {
        if (ctx->timing && a) ctx->end_kernel(name, a);
    }
};

// Wall-clock time of a host-side phase (GPU waits included), recorded under its name
// in the same table as the kernels when timing is enabled.
struct HostScope {
    Ctx* ctx;
    const char* name;
    bool on;
    std::chrono::steady_clock::time_point t0;
    HostScope(Ctx* c, const char* n) : ctx(c), name(n), on(c->timing) {
        if (on) t0 = std::chrono::steady_clock::now();
    }
    void stop() {
        if (!on) return;
        on = false;
        auto& t = ctx->timings[name];
        t.first += 1;
        t.second += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    ~HostScope() { stop(); }
};

// Device-resident description of a pair batch (pointers into device memory).
struct DevPairs {
    uint64_t n = 0;
    const uint8_t* seq = nullptr;
    uint64_t seq_bytes = 0;
    const uint64_t* q_off = nullptr;
    const uint32_t* q_len = nullptr;
    const uint64_t* t_off = nullptr;
    const uint32_t* t_len = nullptr;
    const uint32_t* q_seed = nullptr;
    const uint32_t* t_seed = nullptr;
    const uint8_t* t_seq = nullptr;   // when set, targets are read from this arena instead of seq
};

// Device-resident output of a pair batch.
struct DevResults {
    phr_alignment* aln = nullptr;  // n entries (device)
    char* cigar = nullptr;         // packed text (device)
    uint64_t cigar_capacity = 0;
    uint64_t cigar_used = 0;       // written (host value) by run_extend
    uint64_t cigar_base = 0;       // added to every cigar_off (text placed after earlier chunks)
};

// Runs `engine` over the device batch, writing device results. Synchronizes the
// context stream before returning (needed to size the packed CIGAR output).
phr_status run_extend(Ctx* ctx, phr_engine engine, const DevPairs& pairs, phr_affine_costs costs,
                      DevResults* out, uint64_t sum_qt_len);

// Sum of a[i] + b[i] over device arrays of n lengths (one reduction kernel, 8 bytes back).
uint64_t device_length_sum(Ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n, cudaError_t* err);

// Upper bound of the device arena bytes run_extend needs for a batch.
size_t extend_arena_need(uint64_t n, uint64_t seq_bytes, uint64_t sum_qt_len);

phr_status set_error(Ctx* ctx, phr_status st, const std::string& msg);
phr_status cuda_status(Ctx* ctx, cudaError_t e, const char* what);

#define PHR_CUDA_TRY(ctx, expr)                                     \
    do {                                                            \
        cudaError_t _e = (expr);                                    \
        if (_e != cudaSuccess) return ::phr::cuda_status(ctx, _e, #expr); \
    } while (0)

// Extra launchers (byte-mode instantiations) defined in myers.cu / wfa.cu.
void launch_myers_bytes(const ExtendParams& p, int grid, int block, cudaStream_t st);
void launch_wfa_linear_bytes(const ExtendParams& p, int grid, int block, cudaStream_t st);
void launch_wfa_affine_bytes(const ExtendParams& p, int grid, int block, cudaStream_t st);

}  // namespace phr

// The opaque context handle of the C ABI.
struct phr_ctx {
    phr::Ctx impl;
};
