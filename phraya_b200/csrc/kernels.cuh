// kernels.cuh -- parameter blocks and launchers shared by the engine's .cu files.
#pragma once

#include "common.cuh"

namespace phr {

// Work list of one extension pass. Pairs are referenced through `order` (sorted by
// bucket and length); task i covers order[task_first[i] .. task_first[i] + task_count[i])
// and is run by one warp split into groups of task_group[i] lanes (one pair per group).
struct TaskList {
    const uint32_t* order;
    const uint32_t* task_first;
    const uint8_t* task_count;
    const uint8_t* task_group;
    const uint32_t* range;   // device {begin, end} of the tasks this launch runs
};

struct ExtendParams {
    const PairDesc* desc;
    PairOut* out;
    const uint32_t* packed2;    // 2-bit arena
    const uint32_t* bytes;      // byte arena (raw input, as words)
    char* text;                 // CIGAR staging text
    const uint64_t* text_off;   // per-pair staging offset
    TaskList tasks;
    uint32_t* queue_head;       // persistent-kernel work counter (zeroed before launch)
    uint8_t* scratch;           // per-warp slots
    uint64_t slot_bytes;
    uint32_t* redo_list;        // pairs whose scratch need exceeded the slot / band
    uint32_t* redo_count;
    unsigned long long* redo_need_max;
    unsigned long long* redo_need;   // need of redo_list[k] (same index), may be NULL
    const uint64_t* task_off;   // when set: task t uses scratch + task_off[t] ...
    const uint64_t* task_len;   // ... with task_len[t] bytes (redo passes); else per-warp slots
    const uint64_t* task_need;  // estimated scratch need per task (main pass), may be NULL
    int32_t engine;             // phr_engine
    int32_t full_band;          // Myers: store every block (no band)
    int32_t band_base;          // Myers: band half-width base
    phr_affine_costs costs;
    uint32_t* error_flag;       // set on an internal inconsistency (bounded loops ran out)
    int32_t big_min;            // linear WFA: pairs with qn+tn >= big_min run one per CTA (0: off)
    uint32_t big_smem;          // dynamic shared memory of the CTA-per-pair kernel (bytes)
    unsigned long long* work;   // [0] banded Myers block-columns, [1] pairs sent to redo,
                                // [2] WFA wavefront diagonals, [3] WFA LCP word compares
    int32_t lane_ckpt;          // banded Myers lane kernel: checkpoints + recomputed segments (1)
                                // or every column's records (0)
};

// task_group bit marking a redo task for the CTA-per-pair kernel
constexpr uint8_t kBigTask = 0x80;
constexpr int kBigThreads = 512;         // threads of the linear CTA-per-pair kernel (two CTAs per SM)
// most threads per CTA of the gap-affine CTA-per-pair kernel, and its default (one CTA
// per SM; the "wfa_affine_big_threads" setting launches 512 or 256, two or four per SM)
constexpr int kBigAffineThreads = 1024;
constexpr uint32_t kBigMinFrameCells = 4096;  // smallest shared frame pair worth staging

// Shared-memory words the CTA-per-pair kernel needs for the two sequences of a pair:
// each is staged by a bulk copy from the 16-byte boundary at or below its first word
// (up to 3 leading words) to the next 16-byte boundary, plus one zero word after it
// (32-bit windows read one word past the last symbol), each copy starting 16-byte
// aligned in shared memory.
__host__ __device__ __forceinline__ uint64_t big_seq_words(int qn, int tn, int mode) {
    const int per = mode == 0 ? 16 : 4;
    return static_cast<uint64_t>((qn + per - 1) / per) + static_cast<uint64_t>((tn + per - 1) / per) + 16;
}

// A WFA pair (linear or gap-affine) long enough that one warp would be latency-bound on
// it: it runs one per CTA.
__host__ __device__ __forceinline__ bool big_pair(int32_t engine, int32_t big_min, uint32_t big_smem, int qn, int tn,
                                                  int mode) {
    (void)big_smem;
    (void)mode;
    return big_min > 0 && (engine == PHR_ENGINE_WFA_LINEAR || engine == PHR_ENGINE_WFA_AFFINE) && qn + tn >= big_min;
}

// Whether the CTA kernel stages a big pair's sequences in its shared memory (with room
// left for the linear kernel's first frames); longer ones are read from global memory.
__host__ __device__ __forceinline__ bool big_staged(uint32_t big_smem, int qn, int tn, int mode) {
    return (big_seq_words(qn, tn, mode) + 2ull * kBigMinFrameCells) * 4 <= big_smem;
}

// First-pass scratch estimate of one WFA pair: room for scores up to 64 + qn/8 (linear:
// 4 bytes of history per cell plus two value frames; affine: three layers of 8-byte
// cells). A pair that needs more overflows and is redone with what it asks for.
__host__ __device__ __forceinline__ uint64_t wfa_region_est(int qn, int tn, bool affine) {
    const uint64_t L = static_cast<uint64_t>(qn + tn);
    const uint64_t s = 64 + static_cast<uint64_t>(qn) / 8;
    if (affine) return (160ull << 10) + 512ull * L;
    const uint64_t cells = s + 2 * (s * s / 2);
    return 16 * L + 4 * cells + 4096;
}

// ---------------------------------------------------------------------------
// Lane-per-pair banded Myers (global mode, 2-bit pairs; myers_lane.cu).
//
// Band of one pair: every cell (i, j) of an alignment of cost ed satisfies
// |i - j| + |(m - i) - (n - j)| <= ed, i.e. its diagonal d = j - i lies in
// [min(0, n-m) - h, max(0, n-m) + h] with h = (ed - |n - m|) / 2. With E >= ed the
// band is [dmin, dmax] below (one spare diagonal each side for the rounding of h).
// A warp runs 32 pairs; its window covers the union of their bands and holds
// P = ceil((dmax - dmin + 127) / 64) query blocks of 64 rows per column (at most nb).
// ---------------------------------------------------------------------------
constexpr int kLaneMaxSlots = 8;
// Records of kLaneColGroup consecutive columns of one lane and slot are adjacent. One
// column per group measured fastest on B200: grouping two or four columns halves the
// traceback's sector reads but the forward pass's interleaved stores cost more.
constexpr int kLaneColGroup = 1;

struct LaneBand {
    int E;
    int dmin, dmax;
};

__host__ __device__ __forceinline__ LaneBand lane_band(int m, int n, int band_base) {
    const int delta = n - m;
    const int ad = delta < 0 ? -delta : delta;
    int E = band_base + ad + (m >> 4);
    if (E > m + n) E = m + n;
    const int h = (E - ad) >> 1;
    LaneBand b;
    b.E = E;
    b.dmin = (delta < 0 ? delta : 0) - h - 1;
    b.dmax = (delta > 0 ? delta : 0) + h + 1;
    return b;
}

__host__ __device__ __forceinline__ int lane_slots(int dmin, int dmax, int nb) {
    const int p = (dmax - dmin + 127 + 63) / 64;
    return p < nb ? p : nb;
}

// Columns per traceback segment of the checkpointed lane kernel: the forward pass keeps
// the window's {VP, VN} after every kSegCols-th column, the traceback recomputes one
// segment of columns at a time into the task's scratch slot and walks it. Per 1,000,000
// pairs of 64-2048 bp: 8 columns 13.43 ms, 4 columns 13.76 ms, 2 columns 15.90 ms (the
// recompute is the same work; fewer checkpoints are fewer stores and dependent loads).
constexpr int kSegCols = 8;

// Scratch of one lane task, then one reverse-run list of (m_max + n_max + 2) words per
// lane. Record mode: 16-byte {VP, HP} records [column group][slot][lane][column in
// group] of every column. Checkpoint mode: 16-byte {VP, VN} states [checkpoint][slot]
// [lane] after columns kSegCols, 2 kSegCols, ... below n_max, then the traceback's
// segment buffer: the {VP, HP} records of one segment [column][slot][lane] (rewritten
// every segment, so it stays in the caches).
__host__ __device__ __forceinline__ uint64_t lane_ckpt_bytes(int n_max, int P) {
    const uint64_t nck = n_max > 0 ? static_cast<uint64_t>((n_max - 1) / kSegCols) : 0;
    return (nck * P * 512 + 255) & ~255ull;
}

__host__ __device__ __forceinline__ uint64_t lane_rec_bytes(int n_max, int P, int ckpt) {
    const uint64_t ng = static_cast<uint64_t>((n_max + kLaneColGroup - 1) / kLaneColGroup);
    return ckpt ? lane_ckpt_bytes(n_max, P) + static_cast<uint64_t>(kSegCols) * P * 512
                : ((ng * kLaneColGroup * P * 512 + 255) & ~255ull);
}

__host__ __device__ __forceinline__ uint64_t lane_task_need(int n_max, int m_max, int P, int ckpt = 0) {
    const uint64_t rec = lane_rec_bytes(n_max, P, ckpt);
    const uint64_t runs = (32ull * static_cast<uint64_t>(m_max + n_max + 2) * 4 + 255) & ~255ull;
    return rec + runs;
}

// Scratch of one pair in the warp-group Myers kernel with every block stored (redo).
__host__ __device__ __forceinline__ uint64_t myers_full_need(int m, int n) {
    const uint64_t nb = static_cast<uint64_t>((m + 63) >> 6);
    uint64_t need = (static_cast<uint64_t>(n) * nb * 16 + 15) & ~15ull;
    if (nb > 32) need += (static_cast<uint64_t>(n) + 15) & ~15ull;
    need += (static_cast<uint64_t>(m + n + 2) * 4 + 15) & ~15ull;
    return need;
}

void launch_myers(const ExtendParams& p, int grid, int block, cudaStream_t st);
void launch_myers_lane(const ExtendParams& p, int grid, cudaStream_t st);
// Resident blocks per SM of the lane kernel in each mode (its shared memory per warp).
int myers_lane_blocks_per_sm(int ckpt);
constexpr int kLaneThreads = 256;
void launch_wfa_linear(const ExtendParams& p, int grid, int block, cudaStream_t st);
void launch_wfa_affine(const ExtendParams& p, int grid, int block, cudaStream_t st);
void launch_wfa_linear_big(const ExtendParams& p, int grid, int mode, cudaStream_t st);
void launch_wfa_affine_big(const ExtendParams& p, int grid, int threads, int mode, cudaStream_t st);

}  // namespace phr
