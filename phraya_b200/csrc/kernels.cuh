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
    int32_t engine;             // phr_engine
    int32_t full_band;          // Myers: store every block (no band)
    int32_t band_base;          // Myers: band half-width base
    phr_affine_costs costs;
    uint32_t* error_flag;       // set on an internal inconsistency (bounded loops ran out)
};

void launch_myers(const ExtendParams& p, int grid, int block, cudaStream_t st);
void launch_wfa_linear(const ExtendParams& p, int grid, int block, cudaStream_t st);
void launch_wfa_affine(const ExtendParams& p, int grid, int block, cudaStream_t st);

}  // namespace phr
