// pipeline.cuh -- device structures of the align_read pipeline (pipeline.cu).
#pragma once

#include <vector>

#include "engine.cuh"

namespace phr {

// Device view of the target minimizer index: open-addressing table value -> (offset,
// count) into `pos` (target positions in sketch order, seeding.rs:31-37).
struct IndexView {
    const uint64_t* keys;
    const uint32_t* off;
    const uint32_t* cnt;   // 0 = empty slot
    const uint32_t* pos;
    uint64_t mask;
    uint32_t occ_cap;      // seed_occurrence_cap(index, 256)
};

// Seeding + chaining results of a batch of query sketches ("units"). Per-seed arrays are
// laid out unit after unit at seed_off[u]; chain records of unit u sit at the same base.
struct ChainResult {
    uint64_t n_units = 0;
    uint64_t total_seeds = 0;
    uint32_t* nseeds = nullptr;
    uint64_t* seed_off = nullptr;
    uint32_t* nchains = nullptr;
    uint64_t* smin = nullptr;
    uint64_t* skey_sorted = nullptr;
    uint32_t* sidx_sorted = nullptr;
    int32_t* f = nullptr;
    int32_t* pred = nullptr;
    int64_t* ch_score = nullptr;
    uint32_t* ch_first = nullptr;
    uint32_t* ch_len = nullptr;
    uint32_t* ch_tstart = nullptr;
    uint64_t* ch_seed_key = nullptr;
    uint64_t* ch_seed_min = nullptr;
};

// Device outputs of align_reads_device (before host packing).
struct AlignOutput {
    phr_read_result* res = nullptr;        // per read
    uint64_t* sel_pair = nullptr;          // per read: (engine slot << 56 | pair index), primary first
    uint32_t sel_cap = 0;
    phr_alignment* eng_aln[3] = {nullptr, nullptr, nullptr};   // Myers fit, WFA linear, WFA affine
    char* eng_cigar[3] = {nullptr, nullptr, nullptr};
    uint64_t eng_pairs[3] = {0, 0, 0};
    uint64_t* stats = nullptr;             // 5 outcome counters
    const uint8_t* qarena = nullptr;       // read r forward at rd_off[r], reverse complement at rd_off[n + r]
    const uint64_t* rd_off = nullptr;
    const uint32_t* rd_len = nullptr;
};

// Caller-layout results on the device (phr_read_result_arena order), kept by pack_to_host.
struct PackedDev {
    const phr_read_result* res = nullptr;
    const phr_alignment* aln = nullptr;
    const char* cigar = nullptr;
};

}  // namespace phr

struct phr_index {
    phr::Ctx* ctx = nullptr;
    phr::IndexView view{};
    uint8_t* d_target = nullptr;
    uint64_t target_len = 0;
    uint64_t n_min = 0, n_distinct = 0, device_bytes = 0;
    int alphabet = 0, k = 21, w = 11;
    void* d_block = nullptr;
    // Tandem-repeat regions of the target (TargetContext::repeat_regions), sorted and
    // non-overlapping, [start, end] with end inclusive; d_rep = starts then ends.
    std::vector<uint32_t> rep_start, rep_end;
    uint32_t* d_rep = nullptr;
    ~phr_index();
};

namespace phr {

phr_status index_create(Ctx* ctx, const uint8_t* target, uint64_t tlen, const phr_sketch* sketch, int alphabet,
                        phr_index** out);

phr_status sketch_device(Ctx* ctx, DeviceArena& A, const uint8_t* seq, const uint64_t* off, const uint32_t* len,
                         uint64_t n, int k, int w, int alphabet, uint64_t** values, uint32_t** positions,
                         uint64_t** sk_off, uint32_t** sk_n, uint64_t* total, const uint64_t* remap_off);

phr_status seed_chain_device(Ctx* ctx, DeviceArena& A, const phr_index* idx, const uint64_t* sk_val,
                             const uint32_t* sk_pos, const uint64_t* sk_off, const uint32_t* sk_n, uint64_t n_units,
                             ChainResult* C);

// Reads are device arrays; stored-sketch arrays may be NULL. Results stay on the device.
phr_status align_reads_device(Ctx* ctx, const phr_index* idx, const uint8_t* d_seq, const uint64_t* d_off,
                              const uint32_t* d_len, uint64_t n, uint64_t seq_bytes, const uint8_t* d_has_stored,
                              const uint64_t* d_s_off, const uint32_t* d_s_n, const uint64_t* d_s_val,
                              const uint32_t* d_s_pos, const phr_align_config& cfg, AlignOutput* out);

// Host batch: upload, align_reads_device, pack into the caller's arena and, when `vout`
// is given, the variant observations of every read with a result.
phr_status align_reads_host(Ctx* ctx, const phr_index* idx, const phr_read_batch* rb, const phr_align_config& cfg,
                            phr_read_result_arena* out, phr_align_stats* stats,
                            const phr_variant_config* vcfg = nullptr, phr_variant_arena* vout = nullptr);

size_t align_arena_need(uint64_t n_reads, uint64_t seq_bytes, uint64_t stored_total);

}  // namespace phr
