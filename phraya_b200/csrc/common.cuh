// common.cuh -- shared device/host helpers of the phraya B200 engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/phraya_gpu.h"

#define PHR_FULL_MASK 0xffffffffu

namespace phr {

// ---------------------------------------------------------------------------
// Per-pair work descriptor prepared on the device from a phr_pair_batch.
// Sequences are the SUFFIXES after the seed anchor (lib.rs:113-114).
// ---------------------------------------------------------------------------
struct PairDesc {
    uint64_t q_word;   // first word of q in the arena of `mode` (2-bit: 16 bases/word; byte: 4 bytes/word)
    uint64_t t_word;   // first word of t
    int32_t qn, tn;    // suffix lengths
    int32_t qs, ts;    // seed offsets (reported coordinates)
    int32_t mode;      // 0 = 2-bit packed pair, 1 = byte pair
    int32_t trivial;   // 1 = result already written by the prep kernel
};

// Result of one pair before CIGAR formatting.
struct PairOut {
    int32_t status;
    int32_t ed;
    int32_t t_consumed;
    int32_t affine_score;
    uint32_t n_runs;     // RLE runs written to the run buffer (reverse order)
    uint32_t text_len;   // formatted CIGAR length
};

// CIGAR run: count << 2 | op, op 0=M 1=X 2=I 3=D.
__host__ __device__ inline char op_char(uint32_t op) {
    return op == 0 ? 'M' : op == 1 ? 'X' : op == 2 ? 'I' : 'D';
}

__host__ __device__ inline uint32_t ndigits(uint32_t v) {
    uint32_t d = 1;
    while (v >= 10) {
        v /= 10;
        ++d;
    }
    return d;
}

// ---------------------------------------------------------------------------
// Packed sequence access. 2-bit mode: base i of a sequence starting at word W is
// bits [2*(i%16), 2*(i%16)+2) of word W + i/16 (A=0,C=1,G=2,T=3). Byte mode: byte i
// is byte (i%4) of word W + i/4 (little endian). Both arenas carry >= 2 words of zero
// padding after every sequence so a funnel shift may read one word past the end.
// ---------------------------------------------------------------------------
// kCoherent: the words are written earlier in the same kernel (a warp stages them and
// reads them back after __syncwarp), so they are read with coherent ld.global.cg loads;
// the read-only path (ld.global.nc) is only for arenas no kernel writes while reading.
struct Seq2 {
    static constexpr int kPerWord = 16;
    static constexpr int kBits = 2;
    static constexpr bool kCoherent = false;
};
struct SeqB {
    static constexpr int kPerWord = 4;
    static constexpr int kBits = 8;
    static constexpr bool kCoherent = false;
};
// Byte mode over words staged by the reading kernel itself.
struct SeqBc {
    static constexpr int kPerWord = 4;
    static constexpr int kBits = 8;
    static constexpr bool kCoherent = true;
};

template <class S>
__device__ __forceinline__ uint32_t seq_word(const uint32_t* p) {
    if constexpr (S::kCoherent) {
        return __ldcg(p);
    } else {
        return __ldg(p);
    }
}

// Returns 32 bits holding symbols [pos, pos + kPerWord) of the sequence at `base`.
template <class S>
__device__ __forceinline__ uint32_t load_window(const uint32_t* __restrict__ base, int32_t pos) {
    const uint32_t w = static_cast<uint32_t>(pos) / S::kPerWord;
    const uint32_t sh = (static_cast<uint32_t>(pos) % S::kPerWord) * S::kBits;
    const uint32_t lo = seq_word<S>(base + w);
    const uint32_t hi = seq_word<S>(base + w + 1);
    return __funnelshift_r(lo, hi, sh);
}

template <class S>
__device__ __forceinline__ uint32_t sym_at(const uint32_t* __restrict__ base, int32_t pos) {
    const uint32_t w = seq_word<S>(base + static_cast<uint32_t>(pos) / S::kPerWord);
    return (w >> ((static_cast<uint32_t>(pos) % S::kPerWord) * S::kBits)) & ((1u << S::kBits) - 1);
}

// Longest common prefix of q[qp..qn) and t[tp..tn) (count_matching_prefix,
// wfa_simd.rs:52-155), comparing a word of symbols per step.
template <class S>
__device__ __forceinline__ int32_t lcp(const uint32_t* __restrict__ q, int32_t qp, int32_t qn,
                                       const uint32_t* __restrict__ t, int32_t tp, int32_t tn) {
    const int32_t lim = min(qn - qp, tn - tp);
    int32_t n = 0;
    while (n < lim) {
        const uint32_t x = load_window<S>(q, qp + n) ^ load_window<S>(t, tp + n);
        if (x != 0) {
            const int32_t first = (__ffs(x) - 1) / S::kBits;
            n += first;
            return n < lim ? n : lim;
        }
        n += S::kPerWord;
    }
    return lim;
}

// extend closure of the WFA fills (wfa_simd.rs:252-262).
template <class S>
__device__ __forceinline__ int32_t wfa_extend(const uint32_t* __restrict__ q, int32_t qn,
                                              const uint32_t* __restrict__ t, int32_t tn, int32_t q_pos,
                                              int32_t k) {
    const int32_t j = q_pos - k;
    if (q_pos < 0 || q_pos >= qn || j < 0 || j >= tn) return q_pos;
    return q_pos + lcp<S>(q, q_pos, qn, t, j, tn);
}

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Inclusive prefix sum over a group of `width` lanes (power of two).
__device__ __forceinline__ uint32_t group_incl_scan(uint32_t v, int width) {
    const int l = lane_id() & (width - 1);
    for (int d = 1; d < width; d <<= 1) {
        uint32_t o = __shfl_up_sync(PHR_FULL_MASK, v, d, width);
        if (l >= d) v += o;
    }
    return v;
}

// Formats `n_runs` RLE runs (stored in REVERSE alignment order at runs[0..n_runs)) as
// CIGAR text into out[0..). Executed by all `width` lanes of a group cooperatively.
// Returns the text length (same on every lane of the group).
__device__ inline uint32_t format_runs_group(const uint32_t* runs, uint32_t n_runs, char* out, int width) {
    const int l = lane_id() & (width - 1);
    uint32_t base = 0;
    for (uint32_t c0 = 0; c0 < n_runs; c0 += width) {
        const uint32_t c = c0 + l;
        uint32_t len = 0, run = 0;
        if (c < n_runs) {
            run = runs[n_runs - 1 - c];
            len = ndigits(run >> 2) + 1;
        }
        const uint32_t incl = group_incl_scan(len, width);
        if (c < n_runs) {
            char* p = out + base + incl - len;
            uint32_t v = run >> 2;
            const uint32_t nd = len - 1;
            for (int d = static_cast<int>(nd) - 1; d >= 0; --d) {
                p[d] = static_cast<char>('0' + v % 10);
                v /= 10;
            }
            p[nd] = op_char(run & 3);
        }
        base += __shfl_sync(PHR_FULL_MASK, incl, width - 1, width);
    }
    return base;
}

// Run-length accumulator for a reverse-order traceback (one lane).
struct RunWriter {
    uint32_t* runs;
    uint32_t cap;
    uint32_t n;
    uint32_t cur_op;
    uint32_t cur_len;
    bool overflow;
    bool writer;  // only the group leader stores; the other lanes track the same state
    __device__ void init(uint32_t* r, uint32_t c, bool w = true) {
        runs = r;
        cap = c;
        n = 0;
        cur_op = 0;
        cur_len = 0;
        overflow = false;
        writer = w;
    }
    __device__ __forceinline__ void push(uint32_t op, uint32_t count) {
        if (count == 0) return;
        if (cur_len != 0 && op == cur_op) {
            cur_len += count;
            return;
        }
        flush();
        cur_op = op;
        cur_len = count;
    }
    __device__ __forceinline__ void flush() {
        if (cur_len == 0) return;
        if (n < cap) {
            if (writer) runs[n] = (cur_len << 2) | cur_op;
        } else {
            overflow = true;
        }
        ++n;
        cur_len = 0;
    }
};

}  // namespace phr
