// wfa.cu -- wavefront alignment, linear and gap-affine, with traceback (sm_100a).
//
// Semantics restated from phraya-align/src/wfa_simd.rs:
//   linear   fill_wfa :231-345, fill_wfa_fitting_impl :360-482, fitting_end_k :940-955,
//            traceback_wfa_with_tend :959-1041 / traceback_wfa :1044-1130
//   affine   fill_wfa_affine_generic :581-779, affine_pos_valid :563-569,
//            affine_traceback :785-886, levenshtein_from_cigar :893-908,
//            fill_wfa_affine_fitting_impl :919-935
//
// GPU design. One pair per group of G lanes; the diagonals of a wavefront are dealt to
// the group's lanes round-robin (diagonal k goes to lane (k + tn) mod G, the same lane
// for every layer and score, so a cell's I/D/M values never cross lanes within a step).
// Match runs are extended with 16-base (2-bit) or 4-byte word compares (common.cuh lcp).
//
// The reference keeps full-width frames (qn+tn+1 diagonals per score). Only cells
// reachable from the origin can ever be set, so each frame is stored over its
// reachable band only: linear [-min(s,tn), min(s,qn)] (the reference's own scan
// range); affine per layer, the union of its source bands shifted by the move, clipped
// to [-tn, qn]. Cells outside a band are UNSET in the reference too, so every stored
// value, op code and tie-break is identical.
//
// History per cell is what the traceback needs: the post-extension value (input to
// later scores) and the pre-extension candidate `raw` with its op code. In both
// tracebacks the match-run start is exactly `raw` (linear: edit_start = pred_pos+1 for
// ops 1/2 and pred_pos for op 3 == the winning candidate; affine: raw of each m_op).
#include <type_traits>

#include "kernels.cuh"

namespace phr {
namespace {

constexpr int32_t UNSET = INT32_MIN;

__device__ __forceinline__ uint64_t align16(uint64_t v) { return (v + 15) & ~15ull; }

template <class S>
__device__ __forceinline__ const uint32_t* seq_base(const ExtendParams& P, uint64_t word) {
    return (S::kBits == 2 ? P.packed2 : P.bytes) + word;
}

// Group-cooperative CIGAR formatting of `nr` reverse-order runs; returns text length.
__device__ uint32_t format_group(const uint32_t* runs, uint32_t nr, char* out, int G) {
    const int gl = lane_id() & (G - 1);
    const uint32_t nrmax = __reduce_max_sync(PHR_FULL_MASK, nr);
    const uint32_t rounds = (nrmax + G - 1) / G;
    uint32_t base = 0;
    for (uint32_t rr = 0; rr < rounds; ++rr) {
        const uint32_t c = rr * G + gl;
        uint32_t len = 0, run = 0;
        if (c < nr) {
            run = runs[nr - 1 - c];
            len = ndigits(run >> 2) + 1;
        }
        const uint32_t incl = group_incl_scan(len, G);
        if (c < nr) {
            char* p = out + base + incl - len;
            uint32_t v = run >> 2;
            const uint32_t nd = len - 1;
            for (int dd = static_cast<int>(nd) - 1; dd >= 0; --dd) {
                p[dd] = static_cast<char>('0' + v % 10);
                v /= 10;
            }
            p[nd] = op_char(run & 3);
        }
        base += __shfl_sync(PHR_FULL_MASK, incl, G - 1, G);
    }
    return base;
}

__device__ __forceinline__ void report_redo(const ExtendParams& P, uint32_t pid, uint64_t need) {
    const uint32_t k = atomicAdd(P.redo_count, 1u);
    P.redo_list[k] = pid;
    atomicMax(P.redo_need_max, static_cast<unsigned long long>(need));
    if (P.redo_need) P.redo_need[k] = need;
}

// 32 bits holding symbols [pos, pos + kPerWord) of a sequence in shared or global memory.
template <class S>
__device__ __forceinline__ uint32_t window_any(const uint32_t* base, int32_t pos) {
    const uint32_t w = static_cast<uint32_t>(pos) / S::kPerWord;
    const uint32_t sh = (static_cast<uint32_t>(pos) % S::kPerWord) * S::kBits;
    return __funnelshift_r(base[w], base[w + 1], sh);
}

// extend closure (wfa_simd.rs:252-262) for a valid position (0 <= qp <= qn, 0 <= qp-k <= tn).
// `words` counts the word compares (the LCP work of the roofline).
template <class S>
__device__ __forceinline__ int32_t extend_valid(const uint32_t* q, int32_t qn, const uint32_t* t, int32_t tn,
                                                int32_t qp, int32_t k, uint32_t& words) {
    const int32_t tp = qp - k;
    const int32_t lim = min(qn - qp, tn - tp);
    int32_t n = 0;
    while (n < lim) {
        ++words;
        const uint32_t x = window_any<S>(q, qp + n) ^ window_any<S>(t, tp + n);
        if (x != 0) return qp + min(n + static_cast<int32_t>(__ffs(x) - 1) / S::kBits, lim);
        n += S::kPerWord;
    }
    return qp + lim;
}

// ===========================================================================
// Linear WFA
// ===========================================================================
// cells stored before frame s: sum_{s'<s} (min(s',qn) + min(s',tn) + 1)
__device__ __forceinline__ uint64_t tri_min(int64_t s, int64_t x) {  // sum_{s'=0}^{s-1} min(s', x)
    if (s <= 0) return 0;
    if (s - 1 <= x) return static_cast<uint64_t>((s - 1) * s / 2);
    return static_cast<uint64_t>(x * (x + 1) / 2 + (s - 1 - x) * x);
}
__device__ __forceinline__ uint64_t lin_base(int64_t s, int64_t qn, int64_t tn) {
    return static_cast<uint64_t>(s) + tri_min(s, qn) + tri_min(s, tn);
}

template <class S>
__device__ void wfa_linear_group(const ExtendParams& P, const PairDesc& d, uint32_t pid, bool act, int G,
                                 uint8_t* region, uint64_t region_bytes) {
    const int gl = lane_id() & (G - 1);
    const int qn = act ? d.qn : 0, tn = act ? d.tn : 0;
    const bool fitting = act && tn > qn + qn / 2 + 10;
    const uint32_t* qb = seq_base<S>(P, d.q_word);
    const uint32_t* tb = seq_base<S>(P, d.t_word);

    // region: [runs (qn+tn+2) u32][two value frames of qn+tn+1 int32][hr u32 cells]
    // Later scores only read the previous frame's values, so values live in two
    // ping-pong frames; the traceback reads only hr = raw << 2 | op of every frame.
    uint32_t* runs = reinterpret_cast<uint32_t*>(region);
    const uint64_t runs_bytes = align16(static_cast<uint64_t>(qn + tn + 2) * 4);
    const uint64_t frame_bytes = align16(static_cast<uint64_t>(qn + tn + 1) * 4);
    const uint64_t fixed = runs_bytes + 2 * frame_bytes;
    const uint64_t cell_cap = region_bytes > fixed ? (region_bytes - fixed) / 4 : 0;
    int32_t* hv_frames = reinterpret_cast<int32_t*>(region + runs_bytes);
    uint32_t* hr = reinterpret_cast<uint32_t*>(region + fixed);
    auto hvf = [&](int sc) -> int32_t* { return hv_frames + (sc & 1) * (frame_bytes / 4); };

    // largest score whose frames fit: lin_base(s+1) <= cell_cap
    const int max_s = qn + tn;
    uint32_t wf_cells = 0, lcp_words = 0;   // work counters: band diagonals, LCP word compares
    bool alive = act;
    bool done = false, overflow = false;
    int s_end = 0, t_end = 0;

    // ---- s = 0 ----
    if (alive) {
        if (lin_base(1, qn, tn) > cell_cap) {
            overflow = true;
            alive = false;
        }
    }
    if (alive && gl == 0) {
        const int32_t v = extend_valid<S>(qb, qn, tb, tn, 0, 0, lcp_words);
        hvf(0)[0] = v;
        hr[0] = 0;
    }
    __syncwarp();
    if (alive) {
        const int32_t v0 = hvf(0)[0];
        if (!fitting) {
            if (qn - tn == 0 && v0 == qn) {  // wfa_simd.rs:277-283 (perfect match only on diagonal 0)
                done = true;
                s_end = 0;
                t_end = tn;
            }
        } else {
            // fitting_end_k over the only set diagonal k = 0 (t_end = qn)
            if (qn <= tn && v0 >= qn) {
                done = true;
                s_end = 0;
                t_end = qn;
            }
        }
    }
    int s = 1;
    for (;;) {
        const bool run = alive && !done && s <= max_s;
        if (!__any_sync(PHR_FULL_MASK, run)) break;
        int lo = 0, hi = -1;
        uint64_t base = 0, pbase = 0;
        int plo = 0, phi = -1;
        if (run) {
            lo = -min(s, tn);
            hi = min(s, qn);
            plo = -min(s - 1, tn);
            phi = min(s - 1, qn);
            base = lin_base(s, qn, tn);
            pbase = lin_base(s - 1, qn, tn);
            if (base + static_cast<uint64_t>(hi - lo + 1) > cell_cap) {
                overflow = true;
                alive = false;
            }
        }
        const bool go = run && alive;
        int best_end_k = INT32_MAX;
        if (go && gl == 0) wf_cells += static_cast<uint32_t>(hi - lo + 1);
        if (go) {
            const int32_t* pv_frame = hvf(s - 1);
            int32_t* cur_frame = hvf(s);
            // lane gl handles diagonals k with (k + tn) mod G == gl (G is a power of two)
            int k = lo + ((gl - lo - tn) & (G - 1));
            for (; k <= hi; k += G) {
                int32_t best_pos = UNSET;
                uint32_t best_op = 0;
                bool have = false;
                // candidates in order [mismatch, ins, del]; the LAST maximal one wins
                if (k >= plo && k <= phi) {
                    const int32_t pv = pv_frame[k - plo];
                    if (pv != UNSET) {
                        best_pos = pv + 1;
                        best_op = 1;
                        have = true;
                    }
                }
                if (k > -tn && k - 1 >= plo && k - 1 <= phi) {
                    const int32_t pv = pv_frame[k - 1 - plo];
                    if (pv != UNSET) {
                        const int32_t c = pv + 1;
                        if (!have || c >= best_pos) {
                            best_pos = c;
                            best_op = 2;
                            have = true;
                        }
                    }
                }
                if (k < qn && k + 1 >= plo && k + 1 <= phi) {
                    const int32_t pv = pv_frame[k + 1 - plo];
                    if (pv != UNSET) {
                        if (!have || pv >= best_pos) {
                            best_pos = pv;
                            best_op = 3;
                            have = true;
                        }
                    }
                }
                int32_t val = UNSET;
                uint32_t aux = 0;
                if (have) {
                    const int32_t j = best_pos - k;
                    if (!(best_pos < 0 || best_pos > qn || j < 0 || j > tn)) {
                        val = extend_valid<S>(qb, qn, tb, tn, best_pos, k, lcp_words);
                        aux = (static_cast<uint32_t>(best_pos) << 2) | best_op;
                    }
                }
                cur_frame[k - lo] = val;
                hr[base + (k - lo)] = aux;
                if (val != UNSET) {
                    if (!fitting) {
                        if (k == qn - tn && val >= qn) best_end_k = k;
                    } else if (k >= qn - tn && k <= qn && val >= qn) {
                        best_end_k = min(best_end_k, k);
                    }
                }
            }
        }
        // reduce the end diagonal over the group (min k = max t_end)
        int kk = best_end_k;
        for (int o = 1; o < G; o <<= 1) kk = min(kk, __shfl_xor_sync(PHR_FULL_MASK, kk, o, G));
        __syncwarp();
        if (go && kk != INT32_MAX) {
            done = true;
            s_end = s;
            t_end = qn - kk;
        }
        if (run) ++s;
    }
    {
        const unsigned cw = __reduce_add_sync(PHR_FULL_MASK, wf_cells), lw = __reduce_add_sync(PHR_FULL_MASK, lcp_words);
        if (lane_id() == 0 && P.work) {
            atomicAdd(P.work + 2, static_cast<unsigned long long>(cw));
            atomicAdd(P.work + 3, static_cast<unsigned long long>(lw));
        }
    }
    const bool failed = act && !done && !overflow;  // loop exhausted: AlignmentFailed
    if (act && overflow && gl == 0) {
        // retry with room for twice the scores reached so far (capped at the full search)
        const int64_t s2 = ::min(static_cast<long long>(max_s) + 1, 2LL * s + 64);
        const uint64_t need = fixed + lin_base(s2, qn, tn) * 4 + 64;
        report_redo(P, pid, need);
    }

    // ---- traceback (wfa_simd.rs:959-1041), one walk per group ----
    RunWriter rw;
    rw.init(runs, static_cast<uint32_t>(qn + tn + 2));
    const bool trace = act && done;
    uint32_t n_x = 0, n_gap = 0;
    if (trace && gl == 0) {
        int qi = qn, ti = t_end, k = qi - ti, ss = s_end;
        while (qi > 0 || ti > 0) {
            if (ss < 0) break;
            if (ss == 0) {
                const int mm = min(qi, ti);
                rw.push(0, static_cast<uint32_t>(mm));
                qi -= mm;
                ti -= mm;
                break;
            }
            const int lo = -min(ss, tn);
            const uint32_t aux = hr[lin_base(ss, qn, tn) + (k - lo)];
            const uint32_t op = aux & 3;
            const int32_t edit_start = static_cast<int32_t>(aux >> 2);
            const int mc = qi - edit_start;
            if (mc > 0) {
                rw.push(0, static_cast<uint32_t>(mc));
                qi -= mc;
                ti -= mc;
            }
            if (op == 1) {
                rw.push(1, 1);
                --qi;
                --ti;
                ++n_x;
            } else if (op == 2) {
                rw.push(3, 1);  // 'D': query advances
                --qi;
                ++n_gap;
                k -= 1;
            } else if (op == 3) {
                rw.push(2, 1);  // 'I': target advances
                --ti;
                ++n_gap;
                k += 1;
            }
            --ss;
        }
        rw.flush();
    }
    const uint32_t nr = __shfl_sync(PHR_FULL_MASK, rw.n, lane_id() & ~(G - 1));
    const bool ovf = __shfl_sync(PHR_FULL_MASK, rw.overflow ? 1 : 0, lane_id() & ~(G - 1)) != 0;
    __syncwarp();
    const uint32_t nr_fmt = (trace && !ovf) ? nr : 0;
    char* out = act ? P.text + P.text_off[pid] : nullptr;
    const uint32_t tl = format_group(runs, nr_fmt, out, G);
    if (act && gl == 0) {
        if (trace && !ovf) {
            PairOut o;
            o.status = PHR_OK;
            o.ed = s_end;
            o.t_consumed = t_end;
            o.affine_score = 0;
            o.n_runs = nr;
            o.text_len = tl;
            P.out[pid] = o;
        } else if (failed) {
            PairOut o = {};
            o.status = PHR_ALIGNMENT_FAILED;
            P.out[pid] = o;
        } else if (trace && ovf) {
            atomicOr(P.error_flag, 2u);
        }
    }
}

// ===========================================================================
// Linear WFA, one CTA per pair (long pairs)
// ===========================================================================
// A warp-per-pair wavefront on a long, divergent pair is latency-bound: every cell is a
// chain of dependent loads (previous frame, both sequences) and one warp cannot hide
// them. Here a CTA of kBigThreads threads takes one pair; both sequences and, while they
// fit, the two value frames live in shared memory; the history (hr) goes to the pair's
// scratch region with coalesced stores (consecutive diagonals on consecutive threads).
// Frames that outgrow shared memory move to the region's global frames, the same layout
// the warp kernel uses, so scratch needs and the redo rule are identical.

// Bulk asynchronous copies (the TMA unit's untiled cp.async.bulk, no multicast) of the
// pair's sequences into shared memory, completing on an mbarrier.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// `bytes` (a positive multiple of 16) from 16-byte aligned global memory to 16-byte
// aligned shared memory; completion is counted on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// Bounded wait for phase `parity` of `bar` (each try itself blocks for a while); false
// when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 32 bits holding symbols [pos, pos + kPerWord) of a sequence staged in shared memory.
template <class S>
__device__ __forceinline__ uint32_t window_sm(const uint32_t* base, int32_t pos) {
    const uint32_t w = static_cast<uint32_t>(pos) / S::kPerWord;
    const uint32_t sh = (static_cast<uint32_t>(pos) % S::kPerWord) * S::kBits;
    return __funnelshift_r(base[w], base[w + 1], sh);
}

template <class S>
__device__ __forceinline__ int32_t extend_sm(const uint32_t* q, int32_t qn, const uint32_t* t, int32_t tn,
                                             int32_t q_pos, int32_t k, uint32_t& words) {
    const int32_t j = q_pos - k;
    if (q_pos < 0 || q_pos >= qn || j < 0 || j >= tn) return q_pos;
    const int32_t lim = min(qn - q_pos, tn - j);
    int32_t n = 0;
    while (n < lim) {
        ++words;
        const uint32_t x = window_sm<S>(q, q_pos + n) ^ window_sm<S>(t, j + n);
        if (x != 0) {
            n += (__ffs(x) - 1) / S::kBits;
            return q_pos + (n < lim ? n : lim);
        }
        n += S::kPerWord;
    }
    return q_pos + lim;
}

// Stages a pair's two sequences in the CTA's shared memory `sm`, each followed by one
// zero word (32-bit windows read one word past the last symbol): one bulk copy per
// sequence from the 16-byte boundary at or below its first word to the next 16-byte
// boundary after its last (the arenas are 256-byte aligned and hold four padding words
// after every sequence, so both ends stay inside them). Called by every thread of the
// CTA; returns the first free word after the staged sequences (16-byte aligned). A pair
// too long for the shared memory (big_staged) is read in place: 0 is returned and the
// output pointers are the global ones.
template <class S>
__device__ uint32_t stage_pair_cta(const ExtendParams& P, const PairDesc& d, uint32_t* sm, uint64_t* bar,
                                   uint32_t& phase, uint32_t** sq_out, uint32_t** st_out) {
    const int tid = threadIdx.x;
    const uint32_t* gq = seq_base<S>(P, d.q_word);
    const uint32_t* gt = seq_base<S>(P, d.t_word);
    if (!big_staged(P.big_smem, d.qn, d.tn, S::kBits == 2 ? 0 : 1)) {
        // too long for shared memory: read in place (each sequence is followed by padding
        // words in its arena, and every match extension is clamped to the sequence ends)
        *sq_out = const_cast<uint32_t*>(gq);
        *st_out = const_cast<uint32_t*>(gt);
        return 0;
    }
    const int qw = (d.qn + S::kPerWord - 1) / S::kPerWord;
    const int tw = (d.tn + S::kPerWord - 1) / S::kPerWord;
    const int lead_q = static_cast<int>((reinterpret_cast<uintptr_t>(gq) & 15) >> 2);
    const int lead_t = static_cast<int>((reinterpret_cast<uintptr_t>(gt) & 15) >> 2);
    const uint32_t t_base = static_cast<uint32_t>(lead_q + qw + 1 + 3) & ~3u;
    uint32_t* sq = sm + lead_q;
    uint32_t* st = sm + t_base + lead_t;
    const uint32_t nb_q = static_cast<uint32_t>((lead_q + qw + 3) & ~3) * 4;
    const uint32_t nb_t = static_cast<uint32_t>((lead_t + tw + 3) & ~3) * 4;
    if (tid == 0) {
        // order this CTA's earlier shared-memory accesses before the async writes
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(bar, nb_q + nb_t);
        if (nb_q) bulk_copy_g2s(sm, gq - lead_q, nb_q, bar);
        if (nb_t) bulk_copy_g2s(sm + t_base, gt - lead_t, nb_t, bar);
    }
    if (!mbar_wait_bounded(bar, phase)) {
        atomicOr(P.error_flag, 32u);
        mbar_wait_bounded(bar, phase);  // the copies may still land: wait once more, bounded
    }
    phase ^= 1u;
    if (tid == 0) {
        sq[qw] = 0u;
        st[tw] = 0u;
    }
    *sq_out = sq;
    *st_out = st;
    return (t_base + static_cast<uint32_t>(lead_t + tw + 1) + 3) & ~3u;
}

template <class S>
__device__ void wfa_linear_cta(const ExtendParams& P, const PairDesc& d, uint32_t pid, uint8_t* region,
                               uint64_t region_bytes, uint32_t* sm, uint32_t sm_words, int* sh_end, uint64_t* bar,
                               uint32_t& phase) {
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int qn = d.qn, tn = d.tn;
    const bool fitting = tn > qn + qn / 2 + 10;

    // ---- stage both sequences (plus one zero word each) in shared memory ----
    uint32_t *sq, *st;
    const uint32_t fr_off = stage_pair_cta<S>(P, d, sm, bar, phase, &sq, &st);
    const int qw = (qn + S::kPerWord - 1) / S::kPerWord;
    const int tw = (tn + S::kPerWord - 1) / S::kPerWord;
    const uint32_t fcap = sm_words > fr_off ? (sm_words - fr_off) / 2 : 0;  // cells per shared frame
    int32_t* sfr = reinterpret_cast<int32_t*>(sm + fr_off);

    // ---- region layout, as in wfa_linear_group ----
    uint32_t* runs = reinterpret_cast<uint32_t*>(region);
    const uint64_t runs_bytes = align16(static_cast<uint64_t>(qn + tn + 2) * 4);
    const uint64_t frame_bytes = align16(static_cast<uint64_t>(qn + tn + 1) * 4);
    const uint64_t fixed = runs_bytes + 2 * frame_bytes;
    const uint64_t cell_cap = region_bytes > fixed ? (region_bytes - fixed) / 4 : 0;
    int32_t* gfr = reinterpret_cast<int32_t*>(region + runs_bytes);
    uint32_t* hr = reinterpret_cast<uint32_t*>(region + fixed);
    bool global_frames = false;
    auto frame = [&](int sc) -> int32_t* {
        return global_frames ? gfr + (sc & 1) * (frame_bytes / 4) : sfr + (sc & 1) * fcap;
    };

    if (tid < 3) sh_end[tid] = INT32_MAX;
    const int max_s = qn + tn;
    bool done = false, overflow = false;
    uint64_t wf_cells = 0;   // band diagonals of the scores computed
    uint32_t lcp_words = 0;  // this thread's word compares of match extension
    int s_end = 0, t_end = 0, s = 1;
    if (lin_base(1, qn, tn) > cell_cap) overflow = true;
    if (fcap < 1) global_frames = true;
    __syncthreads();
    if (!overflow) {
        if (tid == 0) {
            frame(0)[0] = extend_sm<S>(sq, qn, st, tn, 0, 0, lcp_words);
            hr[0] = 0;
        }
        __syncthreads();
        const int32_t v0 = frame(0)[0];
        if (!fitting) {
            if (qn - tn == 0 && v0 == qn) {  // wfa_simd.rs:277-283
                done = true;
                t_end = tn;
            }
        } else if (qn <= tn && v0 >= qn) {
            done = true;
            t_end = qn;
        }
        for (; !done && s <= max_s; ++s) {
            const int lo = -min(s, tn), hi = min(s, qn);
            const int plo = -min(s - 1, tn), phi = min(s - 1, qn);
            const uint64_t base = lin_base(s, qn, tn);
            const int width = hi - lo + 1;
            if (base + static_cast<uint64_t>(width) > cell_cap) {
                overflow = true;
                break;
            }
            wf_cells += static_cast<uint64_t>(width);
            if (!global_frames && static_cast<uint32_t>(width) > fcap) {
                // frames outgrow shared memory: continue on the region's global frames
                const int32_t* src = frame(s - 1);
                int32_t* dst = gfr + ((s - 1) & 1) * (frame_bytes / 4);
                for (int i = tid; i < phi - plo + 1; i += nthr) dst[i] = src[i];
                global_frames = true;
                __syncthreads();
            }
            const int32_t* pv_frame = frame(s - 1);
            int32_t* cur_frame = frame(s);
            if (tid == 0) sh_end[(s + 1) % 3] = INT32_MAX;
            int my_end = INT32_MAX;
            for (int k = lo + tid; k <= hi; k += nthr) {
                int32_t best_pos = UNSET;
                uint32_t best_op = 0;
                bool have = false;
                // candidates in order [mismatch, ins, del]; the LAST maximal one wins
                if (k >= plo && k <= phi) {
                    const int32_t pv = pv_frame[k - plo];
                    if (pv != UNSET) {
                        best_pos = pv + 1;
                        best_op = 1;
                        have = true;
                    }
                }
                if (k > -tn && k - 1 >= plo && k - 1 <= phi) {
                    const int32_t pv = pv_frame[k - 1 - plo];
                    if (pv != UNSET) {
                        const int32_t c = pv + 1;
                        if (!have || c >= best_pos) {
                            best_pos = c;
                            best_op = 2;
                            have = true;
                        }
                    }
                }
                if (k < qn && k + 1 >= plo && k + 1 <= phi) {
                    const int32_t pv = pv_frame[k + 1 - plo];
                    if (pv != UNSET) {
                        if (!have || pv >= best_pos) {
                            best_pos = pv;
                            best_op = 3;
                            have = true;
                        }
                    }
                }
                int32_t val = UNSET;
                uint32_t aux = 0;
                if (have) {
                    const int32_t j = best_pos - k;
                    if (!(best_pos < 0 || best_pos > qn || j < 0 || j > tn)) {
                        val = extend_sm<S>(sq, qn, st, tn, best_pos, k, lcp_words);
                        aux = (static_cast<uint32_t>(best_pos) << 2) | best_op;
                    }
                }
                cur_frame[k - lo] = val;
                hr[base + (k - lo)] = aux;
                if (val != UNSET) {
                    if (!fitting) {
                        if (k == qn - tn && val >= qn) my_end = k;
                    } else if (k >= qn - tn && k <= qn && val >= qn) {
                        my_end = min(my_end, k);
                    }
                }
            }
            my_end = __reduce_min_sync(PHR_FULL_MASK, my_end);
            if ((tid & 31) == 0 && my_end != INT32_MAX) atomicMin(&sh_end[s % 3], my_end);
            __syncthreads();
            const int kk = sh_end[s % 3];
            if (kk != INT32_MAX) {
                done = true;
                s_end = s;
                t_end = qn - kk;
            }
        }
    }
    if (done && s_end == 0) s = 0;
    if (P.work) {  // work counters: band diagonals (the same in every thread), LCP word compares
        if (tid == 0) atomicAdd(P.work + 2, static_cast<unsigned long long>(wf_cells));
        if (lcp_words) atomicAdd(P.work + 3, static_cast<unsigned long long>(lcp_words));
    }
    const bool failed = !done && !overflow;
    if (overflow) {  // CTA-uniform
        // Scratch for the redo: extrapolate the final score from the progress so far (the
        // furthest query offset the last score reached; the wavefront advances about in
        // proportion to the score), plus a quarter as margin, so that one redo usually
        // suffices; at least twice the scores reached, at most the whole search.
        int vm = 0;
        if (s >= 2) {
            const int32_t* pf = frame(s - 1);
            const int plo = -min(s - 1, tn), phi = min(s - 1, qn);
            for (int k = plo + tid; k <= phi; k += nthr) vm = max(vm, pf[k - plo]);
        }
        vm = __reduce_max_sync(PHR_FULL_MASK, vm);
        __syncthreads();  // every thread is done with the end flags
        if (tid == 0) sh_end[0] = 0;
        __syncthreads();
        if ((tid & 31) == 0) atomicMax(&sh_end[0], vm);
        __syncthreads();
        if (tid == 0) {
            const int64_t reach = sh_end[0];
            int64_t s2 = 2LL * s + 64;
            if (reach > 0) {
                int64_t est = static_cast<int64_t>(s) * qn / reach;
                est += est / 4 + 64;
                s2 = ::max(s2, est);
            }
            s2 = ::min(static_cast<int64_t>(max_s) + 1, s2);
            report_redo(P, pid, fixed + lin_base(s2, qn, tn) * 4 + 64);
        }
    }

    // ---- traceback (wfa_simd.rs:959-1041) by thread 0, formatting by warp 0 ----
    if (tid < 32) {
        RunWriter rw;
        rw.init(runs, static_cast<uint32_t>(qn + tn + 2));
        if (done && tid == 0) {
            int qi = qn, ti = t_end, k = qi - ti, ss = s_end;
            while (qi > 0 || ti > 0) {
                if (ss < 0) break;
                if (ss == 0) {
                    const int mm = min(qi, ti);
                    rw.push(0, static_cast<uint32_t>(mm));
                    qi -= mm;
                    ti -= mm;
                    break;
                }
                const int lo = -min(ss, tn);
                const uint32_t aux = hr[lin_base(ss, qn, tn) + (k - lo)];
                const uint32_t op = aux & 3;
                const int32_t edit_start = static_cast<int32_t>(aux >> 2);
                const int mc = qi - edit_start;
                if (mc > 0) {
                    rw.push(0, static_cast<uint32_t>(mc));
                    qi -= mc;
                    ti -= mc;
                }
                if (op == 1) {
                    rw.push(1, 1);
                    --qi;
                    --ti;
                } else if (op == 2) {
                    rw.push(3, 1);
                    --qi;
                    k -= 1;
                } else if (op == 3) {
                    rw.push(2, 1);
                    --ti;
                    k += 1;
                }
                --ss;
            }
            rw.flush();
        }
        const uint32_t nr = __shfl_sync(PHR_FULL_MASK, rw.n, 0);
        const bool ovf = __shfl_sync(PHR_FULL_MASK, rw.overflow ? 1 : 0, 0) != 0;
        __syncwarp();
        const uint32_t tl = format_group(runs, (done && !ovf) ? nr : 0, P.text + P.text_off[pid], 32);
        if (tid == 0) {
            if (done && !ovf) {
                PairOut o;
                o.status = PHR_OK;
                o.ed = s_end;
                o.t_consumed = t_end;
                o.affine_score = 0;
                o.n_runs = nr;
                o.text_len = tl;
                P.out[pid] = o;
            } else if (failed) {
                PairOut o = {};
                o.status = PHR_ALIGNMENT_FAILED;
                P.out[pid] = o;
            } else if (done && ovf) {
                atomicOr(P.error_flag, 2u);
            }
        }
    }
    __syncthreads();  // shared memory and the task slot are reused by the next pair
}

template <class S>
__global__ void __launch_bounds__(kBigThreads, 2) wfa_linear_big_kernel(ExtendParams P) {
    extern __shared__ __align__(16) uint32_t big_sm[];
    __shared__ uint32_t sh_task;
    __shared__ int sh_end[3];
    __shared__ __align__(8) uint64_t sh_bar;
    const uint32_t sm_words = P.big_smem / 4;
    uint32_t phase = 0;  // parity of sh_bar's current phase, the same in every thread
    if (threadIdx.x == 0) mbar_init(&sh_bar, 1);
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) sh_task = P.tasks.range[0] + atomicAdd(P.queue_head, 1u);
        __syncthreads();
        const uint32_t task = sh_task;
        __syncthreads();
        if (task >= P.tasks.range[1]) break;
        if (!(P.tasks.task_group[task] & kBigTask)) continue;
        const uint32_t pid = P.tasks.order[P.tasks.task_first[task]];
        const PairDesc d = P.desc[pid];
        if (d.mode != (S::kBits == 2 ? 0 : 1)) continue;
        wfa_linear_cta<S>(P, d, pid, P.scratch + P.task_off[task], P.task_len[task] & ~15ull, big_sm, sm_words,
                          sh_end, &sh_bar, phase);
    }
}

// ===========================================================================
// Gap-affine WFA
// ===========================================================================
struct LayerBand {
    int lo, hi;          // empty when lo > hi
    uint64_t base;       // first cell of this layer/score in the cell arrays
};

// Frame directory entry per score s: M, I, D bands.
struct AffDir {
    LayerBand L[3];
};


// Directory entry of one score with 32-bit cell indices, kept in a per-group shared
// ring for the recurrence (which looks back at most max(X, O + E) scores).
struct SBand {
    int lo, hi;
    uint32_t base;
};
struct SDir {
    SBand L[3];
};
constexpr int kAffRing = 16;          // scores per ring (power of two)
constexpr int kAffRingGroups = 4;     // rings per warp: groups of 8 or more lanes
// Shared sequence words per warp, split among its groups. Zero: the sequences are read
// through L1, which keeps more of the recent wavefront cells when shared memory is small
// (staging both sequences measured slower: it took L1 capacity from the cells).
constexpr int kWarpSeqWords = 0;

// affine_pos_valid (wfa_simd.rs:563-569); UNSET and UNSET + 1 are negative, so invalid.
__device__ __forceinline__ bool pos_ok(int32_t pos, int k, int qn, int tn) {
    return static_cast<uint32_t>(pos) <= static_cast<uint32_t>(qn) &&
           static_cast<uint32_t>(pos) - static_cast<uint32_t>(k) <= static_cast<uint32_t>(tn);
}

// Traceback (wfa_simd.rs:785-886) of a finished affine wavefront and the pair's result:
// history in `auxs` through the score directory below `dir_top`. Called by all lanes of
// the warp; the leader of each group of G lanes walks its pair.
// With row_g > 0 the history is the register kernel's: one word per (score, k) at
// auxs[(score / row_g) * row_w + k - row_lo] holding raw << 4 | dop << 3 | iop << 2 | mop
// (all three layers' history of the cell), no directory read. With `folded` the same
// words are laid out per score over its M band, found through the directory (the CTA
// kernel).
__device__ void affine_finish(const ExtendParams& P, uint32_t pid, bool act, int G, int qn, int tn, int X, int O,
                              int E, uint32_t* runs, const uint32_t* auxs, const AffDir* dir_top, bool done,
                              bool failed, int s_end, int t_end, int k_end, int layer_end, int row_g = 0,
                              int row_w = 0, int row_lo = 0, const uint32_t* sh_hist = nullptr, int sh_rows = 0,
                              bool folded = false) {
    const int gl = lane_id() & (G - 1);
    auto dir_at = [&](int64_t sc) -> const AffDir& { return dir_top[-1 - sc]; };
    auto aux_at = [&](int ss, int layer, int k) -> uint32_t {
        if (folded) {
            // one word per diagonal of the score's M band (the CTA kernel's layout)
            const LayerBand& b = dir_at(ss).L[0];
            const uint32_t w = auxs[b.base + (k - b.lo)];
            return layer == 0 ? (((w >> 4) << 2) | (w & 3u)) : (w >> (layer + 1)) & 1u;
        }
        if (row_g > 0) {
            // rows below sh_rows of diagonals -16..15 live in shared memory
            // row of score ss (a multiple of g; g is 1 or 2 for the specialised costs)
            const int rr = row_g == 1 ? ss : row_g == 2 ? (ss >> 1) : ss / row_g;
            const uint32_t w = (rr < sh_rows && static_cast<unsigned>(k + 16) < 32u)
                                   ? sh_hist[rr * 32 + (k + 16)]
                                   : auxs[static_cast<uint64_t>(rr) * row_w + (k - row_lo)];
            return layer == 0 ? (((w >> 4) << 2) | (w & 3u)) : (w >> (layer + 1)) & 1u;
        }
        const LayerBand& b = dir_at(ss).L[layer];
        return auxs[b.base + (k - b.lo)];
    };
    RunWriter rw;
    rw.init(runs, static_cast<uint32_t>(qn + tn + 2));
    const bool trace = act && done;
    uint32_t n_edit = 0;
    if (trace && gl == 0) {
        int qi = qn, ti = t_end, k = k_end, ss = s_end, layer = layer_end;
        int guard = 4 * (qn + tn) + 16;
        while ((qi > 0 || ti > 0) && guard-- > 0) {
            if (ss == 0) {
                const int mm = min(qi, ti);
                rw.push(0, static_cast<uint32_t>(mm));
                qi -= mm;
                ti -= mm;
                break;
            }
            if (layer == 0) {
                const uint32_t aux = aux_at(ss, 0, k);
                const uint32_t mop = aux & 3;
                const int32_t raw = static_cast<int32_t>(aux >> 2);
                const int mc = max(qi - raw, 0);
                if (mc > 0) {
                    rw.push(0, static_cast<uint32_t>(mc));
                    qi -= mc;
                    ti -= mc;
                }
                if (mop == 0) {
                    rw.push(1, 1);
                    --qi;
                    --ti;
                    ++n_edit;
                    ss -= X;
                } else {
                    layer = static_cast<int>(mop);
                }
            } else if (layer == 1) {
                rw.push(3, 1);  // ins (query-extra) -> 'D'
                --qi;
                ++n_edit;
                if (aux_at(ss, 1, k) == 0) {
                    ss -= O + E;
                    layer = 0;
                } else {
                    ss -= E;
                }
                k -= 1;
            } else {
                rw.push(2, 1);  // del (target-extra) -> 'I'
                --ti;
                ++n_edit;
                if (aux_at(ss, 2, k) == 0) {
                    ss -= O + E;
                    layer = 0;
                } else {
                    ss -= E;
                }
                k += 1;
            }
        }
        if (guard < 0) atomicOr(P.error_flag, 4u);
        rw.flush();
    }
    const int leader = lane_id() & ~(G - 1);
    const uint32_t nr = __shfl_sync(PHR_FULL_MASK, rw.n, leader);
    const bool ovf = __shfl_sync(PHR_FULL_MASK, rw.overflow ? 1 : 0, leader) != 0;
    const uint32_t ned = __shfl_sync(PHR_FULL_MASK, n_edit, leader);
    __syncwarp();
    const uint32_t nr_fmt = (trace && !ovf) ? nr : 0;
    char* out = act ? P.text + P.text_off[pid] : nullptr;
    const uint32_t tl = format_group(runs, nr_fmt, out, G);
    if (act && gl == 0) {
        if (trace && !ovf) {
            PairOut o;
            o.status = PHR_OK;
            o.ed = static_cast<int32_t>(ned);  // levenshtein_from_cigar: X + I/D lengths
            o.t_consumed = t_end;
            o.affine_score = s_end;
            o.n_runs = nr;
            o.text_len = tl;
            P.out[pid] = o;
        } else if (failed) {
            PairOut o = {};
            o.status = PHR_ALIGNMENT_FAILED;
            P.out[pid] = o;
        } else if (trace && ovf) {
            atomicOr(P.error_flag, 2u);
        }
    }
}

template <class S>
__device__ void wfa_affine_group(const ExtendParams& P, const PairDesc& d, uint32_t pid, bool act, int G,
                                 uint8_t* region, uint64_t region_bytes, SDir* ring, uint32_t* sseq,
                                 int sseq_words) {
    const int gl = lane_id() & (G - 1);
    const int qn = act ? d.qn : 0, tn = act ? d.tn : 0;
    const bool fitting = act && tn > qn + qn / 2 + 10;
    const int X = P.costs.mismatch, O = P.costs.gap_open, E = P.costs.gap_extend;
    const uint32_t* qb = seq_base<S>(P, d.q_word);
    const uint32_t* tb = seq_base<S>(P, d.t_word);
    const int64_t hard_max_s = static_cast<int64_t>(qn + tn) * max(X, 1) + O + E + 4;
    // both sequences into the group's shared words when they fit (one extra word each:
    // windows read one word past the last symbol; the arena pads every sequence)
    {
        const int qw = act ? (qn + S::kPerWord - 1) / S::kPerWord + 1 : 0;
        const int tw = act ? (tn + S::kPerWord - 1) / S::kPerWord + 1 : 0;
        const bool stage = sseq != nullptr && qw + tw <= sseq_words;
        if (stage) {
            for (int i = gl; i < qw; i += G) sseq[i] = qb[i];
            for (int i = gl; i < tw; i += G) sseq[qw + i] = tb[i];
        }
        __syncwarp();
        if (stage) {
            qb = sseq;
            tb = sseq + qw;
        }
    }
    const bool use_ring = ring != nullptr && O + E < kAffRing && X < kAffRing;

    // region: [runs][values: cap int32][aux: cap uint32][... directory growing down]
    // The recurrence reads values only; keeping them apart from the traceback's aux words
    // doubles the cells each cached sector holds. Directory entry of score s is
    // dir_top[-1 - s], in the last quarter of the region.
    uint32_t* runs = reinterpret_cast<uint32_t*>(region);
    const uint64_t runs_bytes = align16(static_cast<uint64_t>(qn + tn + 2) * 4);
    const uint64_t rest = region_bytes > runs_bytes ? region_bytes - runs_bytes : 0;
    const uint64_t dir_cap = (rest / 4) / sizeof(AffDir);
    // cell indices stay 32-bit: a region never holds more than 2^32 - 1 cells here
    const uint64_t cell_bytes = rest - rest % sizeof(AffDir) - dir_cap * sizeof(AffDir);
    const uint64_t cell_cap = min(static_cast<uint64_t>((cell_bytes / 8) & ~3ull), static_cast<uint64_t>(0xFFFFFFFFu));
    int32_t* vals = reinterpret_cast<int32_t*>(region + runs_bytes);
    uint32_t* auxs = reinterpret_cast<uint32_t*>(vals + cell_cap);
    AffDir* dir_top = reinterpret_cast<AffDir*>(region + runs_bytes + rest - (rest % sizeof(AffDir)));
    auto dir_at = [&](int64_t sc) -> AffDir& { return dir_top[-1 - sc]; };
    auto fits = [&](uint64_t ncells, int64_t nscores) -> bool {
        return ncells <= cell_cap && static_cast<uint64_t>(nscores) <= dir_cap;
    };
    auto band_of = [&](int64_t sc, int layer) -> SBand {
        if (use_ring) return ring[sc & (kAffRing - 1)].L[layer];
        const LayerBand& b = dir_at(sc).L[layer];
        return SBand{b.lo, b.hi, static_cast<uint32_t>(b.base)};
    };

    bool alive = act;
    bool done = false, overflow = false;
    int s_end = 0, t_end = 0, k_end = 0, layer_end = 0;
    uint32_t used = 0;
    uint32_t wf_cells = 0, lcp_words = 0;   // work counters: M-band diagonals, LCP word compares

    if (alive && (dir_cap < 1 || cell_cap < 1 || !fits(1, 1))) {
        overflow = true;
        alive = false;
    }
    // ---- s = 0: m0[0] = extend(0, 0) ----
    if (alive && gl == 0) {
        AffDir e;
        e.L[0].lo = 0;
        e.L[0].hi = 0;
        e.L[0].base = 0;
        e.L[1].lo = 1;
        e.L[1].hi = 0;
        e.L[1].base = 1;
        e.L[2].lo = 1;
        e.L[2].hi = 0;
        e.L[2].base = 1;
        dir_at(0) = e;
        if (use_ring) ring[0] = SDir{{{0, 0, 0u}, {1, 0, 1u}, {1, 0, 1u}}};
        vals[0] = extend_valid<S>(qb, qn, tb, tn, 0, 0, lcp_words);
        auxs[0] = 0;
    }
    __syncwarp();
    if (alive) {
        used = 1;
        const int v0 = vals[0];
        // endpoint (wfa_simd.rs:618-650) on frame 0: only diagonal 0 is set
        if (!fitting) {
            if (qn - tn == 0 && v0 == qn) {
                done = true;
                t_end = tn;
                k_end = 0;
                layer_end = 0;
            }
        } else if (qn <= tn && v0 == qn) {
            done = true;
            t_end = qn;
            k_end = 0;
            layer_end = 0;
        }
    }
    const SBand none = {1, 0, 0u};
    // every reachable score is a sum of X, O + E and E: a multiple of g = gcd(X, O, E).
    // Other scores have empty wavefronts (and are never looked up nor traced back), so
    // the loop visits multiples of g only.
    int g = 0;
    for (int v : {X, O, E}) {
        int a = g, b = v < 0 ? -v : v;
        while (b) {
            const int t = a % b;
            a = b;
            b = t;
        }
        g = a;
    }
    const int step = g > 0 ? g : 1;
    int64_t s = step;
    for (;;) {
        const bool run = alive && !done && s <= hard_max_s;
        if (!__any_sync(PHR_FULL_MASK, run)) break;
        SBand bI = none, bD = none, bM = none;
        SBand sMo = none, sIe = none, sDe = none, sMx = none;
        bool go = run;
        if (go) {
            const int64_t so = s - O - E, se = s - E, sx = s - X;
            if (so >= 0) sMo = band_of(so, 0);
            if (se >= 0) {
                sIe = band_of(se, 1);
                sDe = band_of(se, 2);
            }
            if (sx >= 0) sMx = band_of(sx, 0);
            // I: from M[so] (k-1) and I[se] (k-1): bands shifted by +1
            int lo = INT32_MAX, hi = INT32_MIN;
            if (sMo.lo <= sMo.hi) { lo = min(lo, sMo.lo + 1); hi = max(hi, sMo.hi + 1); }
            if (sIe.lo <= sIe.hi) { lo = min(lo, sIe.lo + 1); hi = max(hi, sIe.hi + 1); }
            bI.lo = max(lo, -tn);
            bI.hi = min(hi, qn);
            // D: from M[so] (k+1) and D[se] (k+1): shifted by -1
            lo = INT32_MAX;
            hi = INT32_MIN;
            if (sMo.lo <= sMo.hi) { lo = min(lo, sMo.lo - 1); hi = max(hi, sMo.hi - 1); }
            if (sDe.lo <= sDe.hi) { lo = min(lo, sDe.lo - 1); hi = max(hi, sDe.hi - 1); }
            bD.lo = max(lo, -tn);
            bD.hi = min(hi, qn);
            // M: from M[sx] (k), I[s] (k), D[s] (k)
            lo = INT32_MAX;
            hi = INT32_MIN;
            if (sMx.lo <= sMx.hi) { lo = min(lo, sMx.lo); hi = max(hi, sMx.hi); }
            if (bI.lo <= bI.hi) { lo = min(lo, bI.lo); hi = max(hi, bI.hi); }
            if (bD.lo <= bD.hi) { lo = min(lo, bD.lo); hi = max(hi, bD.hi); }
            bM.lo = max(lo, -tn);
            bM.hi = min(hi, qn);
            if (gl == 0 && bM.lo <= bM.hi) wf_cells += static_cast<uint32_t>(bM.hi - bM.lo + 1);
            const uint32_t wI = bI.lo <= bI.hi ? static_cast<uint32_t>(bI.hi - bI.lo + 1) : 0;
            const uint32_t wD = bD.lo <= bD.hi ? static_cast<uint32_t>(bD.hi - bD.lo + 1) : 0;
            const uint32_t wM = bM.lo <= bM.hi ? static_cast<uint32_t>(bM.hi - bM.lo + 1) : 0;
            bI.base = used;
            bD.base = used + wI;
            bM.base = used + wI + wD;
            if (!fits(static_cast<uint64_t>(used) + wI + wD + wM, s + 1)) {
                overflow = true;
                alive = false;
                go = false;
            } else {
                used += wI + wD + wM;
            }
        }
        int best_end_k = INT32_MAX, best_end_layer = 0;
        if (go && bM.lo <= bM.hi) {
            // union band == M band (it contains the I and D bands); lane gl takes the
            // diagonals k with (k + tn) mod G == gl (G is a power of two)
            const int lo = bM.lo, hi = bM.hi;
            for (int k = lo + ((gl - lo - tn) & (G - 1)); k <= hi; k += G) {
                int32_t ins = UNSET, del = UNSET;
                if (k >= bI.lo && k <= bI.hi) {
                    int32_t best = UNSET, iop = 0;
                    if (k - 1 >= sMo.lo && k - 1 <= sMo.hi) {
                        const int32_t c = vals[sMo.base + (k - 1 - sMo.lo)] + 1;
                        if (pos_ok(c, k, qn, tn) && c > best) { best = c; iop = 0; }
                    }
                    if (k - 1 >= sIe.lo && k - 1 <= sIe.hi) {
                        const int32_t c = vals[sIe.base + (k - 1 - sIe.lo)] + 1;
                        if (pos_ok(c, k, qn, tn) && c > best) { best = c; iop = 1; }
                    }
                    ins = best;
                    vals[bI.base + (k - bI.lo)] = ins;
                    auxs[bI.base + (k - bI.lo)] = static_cast<uint32_t>(iop);
                }
                if (k >= bD.lo && k <= bD.hi) {
                    int32_t best = UNSET, dop = 0;
                    if (k + 1 >= sMo.lo && k + 1 <= sMo.hi) {
                        const int32_t c = vals[sMo.base + (k + 1 - sMo.lo)];
                        if (pos_ok(c, k, qn, tn) && c > best) { best = c; dop = 0; }
                    }
                    if (k + 1 >= sDe.lo && k + 1 <= sDe.hi) {
                        const int32_t c = vals[sDe.base + (k + 1 - sDe.lo)];
                        if (pos_ok(c, k, qn, tn) && c > best) { best = c; dop = 1; }
                    }
                    del = best;
                    vals[bD.base + (k - bD.lo)] = del;
                    auxs[bD.base + (k - bD.lo)] = static_cast<uint32_t>(dop);
                }
                // M (wfa_simd.rs:743-765): [mismatch-extend, ins close, del close], strict >
                int32_t best = UNSET;
                uint32_t mop = 0;
                if (k >= sMx.lo && k <= sMx.hi) {
                    const int32_t c = vals[sMx.base + (k - sMx.lo)] + 1;
                    if (pos_ok(c, k, qn, tn)) { best = c; mop = 0; }
                }
                if (pos_ok(ins, k, qn, tn) && ins > best) { best = ins; mop = 1; }
                if (pos_ok(del, k, qn, tn) && del > best) { best = del; mop = 2; }
                int32_t mval = UNSET;
                uint32_t aux = 0;
                if (best != UNSET) {
                    mval = extend_valid<S>(qb, qn, tb, tn, best, k, lcp_words);
                    aux = (static_cast<uint32_t>(best) << 2) | mop;
                }
                vals[bM.base + (k - bM.lo)] = mval;
                auxs[bM.base + (k - bM.lo)] = aux;
                // endpoint candidates: value == qn in layer order m, ins, del
                const int layer = mval == qn ? 0 : ins == qn ? 1 : del == qn ? 2 : -1;
                if (layer >= 0) {
                    if (!fitting) {
                        if (k == qn - tn) { best_end_k = k; best_end_layer = layer; }
                    } else if (k >= qn - tn && k < best_end_k) {
                        best_end_k = k;
                        best_end_layer = layer;
                    }
                }
            }
        }
        if (go && gl == 0) {
            AffDir e;
            e.L[0] = LayerBand{bM.lo, bM.hi, bM.base};
            e.L[1] = LayerBand{bI.lo, bI.hi, bI.base};
            e.L[2] = LayerBand{bD.lo, bD.hi, bD.base};
            dir_at(s) = e;
            if (use_ring) ring[s & (kAffRing - 1)] = SDir{{bM, bI, bD}};
        }
        // group min over (k, layer): smallest k wins (largest t_end)
        int kk = best_end_k, ll = best_end_layer;
        for (int o = 1; o < G; o <<= 1) {
            const int ok = __shfl_xor_sync(PHR_FULL_MASK, kk, o, G);
            const int ol = __shfl_xor_sync(PHR_FULL_MASK, ll, o, G);
            if (ok < kk) { kk = ok; ll = ol; }
        }
        __syncwarp();
        if (go && kk != INT32_MAX) {
            done = true;
            s_end = static_cast<int>(s);
            t_end = qn - kk;
            k_end = kk;
            layer_end = ll;
        }
        if (run) s += step;
    }
    {
        const unsigned cw = __reduce_add_sync(PHR_FULL_MASK, wf_cells), lw = __reduce_add_sync(PHR_FULL_MASK, lcp_words);
        if (lane_id() == 0 && P.work) {
            atomicAdd(P.work + 2, static_cast<unsigned long long>(cw));
            atomicAdd(P.work + 3, static_cast<unsigned long long>(lw));
        }
    }
    const bool failed = act && !done && !overflow;
    if (act && overflow && gl == 0) {
        // retry with 4x the room used so far (bounded by every diagonal of every score)
        const uint64_t full = runs_bytes + 4ull * static_cast<uint64_t>(hard_max_s + 1) * sizeof(AffDir) +
                              static_cast<uint64_t>(hard_max_s + 1) * 3ull * static_cast<uint64_t>(qn + tn + 1) * 8ull + 4096;
        // the directory gets a quarter of the region, the cells the rest
        const uint64_t grow = runs_bytes + 4ull * (static_cast<uint64_t>(used) * 8 + static_cast<uint64_t>(s + 1) * sizeof(AffDir)) +
                              4096;
        report_redo(P, pid, min(full, grow));
    }

    affine_finish(P, pid, act, G, qn, tn, X, O, E, runs, auxs, dir_top, done, failed, s_end, t_end, k_end,
                  layer_end);
}

// ===========================================================================
// Gap-affine WFA, one CTA per long pair
// ===========================================================================
// The warp-group kernel above runs a long, divergent pair with 32 lanes over bands of
// thousands of diagonals per score, and only a few hundred such pairs exist in a batch:
// most SMs idle. Here a CTA of kBigAffineThreads threads takes one pair; the recurrence, band
// rules, candidate order and tie-breaks are those of wfa_affine_group (values, ops and
// the end cell are identical), the diagonals of each score are dealt to the CTA's
// threads, both sequences sit in shared memory (bulk copies) while they fit, and one
// warp walks the traceback.
// Memory: the recurrence reads values at most max(X, O + E) scores back, so the M, I and
// D values live in a ring of that many score slots, indexed by diagonal; what every
// score keeps is one 32-bit history word per diagonal of its M band (the M source and
// the M value before extension, plus the I and D extend bits; the bands of I and D lie
// inside M's) and a directory entry with the three bands: 4 bytes per cell instead of
// 8 per cell and layer.
template <class S>
__device__ void wfa_affine_cta(const ExtendParams& P, const PairDesc& d, uint32_t pid, uint8_t* region,
                               uint64_t region_bytes, uint32_t* sm, uint64_t* bar, uint32_t& phase, int* sh_red) {
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int qn = d.qn, tn = d.tn;
    const bool fitting = tn > qn + qn / 2 + 10;
    const int X = P.costs.mismatch, O = P.costs.gap_open, E = P.costs.gap_extend;
    const int64_t hard_max_s = static_cast<int64_t>(qn + tn) * max(X, 1) + O + E + 4;
    uint32_t *qb, *tb;
    stage_pair_cta<S>(P, d, sm, bar, phase, &qb, &tb);

    int g = 0;
    for (int v : {X, O, E}) {
        int a = g, b = v < 0 ? -v : v;
        while (b) {
            const int t = a % b;
            a = b;
            b = t;
        }
        g = a;
    }
    const int step = g > 0 ? g : 1;
    // value ring: slot (score / step) % ring_n, layers M, I, D, indexed by k + tn
    const int ring_n = max(max(X, O + E), 1) / step + 1;
    const uint64_t ring_w = static_cast<uint64_t>(qn + tn + 1);

    // region: [runs][value ring][history words ...][... directory growing down]
    uint32_t* runs = reinterpret_cast<uint32_t*>(region);
    const uint64_t runs_bytes = align16(static_cast<uint64_t>(qn + tn + 2) * 4);
    const uint64_t ring_bytes = align16(static_cast<uint64_t>(ring_n) * 3 * ring_w * 4);
    const uint64_t fixed = runs_bytes + ring_bytes;
    const uint64_t rest = region_bytes > fixed ? region_bytes - fixed : 0;
    const uint64_t dir_cap = (rest / 8) / sizeof(AffDir);
    const uint64_t cell_bytes = rest - rest % sizeof(AffDir) - dir_cap * sizeof(AffDir);
    const uint64_t cell_cap = min(static_cast<uint64_t>((cell_bytes / 4) & ~3ull), static_cast<uint64_t>(0xFFFFFFFFu));
    int32_t* ring = reinterpret_cast<int32_t*>(region + runs_bytes);
    uint32_t* auxs = reinterpret_cast<uint32_t*>(region + fixed);
    AffDir* dir_top = reinterpret_cast<AffDir*>(region + fixed + rest - (rest % sizeof(AffDir)));
    auto dir_at = [&](int64_t sc) -> AffDir& { return dir_top[-1 - sc]; };
    auto val = [&](int64_t sc, int layer, int k) -> int32_t* {
        return ring + (static_cast<uint64_t>((sc / step) % ring_n) * 3 + layer) * ring_w + (k + tn);
    };
    auto fits = [&](uint64_t ncells, int64_t nscores) -> bool {
        return ncells <= cell_cap && static_cast<uint64_t>(nscores) <= dir_cap;
    };
    auto band_of = [&](int64_t sc, int layer) -> SBand {
        const LayerBand& b = dir_at(sc).L[layer];
        return SBand{b.lo, b.hi, static_cast<uint32_t>(b.base)};
    };

    bool done = false, overflow = false;
    int s_end = 0, t_end = 0, k_end = 0, layer_end = 0;
    uint32_t used = 0;
    uint32_t wf_cells = 0, lcp_words = 0;
    int32_t reach = 0;  // furthest query offset this thread's cells reached (redo sizing)
    if (region_bytes <= fixed || dir_cap < 1 || cell_cap < 1 || !fits(1, 1)) overflow = true;
    // ---- s = 0 ----
    if (!overflow && tid == 0) {
        AffDir e;
        e.L[0] = LayerBand{0, 0, 0};
        e.L[1] = LayerBand{1, 0, 0};
        e.L[2] = LayerBand{1, 0, 0};
        dir_at(0) = e;
        *val(0, 0, 0) = extend_valid<S>(qb, qn, tb, tn, 0, 0, lcp_words);
        auxs[0] = 0;
    }
    __syncthreads();
    if (!overflow) {
        used = 1;
        const int v0 = *val(0, 0, 0);
        reach = v0;
        if (!fitting) {
            if (qn - tn == 0 && v0 == qn) {
                done = true;
                t_end = tn;
            }
        } else if (qn <= tn && v0 == qn) {
            done = true;
            t_end = qn;
        }
    }
    const SBand none = {1, 0, 0u};
    int64_t s = step;
    // every thread computes the same bands and counters from the directory, so control
    // flow is uniform across the CTA
    while (!done && !overflow && s <= hard_max_s) {
        SBand bI = none, bD = none, bM = none;
        SBand sMo = none, sIe = none, sDe = none, sMx = none;
        const int64_t so = s - O - E, se = s - E, sx = s - X;
        if (so >= 0) sMo = band_of(so, 0);
        if (se >= 0) {
            sIe = band_of(se, 1);
            sDe = band_of(se, 2);
        }
        if (sx >= 0) sMx = band_of(sx, 0);
        int lo = INT32_MAX, hi = INT32_MIN;
        if (sMo.lo <= sMo.hi) { lo = min(lo, sMo.lo + 1); hi = max(hi, sMo.hi + 1); }
        if (sIe.lo <= sIe.hi) { lo = min(lo, sIe.lo + 1); hi = max(hi, sIe.hi + 1); }
        bI.lo = max(lo, -tn);
        bI.hi = min(hi, qn);
        lo = INT32_MAX;
        hi = INT32_MIN;
        if (sMo.lo <= sMo.hi) { lo = min(lo, sMo.lo - 1); hi = max(hi, sMo.hi - 1); }
        if (sDe.lo <= sDe.hi) { lo = min(lo, sDe.lo - 1); hi = max(hi, sDe.hi - 1); }
        bD.lo = max(lo, -tn);
        bD.hi = min(hi, qn);
        lo = INT32_MAX;
        hi = INT32_MIN;
        if (sMx.lo <= sMx.hi) { lo = min(lo, sMx.lo); hi = max(hi, sMx.hi); }
        if (bI.lo <= bI.hi) { lo = min(lo, bI.lo); hi = max(hi, bI.hi); }
        if (bD.lo <= bD.hi) { lo = min(lo, bD.lo); hi = max(hi, bD.hi); }
        bM.lo = max(lo, -tn);
        bM.hi = min(hi, qn);
        if (tid == 0 && bM.lo <= bM.hi) wf_cells += static_cast<uint32_t>(bM.hi - bM.lo + 1);
        const uint32_t wM = bM.lo <= bM.hi ? static_cast<uint32_t>(bM.hi - bM.lo + 1) : 0;
        bM.base = used;
        bI.base = bD.base = used;  // their history bits sit in M's words
        if (!fits(static_cast<uint64_t>(used) + wM, s + 1)) {
            overflow = true;
            break;
        }
        used += wM;
        int best_end_k = INT32_MAX, best_end_layer = 0;
        // (an empty band has lo = INT32_MAX, where lo + tid would wrap: its k loop starts
        // past hi)
        const int k0 = wM > 0 ? bM.lo + tid : 1, k1 = wM > 0 ? bM.hi : 0;
        // ring rows of this score's sources and of the score itself, indexed by diagonal
        // (the slot arithmetic once per score, not per cell; a negative score's row is
        // never read: its band is empty)
        auto row = [&](int64_t sc, int layer) -> int32_t* {
            return sc < 0 ? nullptr : val(sc, layer, 0);
        };
        const int32_t* rMo = row(so, 0);
        const int32_t* rIe = row(se, 1);
        const int32_t* rDe = row(se, 2);
        const int32_t* rMx = row(sx, 0);
        int32_t* cM = row(s, 0);
        int32_t* cI = row(s, 1);
        int32_t* cD = row(s, 2);
        for (int k = k0; k <= k1; k += nthr) {
            int32_t ins = UNSET, del = UNSET;
            uint32_t iop = 0, dop = 0;
            if (k >= bI.lo && k <= bI.hi) {
                int32_t best = UNSET;
                if (k - 1 >= sMo.lo && k - 1 <= sMo.hi) {
                    const int32_t c = rMo[k - 1] + 1;
                    if (pos_ok(c, k, qn, tn) && c > best) { best = c; iop = 0; }
                }
                if (k - 1 >= sIe.lo && k - 1 <= sIe.hi) {
                    const int32_t c = rIe[k - 1] + 1;
                    if (pos_ok(c, k, qn, tn) && c > best) { best = c; iop = 1; }
                }
                ins = best;
                cI[k] = ins;
            }
            if (k >= bD.lo && k <= bD.hi) {
                int32_t best = UNSET;
                if (k + 1 >= sMo.lo && k + 1 <= sMo.hi) {
                    const int32_t c = rMo[k + 1];
                    if (pos_ok(c, k, qn, tn) && c > best) { best = c; dop = 0; }
                }
                if (k + 1 >= sDe.lo && k + 1 <= sDe.hi) {
                    const int32_t c = rDe[k + 1];
                    if (pos_ok(c, k, qn, tn) && c > best) { best = c; dop = 1; }
                }
                del = best;
                cD[k] = del;
            }
            int32_t best = UNSET;
            uint32_t mop = 0;
            if (k >= sMx.lo && k <= sMx.hi) {
                const int32_t c = rMx[k] + 1;
                if (pos_ok(c, k, qn, tn)) { best = c; mop = 0; }
            }
            if (pos_ok(ins, k, qn, tn) && ins > best) { best = ins; mop = 1; }
            if (pos_ok(del, k, qn, tn) && del > best) { best = del; mop = 2; }
            int32_t mval = UNSET;
            uint32_t aux = (dop << 3) | (iop << 2);
            if (best != UNSET) {
                mval = extend_valid<S>(qb, qn, tb, tn, best, k, lcp_words);
                aux |= (static_cast<uint32_t>(best) << 4) | mop;
                reach = max(reach, mval);
            }
            cM[k] = mval;
            auxs[bM.base + (k - bM.lo)] = aux;
            const int layer = mval == qn ? 0 : ins == qn ? 1 : del == qn ? 2 : -1;
            if (layer >= 0) {
                if (!fitting) {
                    if (k == qn - tn) { best_end_k = k; best_end_layer = layer; }
                } else if (k >= qn - tn && k < best_end_k) {
                    best_end_k = k;
                    best_end_layer = layer;
                }
            }
        }
        if (tid == 0) {
            AffDir e;
            e.L[0] = LayerBand{bM.lo, bM.hi, bM.base};
            e.L[1] = LayerBand{bI.lo, bI.hi, bI.base};
            e.L[2] = LayerBand{bD.lo, bD.hi, bD.base};
            dir_at(s) = e;
        }
        // CTA min over (k, layer): smallest k wins (largest t_end); one key per thread
        const long long key = best_end_k == INT32_MAX
                                  ? LLONG_MAX
                                  : static_cast<long long>(best_end_k) * 4 + best_end_layer;  // layer < 4
        long long wkey = key;
        for (int o = 16; o > 0; o >>= 1) wkey = min(wkey, __shfl_xor_sync(PHR_FULL_MASK, wkey, o));
        long long* red = reinterpret_cast<long long*>(sh_red);
        if ((tid & 31) == 0) red[tid >> 5] = wkey;
        __syncthreads();  // this score's cells, directory entry and partial minima are visible
        long long best = LLONG_MAX;
        for (int w = 0; w < nthr / 32; ++w) best = min(best, red[w]);
        __syncthreads();  // `red` and the ring slot of s - ring_n * step are rewritten next
        if (best != LLONG_MAX) {
            done = true;
            s_end = static_cast<int>(s);
            k_end = static_cast<int>(best >> 2);   // floor(best / 4), also for negative k
            layer_end = static_cast<int>(best & 3);
            t_end = qn - k_end;
        }
        s += step;
    }
    if (P.work) {
        if (tid == 0) atomicAdd(P.work + 2, static_cast<unsigned long long>(wf_cells));
        if (lcp_words) atomicAdd(P.work + 3, static_cast<unsigned long long>(lcp_words));
    }
    const bool failed = !done && !overflow;
    if (overflow) {  // CTA-uniform
        // Scratch for the redo: extrapolate the final score from the furthest query offset
        // reached so far (the wavefront advances about in proportion to the score), plus a
        // quarter as margin, and the history from the cells so far (bands grow linearly,
        // so cells grow with the square of the score); at least four times what was used,
        // at most the whole search.
        long long* red = reinterpret_cast<long long*>(sh_red);
        int32_t wr = reach;
        for (int o = 16; o > 0; o >>= 1) wr = max(wr, __shfl_xor_sync(PHR_FULL_MASK, wr, o));
        if ((tid & 31) == 0) red[tid >> 5] = wr;
        __syncthreads();
        if (tid == 0) {
            int64_t rmax = 0;
            for (int w = 0; w < nthr / 32; ++w) rmax = ::max(rmax, static_cast<int64_t>(red[w]));
            const uint64_t full_cells = static_cast<uint64_t>(hard_max_s / step + 1) * ring_w;
            uint64_t s_est = static_cast<uint64_t>(hard_max_s) + 1, cells = full_cells;
            if (rmax > 0 && s > step) {
                uint64_t e = static_cast<uint64_t>(s) * static_cast<uint64_t>(qn) / static_cast<uint64_t>(rmax);
                e += e / 4 + 64;
                if (e < s_est) {
                    s_est = e;
                    const double r = static_cast<double>(e) / static_cast<double>(s);
                    cells = ::min(full_cells, static_cast<uint64_t>(static_cast<double>(used) * r * r) + 1024);
                }
            }
            cells = ::max(cells, static_cast<uint64_t>(4ull * used + 1024));
            const uint64_t need_rest =
                ::max(static_cast<uint64_t>(cells * 4 * 8 / 7 + 4096), static_cast<uint64_t>(8 * (s_est + 1) * sizeof(AffDir))) + 64;
            report_redo(P, pid, fixed + need_rest + 4096);
        }
    }
    __syncthreads();
    if (tid < 32)
        affine_finish(P, pid, true, 32, qn, tn, X, O, E, runs, auxs, dir_top, done, failed, s_end, t_end, k_end,
                      layer_end, 0, 0, 0, nullptr, 0, true);
    __syncthreads();
}

template <class S>
__global__ void __launch_bounds__(kBigAffineThreads, 1) wfa_affine_big_kernel(ExtendParams P) {
    extern __shared__ __align__(16) uint32_t big_sm[];
    __shared__ uint32_t sh_task;
    __shared__ __align__(8) long long sh_red[kBigAffineThreads / 32];
    __shared__ __align__(8) uint64_t sh_bar;
    uint32_t phase = 0;  // parity of sh_bar's current phase, the same in every thread
    if (threadIdx.x == 0) mbar_init(&sh_bar, 1);
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) sh_task = P.tasks.range[0] + atomicAdd(P.queue_head, 1u);
        __syncthreads();
        const uint32_t task = sh_task;
        __syncthreads();
        if (task >= P.tasks.range[1]) break;
        if (!(P.tasks.task_group[task] & kBigTask)) continue;
        const uint32_t pid = P.tasks.order[P.tasks.task_first[task]];
        const PairDesc d = P.desc[pid];
        if (d.mode != (S::kBits == 2 ? 0 : 1)) continue;
        wfa_affine_cta<S>(P, d, pid, P.scratch + P.task_off[task], P.task_len[task] & ~15ull, big_sm, &sh_bar, phase,
                          reinterpret_cast<int*>(sh_red));
    }
}

// ===========================================================================
// Gap-affine WFA, one pair per warp, wavefronts in registers
// ===========================================================================
// Every reachable cell of score s lies on a diagonal |k| <= (s - O) / E (a gap of length
// L costs O + L E), so a window of kRegWin diagonals (slots of 32, lane = offset in the
// slot) holds whole wavefronts while that bound stays inside it. Each lane keeps the M,
// I and D values of its diagonals for the last scores the recurrence looks back to
// (X, O + E and E, in steps of g = gcd(X, O, E)) in shift registers; neighbour diagonals
// k - 1 and k + 1 come from the adjacent lane by shuffle. Cells are computed exactly as
// in wfa_affine_group (candidate order, strict >, validity), so values, ops and the end
// cell are identical; only the traceback's aux words go to memory, in the same history
// layout (one row of kRegWin words per layer and score), so the same traceback runs.
// A pair whose reachable band would leave the window stops and is redone by
// wfa_affine_group.
// Slots of 32 diagonals, centred on diagonal 0 so that the band of the early scores (and
// of most pairs' whole search) is one slot: 0 = [-16, 15], 1 = [-48, -17], 2 = [16, 47],
// 3 = [-80, -49], 4 = [48, 79].
constexpr int kRegSlots = 5;
constexpr int kRegMaxLen = 1024;  // qlen + tlen below which a pair tries the register kernel
constexpr int kRegWin = 32 * kRegSlots;
constexpr int kRegLo = -kRegWin / 2;
__host__ __device__ constexpr int reg_slot_lo(int h) { return h == 0 ? -16 : h == 1 ? -48 : h == 2 ? 16 : h == 3 ? -80 : 48; }
__host__ __device__ constexpr int reg_left(int h) { return h == 0 ? 1 : h == 1 ? 3 : h == 2 ? 0 : h == 4 ? 2 : -1; }
__host__ __device__ constexpr int reg_right(int h) { return h == 0 ? 2 : h == 1 ? 0 : h == 2 ? 4 : h == 3 ? 1 : -1; }

// value at diagonal k - 1 (UP) or k + 1 of slot h, across lanes and into the adjacent slot;
// SOLO: the band has never left slot h, so the adjacent slot holds UNSET everywhere
template <bool UP, bool SOLO>
__device__ __forceinline__ int32_t reg_neighbor(const int32_t (&v)[kRegSlots], int h) {
    const int lane = lane_id();
    if (UP) {
        const int32_t a = __shfl_up_sync(PHR_FULL_MASK, v[h], 1);
        const int32_t b =
            SOLO ? UNSET : __shfl_sync(PHR_FULL_MASK, reg_left(h) >= 0 ? v[reg_left(h)] : UNSET, 31);
        return lane == 0 ? b : a;
    }
    const int32_t a = __shfl_down_sync(PHR_FULL_MASK, v[h], 1);
    const int32_t b = SOLO ? UNSET : __shfl_sync(PHR_FULL_MASK, reg_right(h) >= 0 ? v[reg_right(h)] : UNSET, 0);
    return lane == 31 ? b : a;
}

// History rows of slot 0 (diagonals -16..15) kept in the warp's shared memory: rows of
// scores 0 .. (kRegShRows - 1) g, which hold the whole history of most short pairs, so
// their traceback reads shared memory.
constexpr int kRegShRows = 32;
// Words of a short pair's two staged sequences (qlen + tlen < kRegMaxLen, each followed by
// one padding word for the 32-bit windows that read one word ahead).
constexpr int kRegSeqWords = 1024 / 16 + 4;
// Shared memory of one warp on the register path: the history rows, then the staged
// sequences of its pair.
constexpr int kRegWarpSmem = kRegShRows * 128 + kRegSeqWords * 4;

// Copies a short 2-bit pair's words into `dst` (q first, then t) with the W lanes of
// its segment; the caller synchronises the warp before reading them. Match extension
// then reads shared memory instead of L1/L2.
template <int W>
__device__ __forceinline__ void stage_pair_words(uint32_t* dst, const uint32_t* q, int qn, const uint32_t* t, int tn,
                                                 int ls, const uint32_t** sq, const uint32_t** st) {
    const int qw = (qn + 15) / 16 + 1, tw = (tn + 15) / 16 + 1;
    for (int i = ls; i < qw; i += W) dst[i] = __ldg(q + i);
    for (int i = ls; i < tw; i += W) dst[qw + i] = __ldg(t + i);
    *sq = dst;
    *st = dst + qw;
}

// Returns true when the pair's band left the window: nothing is written for it and the
// caller runs it through wfa_affine_group.
template <class S, int XS, int OES, int ES>
__device__ bool wfa_affine_reg(const ExtendParams& P, const PairDesc& d, uint32_t pid, uint8_t* region,
                               uint64_t region_bytes, uint32_t* sh_hist) {
    constexpr int RM = (XS > OES ? XS : OES);  // M values kept: steps 1..RM back
    const int lane = lane_id();
    const int qn = d.qn, tn = d.tn;
    const bool fitting = tn > qn + qn / 2 + 10;
    const int X = P.costs.mismatch, O = P.costs.gap_open, E = P.costs.gap_extend;
    const int g = X / XS;  // the step of reachable scores
    const uint32_t *qb, *tb;
    stage_pair_words<32>(sh_hist + kRegShRows * 32, seq_base<S>(P, d.q_word), qn, seq_base<S>(P, d.t_word), tn, lane,
                         &qb, &tb);
    __syncwarp();
    const int64_t hard_max_s = static_cast<int64_t>(qn + tn) * max(X, 1) + O + E + 4;

    // region: [runs][aux rows: kRegWin words per visited score, each word the M, I and D
    // history of one diagonal]; row r holds score r * g, so the traceback needs no
    // directory
    uint32_t* runs = reinterpret_cast<uint32_t*>(region);
    const uint64_t runs_bytes = align16(static_cast<uint64_t>(qn + tn + 2) * 4);
    const uint64_t rest = region_bytes > runs_bytes ? region_bytes - runs_bytes : 0;
    const uint64_t row_cap = rest / (kRegWin * 4);
    uint32_t* auxs = reinterpret_cast<uint32_t*>(region + runs_bytes);
    const int wlo = max(kRegLo, -tn), whi = min(kRegLo + kRegWin - 1, qn);  // window clipped to [-tn, qn]

    int32_t M[RM][kRegSlots], I[ES][kRegSlots], D[ES][kRegSlots];
#pragma unroll
    for (int h = 0; h < kRegSlots; ++h) {
#pragma unroll
        for (int r = 0; r < RM; ++r) M[r][h] = UNSET;
#pragma unroll
        for (int r = 0; r < ES; ++r) {
            I[r][h] = UNSET;
            D[r][h] = UNSET;
        }
    }
    uint32_t wf_cells = 0, lcp_words = 0;
    bool done = false, overflow = row_cap < 2;
    int s_end = 0, t_end = 0, k_end = 0, layer_end = 0;
    // ---- s = 0: M[0][0] = extend(0, 0), at slot -kRegLo / 32, lane 0 ----
    int32_t v0 = 0;
    if (!overflow) {
        if (lane == 0) v0 = extend_valid<S>(qb, qn, tb, tn, 0, 0, lcp_words);
        v0 = __shfl_sync(PHR_FULL_MASK, v0, 0);
        if (lane == 0) sh_hist[16] = 0;  // row 0 = score 0, diagonal 0 (slot 0, lane 16)
        if (lane == 16) M[0][0] = v0;  // diagonal 0: slot 0, lane 16
        if (!fitting) {
            if (qn - tn == 0 && v0 == qn) done = true, t_end = tn;
        } else if (qn <= tn && v0 == qn) {
            done = true;
            t_end = qn;
        }
    }
    uint64_t row = 1;
    int64_t s = g;
    // half-width of the reachable band, floor((s - O) / E) from score O + E on, kept
    // incrementally; `active` marks the slots the band has reached (they stay reached)
    int hw = 0;
    int64_t next_hw = static_cast<int64_t>(O) + E;
    uint32_t active = 1u;
    for (; !done && !overflow && s <= hard_max_s; s += g) {
        // reachable diagonals of this score; leaving the window ends this kernel's attempt
        while (s >= next_hw) {
            ++hw;
            next_hw += E;
        }
        const int blo = max(-tn, -hw);
        const int bhi = min(qn, hw);
        if (blo < wlo || bhi > whi || row >= row_cap) {
            overflow = true;
            break;
        }
        if (lane == 0) wf_cells += static_cast<uint32_t>(bhi - blo + 1);
        uint32_t* arow = auxs + row * kRegWin;
        uint32_t* srow = row < kRegShRows ? sh_hist + row * 32 : nullptr;
        int32_t nM[kRegSlots], nI[kRegSlots], nD[kRegSlots];
        int best_k = INT32_MAX, best_l = 0;
        // one slot of this score; h and SOLO are compile-time
        auto step_slot = [&](auto hc, auto soloc) {
            constexpr int h = decltype(hc)::value;
            constexpr bool solo = decltype(soloc)::value;
            nM[h] = nI[h] = nD[h] = UNSET;
            constexpr int klo = reg_slot_lo(h);
            if (klo + 31 < blo || klo > bhi) return;  // warp-uniform: slot outside the band
            active |= 1u << h;
            const int k = klo + lane;
            // affine_pos_valid for this diagonal as one unsigned range test: pos in
            // [max(0, k), min(qn, tn + k)] (an empty range admits nothing; UNSET and
            // UNSET + 1 wrap far above any span)
            const int vl = max(0, k), vh = min(qn, tn + k);
            const uint32_t vlo = vh >= vl ? static_cast<uint32_t>(vl) : 0x40000000u;
            const uint32_t vspan = vh >= vl ? static_cast<uint32_t>(vh - vl) : 0u;
            auto ok = [&](int32_t pos) { return static_cast<uint32_t>(pos) - vlo <= vspan; };
            const int32_t mo_dn = reg_neighbor<true, solo>(M[OES - 1], h);   // M[s - O - E][k - 1]
            const int32_t ie_dn = reg_neighbor<true, solo>(I[ES - 1], h);    // I[s - E][k - 1]
            const int32_t mo_up = reg_neighbor<false, solo>(M[OES - 1], h);  // M[s - O - E][k + 1]
            const int32_t de_up = reg_neighbor<false, solo>(D[ES - 1], h);   // D[s - E][k + 1]
            // I (wfa_simd.rs:682-738): [open from M, extend I], strict >
            int32_t ins = UNSET;
            uint32_t iop = 0;
            if (ok(mo_dn + 1)) ins = mo_dn + 1;
            if (ok(ie_dn + 1) && ie_dn + 1 > ins) {
                ins = ie_dn + 1;
                iop = 1;
            }
            int32_t del = UNSET;
            uint32_t dop = 0;
            if (ok(mo_up)) del = mo_up;
            if (ok(de_up) && de_up > del) {
                del = de_up;
                dop = 1;
            }
            // M (wfa_simd.rs:743-765): [mismatch-extend, ins close, del close], strict >
            // (ins and del are UNSET or valid already)
            int32_t best = UNSET;
            uint32_t mop = 0;
            if (ok(M[XS - 1][h] + 1)) best = M[XS - 1][h] + 1;
            if (ins != UNSET && ins > best) {
                best = ins;
                mop = 1;
            }
            if (del != UNSET && del > best) {
                best = del;
                mop = 2;
            }
            int32_t mval = UNSET;
            uint32_t aux = (dop << 3) | (iop << 2);
            if (best != UNSET) {
                mval = extend_valid<S>(qb, qn, tb, tn, best, k, lcp_words);
                aux |= (static_cast<uint32_t>(best) << 4) | mop;
            }
            nM[h] = mval;
            nI[h] = ins;
            nD[h] = del;
            if (h == 0 && srow)
                srow[lane] = aux;
            else
                arow[k - kRegLo] = aux;
            // end cell: value == qn in layer order m, ins, del; smallest k (largest t_end)
            const int layer = mval == qn ? 0 : ins == qn ? 1 : del == qn ? 2 : -1;
            const bool cand = layer >= 0 && (fitting ? k >= qn - tn : k == qn - tn);
            const unsigned bal = __ballot_sync(PHR_FULL_MASK, cand);
            if (bal) {
                const int src = __ffs(bal) - 1;
                const int l = __shfl_sync(PHR_FULL_MASK, layer, src);
                if (klo + src < best_k) {
                    best_k = klo + src;
                    best_l = l;
                }
            }
        };
        // shift the history of slot h: this score becomes one step back
        auto shift_slot = [&](int h) {
#pragma unroll
            for (int r = RM - 1; r > 0; --r) M[r][h] = M[r - 1][h];
            M[0][h] = nM[h];
#pragma unroll
            for (int r = ES - 1; r > 0; --r) {
                I[r][h] = I[r - 1][h];
                D[r][h] = D[r - 1][h];
            }
            I[0][h] = nI[h];
            D[0][h] = nD[h];
        };
        if (blo >= -16 && bhi <= 15) {
            // the band has never left slot 0 (it only grows): one slot, no cross-slot shuffles
            step_slot(std::integral_constant<int, 0>{}, std::true_type{});
            shift_slot(0);
        } else {
            step_slot(std::integral_constant<int, 0>{}, std::false_type{});
            step_slot(std::integral_constant<int, 1>{}, std::false_type{});
            step_slot(std::integral_constant<int, 2>{}, std::false_type{});
            step_slot(std::integral_constant<int, 3>{}, std::false_type{});
            step_slot(std::integral_constant<int, 4>{}, std::false_type{});
            static_assert(kRegSlots == 5, "one step_slot call per slot");
#pragma unroll
            for (int h = 0; h < kRegSlots; ++h)
                if ((active >> h) & 1u) shift_slot(h);
        }
        ++row;  // the traceback addresses row s / g directly (no directory)
        if (best_k != INT32_MAX) {
            done = true;
            s_end = static_cast<int>(s);
            t_end = qn - best_k;
            k_end = best_k;
            layer_end = best_l;
        }
    }
    {
        const unsigned lw = __reduce_add_sync(PHR_FULL_MASK, lcp_words);
        if (lane == 0 && P.work) {
            atomicAdd(P.work + 2, static_cast<unsigned long long>(wf_cells));
            atomicAdd(P.work + 3, static_cast<unsigned long long>(lw));
        }
    }
    __syncwarp();
    if (overflow) return true;  // wfa_affine_group takes it, which sizes its bands per score
    affine_finish(P, pid, true, 32, qn, tn, X, O, E, runs, auxs, nullptr, done, !done, s_end, t_end, k_end,
                  layer_end, g, kRegWin, kRegLo, sh_hist, kRegShRows);
    return false;
}

// Persistent kernel: warps pull tasks; each task's groups split the warp's slot evenly.
constexpr int kAffGroupSmem = kAffRingGroups * kAffRing * static_cast<int>(sizeof(SDir)) + kWarpSeqWords * 4;
constexpr int kAffWarpSmem = kAffGroupSmem > kRegWarpSmem ? kAffGroupSmem : kRegWarpSmem;

template <class S, bool kAffine>
__global__ void __launch_bounds__(256, kAffine ? 2 : 4) wfa_kernel(ExtendParams P) {
    extern __shared__ __align__(16) uint8_t wfa_smem[];
    const int lane = lane_id();
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = P.tasks.range[0] + atomicAdd(P.queue_head, 1u);
        task = __shfl_sync(PHR_FULL_MASK, task, 0);
        if (task >= P.tasks.range[1]) break;
        uint8_t* slot = P.task_off ? P.scratch + P.task_off[task] : P.scratch + warp_global * P.slot_bytes;
        const uint64_t slot_bytes = P.task_off ? P.task_len[task] : P.slot_bytes;
        const uint8_t tg = P.tasks.task_group[task];
        if (tg & kBigTask) continue;  // a redo task of a CTA-per-pair kernel
        const int G = tg;
        const int count = P.tasks.task_count[task];
        const int grp = lane / G;
        bool act = grp < count;
        const uint32_t pid = act ? P.tasks.order[P.tasks.task_first[task] + grp] : 0;
        PairDesc d = {};
        if (act) d = P.desc[pid];
        // pairs of the other symbol mode run in the other instantiation
        act = act && d.mode == (S::kBits == 2 ? 0 : 1);
        // long pairs run one per CTA: deferred from the main pass to the redo passes,
        // where wfa_linear_big_kernel / wfa_affine_big_kernel take them
        if (act && !P.task_off && big_pair(P.engine, P.big_min, P.big_smem, d.qn, d.tn, d.mode)) {
            if ((lane & (G - 1)) == 0)
                report_redo(P, pid, wfa_region_est(d.qn, d.tn, kAffine));
            act = false;
        }
        if (!__any_sync(PHR_FULL_MASK, act)) continue;
        // redo tasks hold one pair, which gets the whole task region
        const uint64_t region_bytes = (P.task_off ? slot_bytes : slot_bytes / (32 / G)) & ~15ull;
        uint8_t* region = slot + static_cast<uint64_t>(grp) * region_bytes;
        // a task whose estimated need exceeds the slot goes straight to a redo pass
        if (!P.task_off && P.task_need && P.task_need[task] > slot_bytes) {
            if (act && (lane & (G - 1)) == 0) report_redo(P, pid, P.task_need[task] / (32 / G));
            continue;
        }
        if constexpr (kAffine && S::kBits == 2) {
            // short 2-bit pairs of one warp each, costs with a register specialisation:
            // wavefronts in registers (redo passes and wide bands take the group kernel)
            if (G == 32 && !P.task_off && act && d.qn + d.tn < kRegMaxLen) {
                const int X = P.costs.mismatch, O = P.costs.gap_open, E = P.costs.gap_extend;
                uint32_t* sh_hist = reinterpret_cast<uint32_t*>(wfa_smem + static_cast<size_t>(threadIdx.x >> 5) *
                                                                                  kAffWarpSmem);
                bool wide = true;  // the band left the register window (or no specialisation)
                if (X == 4 && O == 6 && E == 2) wide = wfa_affine_reg<S, 2, 4, 1>(P, d, pid, region, region_bytes, sh_hist);
                else if (X == 2 && O == 4 && E == 1)
                    wide = wfa_affine_reg<S, 2, 5, 1>(P, d, pid, region, region_bytes, sh_hist);
                if (!wide) continue;
                // otherwise the group kernel below takes the pair in place (no redo pass)
            }
        }
        if (kAffine) {
            // per warp: one directory ring per group of >= 4 lanes, then the sequence words
            uint8_t* wsm = wfa_smem + static_cast<size_t>(threadIdx.x >> 5) * kAffWarpSmem;
            SDir* ring = 32 / G <= kAffRingGroups ? reinterpret_cast<SDir*>(wsm) + grp * kAffRing : nullptr;
            const int seq_words = kWarpSeqWords / (32 / G);
            uint32_t* sseq = seq_words > 0 ? reinterpret_cast<uint32_t*>(wsm + kAffRingGroups * kAffRing * sizeof(SDir)) +
                                                 grp * seq_words
                                           : nullptr;
            wfa_affine_group<S>(P, d, pid, act, G, region, region_bytes, ring, sseq, seq_words);
        }
        else
            wfa_linear_group<S>(P, d, pid, act, G, region, region_bytes);
    }
}

}  // namespace

void launch_wfa_linear(const ExtendParams& p, int grid, int block, cudaStream_t st) {
    wfa_kernel<Seq2, false><<<grid, block, 0, st>>>(p);
}
void launch_wfa_linear_bytes(const ExtendParams& p, int grid, int block, cudaStream_t st) {
    wfa_kernel<SeqB, false><<<grid, block, 0, st>>>(p);
}
void launch_wfa_linear_big(const ExtendParams& p, int grid, int mode, cudaStream_t st) {
    if (mode == 0) {
        cudaFuncSetAttribute(wfa_linear_big_kernel<Seq2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(p.big_smem));
        wfa_linear_big_kernel<Seq2><<<grid, kBigThreads, p.big_smem, st>>>(p);
    } else {
        cudaFuncSetAttribute(wfa_linear_big_kernel<SeqB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(p.big_smem));
        wfa_linear_big_kernel<SeqB><<<grid, kBigThreads, p.big_smem, st>>>(p);
    }
}
void launch_wfa_affine_big(const ExtendParams& p, int grid, int threads, int mode, cudaStream_t st) {
    if (mode == 0) {
        cudaFuncSetAttribute(wfa_affine_big_kernel<Seq2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(p.big_smem));
        wfa_affine_big_kernel<Seq2><<<grid, threads, p.big_smem, st>>>(p);
    } else {
        cudaFuncSetAttribute(wfa_affine_big_kernel<SeqB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(p.big_smem));
        wfa_affine_big_kernel<SeqB><<<grid, threads, p.big_smem, st>>>(p);
    }
}

void launch_wfa_affine(const ExtendParams& p, int grid, int block, cudaStream_t st) {
    const int smem = (block / 32) * kAffWarpSmem;
    cudaFuncSetAttribute(wfa_kernel<Seq2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    wfa_kernel<Seq2, true><<<grid, block, smem, st>>>(p);
}
void launch_wfa_affine_bytes(const ExtendParams& p, int grid, int block, cudaStream_t st) {
    const int smem = (block / 32) * kAffWarpSmem;
    cudaFuncSetAttribute(wfa_kernel<SeqB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    wfa_kernel<SeqB, true><<<grid, block, smem, st>>>(p);
}

}  // namespace phr
