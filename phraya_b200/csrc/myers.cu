// myers.cu -- Myers bit-parallel edit distance with CIGAR traceback (sm_100a).
//
// Semantics restated from phraya-align/src/wfa_simd.rs:
//   forward pass      myers_forward_flat_with_cutoff   :3552-3648
//   global entry      myers_edit_distance_impl         :3657-3673
//   fitting entry     myers_fitting_impl               :3783-3814
//   traceback         myers_backtrace_flat             :3702-3781 (precedence D, I, diagonal)
//
// GPU design. A pair is owned by a group of G lanes (G = next power of two >= the
// number of 64-bit query blocks, capped at 32); lane l owns query block l (rows
// 64l+1 .. 64l+64). The group runs an anti-diagonal pipeline: at step s lane l updates
// its block for target column s-l, receiving the add/hp/hn carries and the target
// symbol from lane l-1 through one __shfl_up_sync. Queries longer than 32 blocks are
// processed in stripes of G blocks whose boundary carries go through scratch memory.
//
// The reference reconstructs whole DP columns from VP/VN during traceback. Its
// decisions only need two delta bits per cell: `cur == above + 1` is VP(i-1) of
// column j and `cur == left + 1` is HP(i-1) (the horizontal delta the forward pass
// already computes); a diagonal move is M or X by comparing the two bytes, exactly as
// the reference does. So the forward pass stores {VP, HP} per (column, block) and the
// traceback walks bits, never values. Only the blocks within
// a band |i - j| <= E + 2 are stored: every cell of an alignment of cost ed satisfies
// |i - j| <= ed, so the walk stays in the band whenever ed <= E; pairs with ed > E are
// redone with every block stored (full_band).
#include <mutex>

#include "kernels.cuh"

namespace phr {
namespace {

constexpr int kRecBytes = 16;  // VP and HP of one 64-bit block of one column

__device__ __forceinline__ uint32_t compress_even(uint32_t x) {
    x &= 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
    x = (x | (x >> 4)) & 0x00FF00FFu;
    x = (x | (x >> 8)) & 0x0000FFFFu;
    return x;
}

__device__ __forceinline__ uint64_t align16(uint64_t v) { return (v + 15) & ~15ull; }

struct Band {
    int E;      // band half-width used for the redo decision
    int W;      // stored blocks per column
    int nb;
    __device__ __forceinline__ int blo(int J) const {  // first stored block of DP column J (1-based)
        int r = J - (E + 2) - 1;
        int lo = r > 0 ? (r >> 6) : 0;
        return min(lo, nb - W);
    }
};

__device__ __forceinline__ Band make_band(int m, int n, int nb, int full, int base) {
    Band b;
    b.nb = nb;
    if (full) {
        b.E = max(m, n);
        b.W = nb;
    } else {
        int E = base + abs(m - n) + (m >> 4);
        E = min(E, max(m, n));
        b.E = E;
        int W = (2 * (E + 2) + 1 + 63) / 64 + 1;
        b.W = min(W, nb);
    }
    return b;
}

// Scratch bytes one pair needs: band records + stripe carries + reverse runs.
__device__ __forceinline__ uint64_t pair_need(int m, int n, int nb, int G, const Band& b) {
    uint64_t need = align16(static_cast<uint64_t>(n) * b.W * kRecBytes);
    if (nb > G) need += align16(static_cast<uint64_t>(n));
    need += align16(static_cast<uint64_t>(m + n + 2) * 4);
    return need;
}

template <class S>
struct QueryBlock;

template <>
struct QueryBlock<Seq2> {
    uint64_t p0, p1, p2, p3;
    __device__ __forceinline__ void load(const uint32_t* q, int qsh, int blk, uint64_t mask) {
        p0 = p1 = p2 = p3 = 0;
#pragma unroll
        for (int wi = 0; wi < 4; ++wi) {
            const uint32_t w = __ldg(q + blk * 4 + wi);
            const int sh = wi * 16;
            p0 |= static_cast<uint64_t>(compress_even(~(w | (w >> 1)))) << sh;
            const uint32_t x1 = w ^ 0x55555555u;
            p1 |= static_cast<uint64_t>(compress_even(~(x1 | (x1 >> 1)))) << sh;
            const uint32_t x2 = w ^ 0xAAAAAAAAu;
            p2 |= static_cast<uint64_t>(compress_even(~(x2 | (x2 >> 1)))) << sh;
            const uint32_t x3 = ~w;
            p3 |= static_cast<uint64_t>(compress_even(~(x3 | (x3 >> 1)))) << sh;
        }
        p0 &= mask;
        p1 &= mask;
        p2 &= mask;
        p3 &= mask;
    }
    __device__ __forceinline__ uint64_t eq(uint32_t c) const {
        const uint64_t a = (c & 1) ? p1 : p0;
        const uint64_t b = (c & 1) ? p3 : p2;
        return (c & 2) ? b : a;
    }
};

template <class S>
struct QueryBlockBytes {
    uint32_t w[16];
    uint64_t mask;
    __device__ __forceinline__ void load(const uint32_t* q, int qsh, int blk, uint64_t msk) {
#pragma unroll
        for (int k = 0; k < 16; ++k) w[k] = load_window<S>(q, qsh + blk * 64 + 4 * k);
        mask = msk;
    }
    __device__ __forceinline__ uint64_t eq(uint32_t c) const {
        const uint32_t c4 = c * 0x01010101u;
        uint64_t e = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const uint32_t v = __vcmpeq4(w[k], c4) & 0x01010101u;
            e |= static_cast<uint64_t>(((v * 0x204081u) >> 21) & 0xFu) << (4 * k);
        }
        return e & mask;
    }
};

template <>
struct QueryBlock<SeqB> : QueryBlockBytes<SeqB> {};
template <>
struct QueryBlock<SeqBc> : QueryBlockBytes<SeqBc> {};

template <class S>
__device__ __forceinline__ const uint32_t* seq_base(const ExtendParams& P, uint64_t word) {
    return (S::kBits == 2 ? P.packed2 : P.bytes) + word;
}

// 64-bit a + b + carry_in with carry out (one add chain).
__device__ __forceinline__ uint64_t add_carry64(uint64_t a, uint64_t b, uint32_t cin, uint32_t* cout) {
    uint32_t lo, hi, c;
    const uint32_t alo = static_cast<uint32_t>(a), ahi = static_cast<uint32_t>(a >> 32);
    const uint32_t blo = static_cast<uint32_t>(b), bhi = static_cast<uint32_t>(b >> 32);
    asm("{\n\t"
        ".reg .u32 t;\n\t"
        "add.cc.u32 t, %5, 0xFFFFFFFF;\n\t"  // carry flag := (cin != 0)
        "addc.cc.u32 %0, %3, %4;\n\t"
        "addc.cc.u32 %1, %6, %7;\n\t"
        "addc.u32 %2, 0, 0;\n\t"
        "}"
        : "=r"(lo), "=r"(hi), "=r"(c)
        : "r"(alo), "r"(blo), "r"(cin), "r"(ahi), "r"(bhi));
    *cout = c;
    return (static_cast<uint64_t>(hi) << 32) | lo;
}

// Bit r (window row offset 0..127) of the 128-bit word hi:lo.
__device__ __forceinline__ uint32_t bit128(uint64_t lo, uint64_t hi, int r) {
    const uint64_t w = r >= 64 ? hi : lo;
    return static_cast<uint32_t>((w >> (r & 63)) & 1ull);
}

// Runs one Myers alignment per active group of the warp. All 32 lanes call this with
// warp-uniform control flow; `act` marks lanes whose group holds a pair.
template <class S>
__device__ void myers_group(const ExtendParams& P, const PairDesc& d, uint32_t pid, bool act, int G,
                            uint8_t* slot, uint64_t slot_off, bool fits) {
    const int lane = lane_id();
    const int gl = lane & (G - 1);
    const int m = act ? d.qn : 0;
    const int n = act ? d.tn : 0;
    const int nb = (m + 63) >> 6;
    const bool fitting = act && P.engine == PHR_ENGINE_MYERS_FIT && n > m + m / 2 + 10;
    const Band band = make_band(m, n, nb, P.full_band, P.band_base);
    const uint32_t* qb = seq_base<S>(P, d.q_word);
    const uint32_t* tb = seq_base<S>(P, d.t_word);

    uint8_t* recs = slot + slot_off;
    uint64_t off = align16(static_cast<uint64_t>(n) * band.W * kRecBytes);
    uint8_t* stripe_buf = recs + off;
    if (nb > G) off += align16(static_cast<uint64_t>(n));
    uint32_t* runs = reinterpret_cast<uint32_t*>(recs + off);

    const bool go = act && fits;
    const int R = go ? (nb + G - 1) / G : 0;
    const int Rmax = __reduce_max_sync(PHR_FULL_MASK, static_cast<unsigned>(R));
    const int last_lane = (nb - 1) % G;
    const int score_bit = (m - 1) & 63;
    const int margin = m / 10 + 1;
    const bool any_fit = __any_sync(PHR_FULL_MASK, fitting);

    int score = m, best = m, best_col = 0;
    bool stopped = false;
    int colsum = 0;  // global mode: sum of VP - VN bits of the final column (rows < m)

    // ---- forward pass: anti-diagonal lane pipeline -------------------------------
    // Bits at or above m in the last block are never masked: carries and shifts only move
    // upward, so they cannot reach a bit below m, and nothing above m is ever read.
    for (int r = 0; r < Rmax; ++r) {
        const int blk = r * G + gl;
        const bool blk_act = go && r < R && blk < nb;
        const uint64_t smask = (blk_act && blk == nb - 1) ? (1ull << score_bit) : 0ull;
        QueryBlock<S> qbk;
        if (blk_act) qbk.load(qb, 0, blk, ~0ull);
        uint64_t vp = ~0ull, vn = 0;
        const int steps = (go && r < R) ? n + G - 1 : 0;
        const int smax = __reduce_max_sync(PHR_FULL_MASK, static_cast<unsigned>(steps));
        uint32_t payload = 0;
        uint32_t tword = 0;
        bool stop_r = false;
        // first stored block of column J = j0 + 1, tracked incrementally (Band::blo)
        int blo_cur = band.blo(1 - gl > 1 ? 1 - gl : 1);
        for (int s = 0; s < smax; ++s) {
            uint32_t in = __shfl_up_sync(PHR_FULL_MASK, payload, 1, G);
            const int j0 = s - gl;
            const bool live = blk_act && j0 >= 0 && j0 < n && !stop_r;
            // every lane keeps the group's current target word; only lane 0 reads it
            if ((s % S::kPerWord) == 0 && s < n && go) tword = seq_word<S>(tb + s / S::kPerWord);
            if (live) {
                if (gl == 0) {
                    // lane 0: target symbol j0 and the carries entering block 0 of the stripe
                    const uint32_t c0 = (tword >> ((s % S::kPerWord) * S::kBits)) & ((1u << S::kBits) - 1);
                    const uint32_t cb = r == 0 ? 2u : static_cast<uint32_t>(stripe_buf[j0]);
                    in = c0 * 256u + cb;
                }
                const uint32_t c = in >> 8;
                const uint32_t addc = in & 1u;
                const uint32_t hpc = (in >> 1) & 1u;
                const uint32_t hnc = (in >> 2) & 1u;
                const uint64_t eq = qbk.eq(c);
                const uint64_t xh = eq | vn;
                uint32_t add_out;
                const uint64_t s2 = add_carry64(vp, xh & vp, addc, &add_out);
                const uint64_t d0 = (s2 ^ vp) | xh;
                const uint64_t hn = vp & d0;
                const uint64_t hp = vn | ~(vp | d0);
                const uint32_t hp_out = static_cast<uint32_t>(hp >> 63);
                const uint32_t hn_out = static_cast<uint32_t>(hn >> 63);
                const uint64_t x = (hp << 1) | hpc;
                const uint64_t hns = (hn << 1) | hnc;
                vn = x & d0;
                vp = hns | ~(d0 | x);
                payload = c * 256u + add_out + hp_out * 2u + hn_out * 4u;
                if (r < R - 1 && gl == G - 1) stripe_buf[j0] = static_cast<uint8_t>(payload & 7u);
                // band store of column J = j0 + 1; blo(J) steps by one every 64 columns
                if (((j0 + 1) - (band.E + 3)) > 0 && (((j0 + 1) - (band.E + 3)) & 63) == 0)
                    blo_cur = min(blo_cur + 1, nb - band.W);
                const int slotb = blk - blo_cur;
                if (slotb >= 0 && slotb < band.W) {
                    uint4* dst = reinterpret_cast<uint4*>(recs + (static_cast<uint64_t>(j0) * band.W + slotb) * kRecBytes);
                    *dst = make_uint4(static_cast<uint32_t>(vp), static_cast<uint32_t>(vp >> 32),
                                      static_cast<uint32_t>(hp), static_cast<uint32_t>(hp >> 32));
                }
                // fitting: score of the last block's bit m-1 per column (other lanes have
                // smask = 0); global mode reads the distance off the final column instead
                if (any_fit && !stopped) {
                    const int sc = score + ((hp & smask) ? 1 : 0) - ((hn & smask) ? 1 : 0);
                    score = sc > 0 ? sc : 0;
                    if (score < best) {
                        best = score;
                        best_col = j0 + 1;
                    }
                    if (fitting && smask && score > best + margin) stopped = true;
                }
            }
            if (any_fit && (s & 15) == 15) {
                // the group's last lane owns the score; all stop once it abandoned
                const uint32_t sv = __shfl_sync(PHR_FULL_MASK, stopped ? 1u : 0u, last_lane, G);
                if (fitting && r == R - 1) stop_r = sv != 0;
            }
        }
        if (blk_act) {
            const uint64_t rows = (blk == nb - 1 && (m & 63)) ? ((1ull << (m & 63)) - 1) : ~0ull;
            colsum += __popcll(vp & rows) - __popcll(vn & rows);
        }
        __syncwarp();
    }
    // D[m][n] = D[0][n] + sum of the vertical deltas of column n = n + sum(VP) - sum(VN)
    for (int o = 1; o < G; o <<= 1) colsum += __shfl_xor_sync(PHR_FULL_MASK, colsum, o, G);
    if (!fitting) score = n + colsum;

    // results of each group, from the lane owning the last block
    const int ed_all = __shfl_sync(PHR_FULL_MASK, fitting ? best : score, last_lane, G);
    const int end_all = __shfl_sync(PHR_FULL_MASK, fitting ? best_col : n, last_lane, G);
    const bool band_ok = ed_all <= band.E;
    const bool trace = go && band_ok;
    if (act && gl == 0 && (!fits || (go && !band_ok))) {
        const uint32_t k = atomicAdd(P.redo_count, 1u);
        P.redo_list[k] = pid;
        const uint64_t need_full = pair_need(m, n, nb, G, make_band(m, n, nb, 1, 0));
        atomicMax(P.redo_need_max, static_cast<unsigned long long>(need_full));
        if (P.redo_need) P.redo_need[k] = need_full;
    }

    // ---- traceback: every group walks its own pair, all groups in lockstep ----------
    // Window: group lane L holds column jw - L (G columns) and query blocks bw, bw+1 (128
    // rows). Each iteration classifies the current cell and consumes the whole run of
    // that move type: a D run from the column's VP bits, an I run from a ballot over the
    // row's VP/HP bits, an M or X run from a ballot along the diagonal.
    const int gbase = lane & ~(G - 1);
    const unsigned gmask = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
    RunWriter rw;
    rw.init(runs, static_cast<uint32_t>(m + n + 2), gl == 0);
    int i = trace ? m : 0, j = trace ? end_all : 0;
    int jw = -1, bw = -2;
    uint64_t lvp = 0, lhp = 0, hvp = 0, hhp = 0;
    for (;;) {
        const bool want = trace && i > 0 && j > 0;
        if (!__any_sync(PHR_FULL_MASK, want)) break;
        const int r1 = i - 1;
        const bool reload = want && (jw < 0 || j <= jw - G || (r1 >> 6) > bw + 1 || r1 < 64 * bw);
        if (reload) {
            jw = j;
            bw = (r1 >> 6) - 1;
            const int col = jw - gl;
            lvp = lhp = hvp = hhp = 0;
            if (col >= 1) {
                const int blo = band.blo(col);
                const uint8_t* base = recs + static_cast<uint64_t>(col - 1) * band.W * kRecBytes;
                const int sh = bw + 1 - blo;
                if (sh >= 0 && sh < band.W) {
                    const uint4 a = *reinterpret_cast<const uint4*>(base + sh * kRecBytes);
                    hvp = a.x | (static_cast<uint64_t>(a.y) << 32);
                    hhp = a.z | (static_cast<uint64_t>(a.w) << 32);
                }
                const int sl = bw - blo;
                if (bw >= 0 && sl >= 0 && sl < band.W) {
                    const uint4 a = *reinterpret_cast<const uint4*>(base + sl * kRecBytes);
                    lvp = a.x | (static_cast<uint64_t>(a.y) << 32);
                    lhp = a.z | (static_cast<uint64_t>(a.w) << 32);
                }
            }
        }
        const int src = want ? jw - j : 0;   // group lane holding the current column
        const int base_row = 64 * bw;        // window row 0 (may be -64)
        const int dlt = gl - src;            // diagonal offset of this lane's cell
        const int col = jw - gl;
        const int p1 = r1 - base_row;        // current row in the window, 0..127
        uint32_t vp1 = 0, hp1 = 0, dcode = 3;
        bool isI = false;
        int drun = 1;
        if (want) {
            vp1 = bit128(lvp, hvp, p1);
            hp1 = bit128(lhp, hhp, p1);
            isI = dlt >= 0 && col >= 1 && !vp1 && hp1;
            // this lane's cell on the current diagonal: 0 M, 1 X, 2 not diagonal, 3 invalid
            const int rd = r1 - dlt;
            const int pd = rd - base_row;
            if (dlt >= 0 && col >= 1 && rd >= 0 && pd >= 0) {
                if (bit128(lvp, hvp, pd) | bit128(lhp, hhp, pd)) {
                    dcode = 2;
                } else {  // diagonal: M when query byte rd equals target byte col-1
                    dcode = sym_at<S>(qb, rd) == sym_at<S>(tb, col - 1) ? 0u : 1u;
                }
            }
            // D run down this lane's column from row r1 (consecutive VP bits, downward)
            const int p = p1;
            const uint64_t hi = p >= 64 ? (p == 127 ? hvp : ((hvp << (127 - p)) | (lvp >> (p - 63)))) : (lvp << (63 - p));
            const uint64_t lo = p >= 64 ? (lvp << (127 - p)) : 0ull;
            drun = ~hi ? __clzll(~hi) : 64 + (~lo ? __clzll(~lo) : 64);
            drun = min(drun, p + 1);
        }
        const int src_lane = gbase + src;
        const uint32_t cur = __shfl_sync(PHR_FULL_MASK, vp1 | (hp1 << 1) | (dcode << 2), src_lane);
        const int drun_src = __shfl_sync(PHR_FULL_MASK, drun, src_lane);
        const unsigned mI = (__ballot_sync(PHR_FULL_MASK, isI) >> gbase) & gmask;
        const unsigned mM = (__ballot_sync(PHR_FULL_MASK, dcode == 0) >> gbase) & gmask;
        const unsigned mX = (__ballot_sync(PHR_FULL_MASK, dcode == 1) >> gbase) & gmask;
        if (want) {
            int op, run;
            if (cur & 1u) {
                op = 3;  // D: query-extra
                run = drun_src;
            } else {
                unsigned sh;
                if (cur & 2u) {
                    op = 2;  // I: target-extra
                    sh = mI >> src;
                } else {
                    op = ((cur >> 2) & 3u) == 0 ? 0 : 1;
                    sh = (op == 0 ? mM : mX) >> src;
                }
                run = (~sh) ? __ffs(~sh) - 1 : 32 - src;
                run = min(run, G - src);
            }
            run = max(run, 1);
            rw.push(static_cast<uint32_t>(op), static_cast<uint32_t>(run));
            if (op == 3) {
                i -= run;
            } else if (op == 2) {
                j -= run;
            } else {
                i -= run;
                j -= run;
            }
        }
    }
    if (trace) {
        if (i > 0) rw.push(3, static_cast<uint32_t>(i));
        if (j > 0) rw.push(2, static_cast<uint32_t>(j));
        rw.flush();
    }
    __syncwarp();
    // every group lane tracked the same runs; the group leader stored them
    const uint32_t nr = rw.n;
    const bool fmt = trace && !rw.overflow;
    const uint32_t nr_fmt = fmt ? nr : 0;
    const uint32_t nrmax = __reduce_max_sync(PHR_FULL_MASK, nr_fmt);
    const uint32_t rounds = (nrmax + G - 1) / G;
    char* out = act ? P.text + P.text_off[pid] : nullptr;
    uint32_t tl = 0;
    for (uint32_t rr = 0; rr < rounds; ++rr) {
        const uint32_t c = rr * G + gl;
        uint32_t len = 0, run = 0;
        if (c < nr_fmt) {
            run = runs[nr_fmt - 1 - c];
            len = ndigits(run >> 2) + 1;
        }
        const uint32_t incl = group_incl_scan(len, G);
        if (c < nr_fmt) {
            char* pp = out + tl + incl - len;
            uint32_t v = run >> 2;
            const uint32_t nd = len - 1;
            for (int dd = static_cast<int>(nd) - 1; dd >= 0; --dd) {
                pp[dd] = static_cast<char>('0' + v % 10);
                v /= 10;
            }
            pp[nd] = op_char(run & 3);
        }
        tl += __shfl_sync(PHR_FULL_MASK, incl, G - 1, G);
    }
    if (fmt && gl == 0) {
        PairOut o;
        o.status = PHR_OK;
        o.ed = ed_all;
        o.t_consumed = end_all;
        o.affine_score = 0;
        o.n_runs = nr;
        o.text_len = tl;
        P.out[pid] = o;
    }
    if (trace && rw.overflow && gl == 0) atomicOr(P.error_flag, 1u);
}

template <class S>
__global__ void __launch_bounds__(256, 3) myers_kernel(ExtendParams P) {
    const int lane = lane_id();
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = P.tasks.range[0] + atomicAdd(P.queue_head, 1u);
        task = __shfl_sync(PHR_FULL_MASK, task, 0);
        if (task >= P.tasks.range[1]) break;
        uint8_t* slot = P.task_off ? P.scratch + P.task_off[task] : P.scratch + warp_global * P.slot_bytes;
        const uint64_t slot_bytes = P.task_off ? P.task_len[task] : P.slot_bytes;
        const int G = P.tasks.task_group[task];
        const int count = P.tasks.task_count[task];
        const int grp = lane / G;
        const bool act = grp < count;
        const uint32_t pid = act ? P.tasks.order[P.tasks.task_first[task] + grp] : 0;
        PairDesc d = {};
        if (act) d = P.desc[pid];
        // skip pairs of the other symbol mode; they run in the other instantiation
        const bool mine = act && (d.mode == (S::kBits == 2 ? 0 : 1));
        const int m = mine ? d.qn : 0, n = mine ? d.tn : 0;
        const int nb = (m + 63) >> 6;
        const Band band = make_band(m, n, nb, P.full_band, P.band_base);
        const uint64_t need = mine ? pair_need(m, n, nb, G, band) : 0;
        // exclusive prefix of needs over the groups of this warp (one value per group)
        uint64_t excl = 0, total = 0;
        for (int g = 0; g < 32 / G; ++g) {
            const uint64_t v = __shfl_sync(PHR_FULL_MASK, need, g * G);
            if (g < grp) excl += v;
            total += v;
        }
        const bool fits = total <= slot_bytes;
        if (!__any_sync(PHR_FULL_MASK, mine)) continue;
        myers_group<S>(P, d, pid, mine, G, slot, excl, fits);
    }
}

}  // namespace

void launch_myers(const ExtendParams& p, int grid, int block, cudaStream_t st) {
    myers_kernel<Seq2><<<grid, block, 0, st>>>(p);
}

void launch_myers_bytes(const ExtendParams& p, int grid, int block, cudaStream_t st) {
    myers_kernel<SeqB><<<grid, block, 0, st>>>(p);
}

}  // namespace phr

// ===========================================================================
// Allocation-free Myers fitting extension (phr_myers_extend_noalloc).
//
// Its scratch is the file-scope array below: 256 bytes of control words (pair counter,
// error flags) followed by one fixed slice per worker warp. A slice holds the pair's
// bookkeeping header, both sequences copied into word-aligned staging, and the
// full-band records + runs myers_group needs; the length limits make every pair fit
// its slice, so no redo pass (and no allocation) is ever needed.
// ===========================================================================
namespace phr {
namespace {

constexpr int kNoAllocWarps = 128;
// Control block at the start of the array (zeroed by every call): the error flags word
// (bit 0: a pair beyond the length limits, bit 1: a pair that did not finish) at byte
// kNoAllocFlagsByte, read back by the host, and the 64-bit next-pair counter at byte
// kNoAllocCounterByte.
constexpr uint64_t kNoAllocCtl = 256;
constexpr uint64_t kNoAllocFlagsByte = 4;
constexpr uint64_t kNoAllocCounterByte = 8;
constexpr uint64_t kNoAllocSlice = (PHR_NOALLOC_SCRATCH_BYTES - kNoAllocCtl) / kNoAllocWarps / 256 * 256;
constexpr uint64_t kNoAllocHeader = 256;
constexpr uint64_t kNoAllocStageQ = (PHR_NOALLOC_MAX_QUERY / 4 + 8) * 4;
constexpr uint64_t kNoAllocStageT = (PHR_NOALLOC_MAX_TARGET / 4 + 8) * 4;
constexpr uint64_t kNoAllocWork = kNoAllocHeader + kNoAllocStageQ + kNoAllocStageT;
// worst pair: full band of ceil(512/64) = 8 blocks x 1024 columns x 32 B + runs
static_assert(kNoAllocWork + 1024ull * 8 * 32 + (1024 + 512 + 2) * 4 + 64 <= kNoAllocSlice,
              "no-alloc slice too small for the stated limits");

struct NoAllocArgs {
    const uint8_t* seq;
    const uint64_t* q_off;
    const uint32_t* q_len;
    const uint64_t* t_off;
    const uint32_t* t_len;
    uint64_t n;
    int32_t* status;
    uint32_t* ed;
    uint32_t* consumed;
    char* cigar;
    uint32_t stride;
    uint32_t* cigar_len;
    uint8_t* scratch;    // device address of g_noalloc_scratch
};

__device__ uint32_t noalloc_write_count_op(char* p, uint32_t n, char op) {
    const uint32_t nd = ndigits(n);
    for (int d = static_cast<int>(nd) - 1; d >= 0; --d) {
        p[d] = static_cast<char>('0' + n % 10);
        n /= 10;
    }
    p[nd] = op;
    return nd + 1;
}

__global__ void __launch_bounds__(256) myers_noalloc_kernel(NoAllocArgs A) {
    const int lane = lane_id();
    const uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    uint32_t* flags = reinterpret_cast<uint32_t*>(A.scratch + kNoAllocFlagsByte);
    unsigned long long* next_pair = reinterpret_cast<unsigned long long*>(A.scratch + kNoAllocCounterByte);
    uint8_t* slice = A.scratch + kNoAllocCtl + w * kNoAllocSlice;
    PairOut* pout = reinterpret_cast<PairOut*>(slice);
    uint64_t* toff = reinterpret_cast<uint64_t*>(slice + 64);
    uint32_t* err = reinterpret_cast<uint32_t*>(slice + 72);
    uint32_t* rcount = reinterpret_cast<uint32_t*>(slice + 76);
    unsigned long long* rneed = reinterpret_cast<unsigned long long*>(slice + 80);
    uint32_t* rlist = reinterpret_cast<uint32_t*>(slice + 88);
    uint32_t* stage = reinterpret_cast<uint32_t*>(slice + kNoAllocHeader);
    uint8_t* work = slice + kNoAllocWork;
    for (;;) {
        uint64_t i = 0;
        if (lane == 0) i = atomicAdd(next_pair, 1ull);
        i = __shfl_sync(PHR_FULL_MASK, i, 0);
        if (i >= A.n) break;
        const uint32_t ql = A.q_len[i], tl = A.t_len[i];
        char* text = A.cigar + i * A.stride;
        if (ql > PHR_NOALLOC_MAX_QUERY || tl > PHR_NOALLOC_MAX_TARGET) {
            if (lane == 0) {
                A.status[i] = PHR_ERR_ARG;
                A.ed[i] = 0;
                A.consumed[i] = 0;
                A.cigar_len[i] = 0;
                atomicOr(flags, 1u);
            }
            continue;
        }
        if (ql == 0 || tl == 0) {  // wfa_simd.rs:3793-3798
            if (lane == 0) {
                A.status[i] = PHR_OK;
                A.ed[i] = ql;
                A.consumed[i] = 0;
                A.cigar_len[i] = ql ? noalloc_write_count_op(text, ql, 'D') : 0;
            }
            continue;
        }
        // word-aligned staging of both sequences (byte mode: 4 symbols per word)
        const uint32_t qw = (ql + 3) / 4 + 4;
        const uint8_t* qs = A.seq + A.q_off[i];
        const uint8_t* ts = A.seq + A.t_off[i];
        for (uint32_t k = lane; k < qw; k += 32) {
            uint32_t word = 0;
            for (uint32_t b = 0; b < 4; ++b) {
                const uint32_t p = 4 * k + b;
                if (p < ql) word |= static_cast<uint32_t>(qs[p]) << (8 * b);
            }
            stage[k] = word;
        }
        const uint32_t tw = (tl + 3) / 4 + 4;
        for (uint32_t k = lane; k < tw; k += 32) {
            uint32_t word = 0;
            for (uint32_t b = 0; b < 4; ++b) {
                const uint32_t p = 4 * k + b;
                if (p < tl) word |= static_cast<uint32_t>(ts[p]) << (8 * b);
            }
            stage[qw + k] = word;
        }
        if (lane == 0) {
            *toff = i * A.stride;
            *err = 0;
            *rcount = 0;
            *rneed = 0;
            PairOut o = {};
            o.status = -1;
            *pout = o;
        }
        __syncwarp();
        ExtendParams P{};
        P.out = pout;
        P.bytes = stage;
        P.packed2 = stage;
        P.text = A.cigar;
        P.text_off = toff;
        P.redo_list = rlist;
        P.redo_count = rcount;
        P.redo_need_max = rneed;
        P.engine = PHR_ENGINE_MYERS_FIT;
        P.full_band = 1;
        P.band_base = 0;
        P.error_flag = err;
        PairDesc d = {};
        d.q_word = 0;
        d.t_word = qw;
        d.qn = static_cast<int32_t>(ql);
        d.tn = static_cast<int32_t>(tl);
        d.mode = 1;
        int G = 1;
        const int nb = static_cast<int>((ql + 63) / 64);
        while (G < nb) G <<= 1;
        // the staged words were written by this warp above: coherent loads (SeqBc)
        myers_group<SeqBc>(P, d, 0, lane < G, G, work, 0, true);
        __syncwarp();
        if (lane == 0) {
            const PairOut o = *pout;
            const bool ok = o.status == PHR_OK && *err == 0 && *rcount == 0;
            A.status[i] = ok ? PHR_OK : PHR_ERR_CUDA;
            A.ed[i] = ok ? static_cast<uint32_t>(o.ed) : 0;
            A.consumed[i] = ok ? static_cast<uint32_t>(o.t_consumed) : 0;
            A.cigar_len[i] = ok ? o.text_len : 0;
            if (!ok) atomicOr(flags, 2u);
        }
        __syncwarp();
    }
}

}  // namespace

// One fixed scratch array per GPU that loads the library.
static __device__ __align__(256) uint8_t g_noalloc_scratch[PHR_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch for the current device, looked up once per device.
static cudaError_t noalloc_scratch_address(uint8_t** out) {
    static std::mutex mu;
    static uint8_t* addr[256] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        addr[dev] = static_cast<uint8_t*>(p);
    }
    *out = addr[dev];
    return cudaSuccess;
}

}  // namespace phr

extern "C" phr_status phr_myers_extend_noalloc(const uint8_t* seq, const uint64_t* q_off, const uint32_t* q_len,
                                               const uint64_t* t_off, const uint32_t* t_len, uint64_t n_pairs,
                                               int32_t* status, uint32_t* edit_distance, uint32_t* target_consumed,
                                               char* cigar, uint32_t cigar_stride, uint32_t* cigar_len,
                                               void* stream) {
    if (n_pairs == 0) return PHR_OK;
    if (!seq || !q_off || !q_len || !t_off || !t_len || !status || !edit_distance || !target_consumed || !cigar ||
        !cigar_len)
        return PHR_ERR_ARG;
    if (cigar_stride < PHR_NOALLOC_CIGAR_STRIDE) return PHR_ERR_ARG;
    uint8_t* scratch = nullptr;
    if (phr::noalloc_scratch_address(&scratch) != cudaSuccess) return PHR_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the control words (pair counter, error flags) must start at zero on every call
    if (cudaMemsetAsync(scratch, 0, phr::kNoAllocCtl, st) != cudaSuccess) return PHR_ERR_CUDA;
    phr::NoAllocArgs A{seq, q_off, q_len, t_off, t_len, n_pairs, status, edit_distance, target_consumed,
                       cigar, cigar_stride, cigar_len, scratch};
    phr::myers_noalloc_kernel<<<phr::kNoAllocWarps * 32 / 256, 256, 0, st>>>(A);
    if (cudaGetLastError() != cudaSuccess) return PHR_ERR_CUDA;
    uint32_t flags = 0;
    if (cudaMemcpyAsync(&flags, scratch + phr::kNoAllocFlagsByte, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return PHR_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PHR_ERR_CUDA;
    if (flags & 2u) return PHR_ERR_CUDA;
    if (flags & 1u) return PHR_ERR_ARG;
    return PHR_OK;
}
