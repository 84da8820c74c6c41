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
// already computes); a diagonal move is a match iff -VN(i-1) + dh(i-1, j) == 0, with
// dh(0, j) = 1 (top row D[0][j] = j). So the forward pass stores {VP, VN, HP, HN} per
// (column, block) and the traceback walks bits, never values. Only the blocks within
// a band |i - j| <= E + 2 are stored: every cell of an alignment of cost ed satisfies
// |i - j| <= ed, so the walk stays in the band whenever ed <= E; pairs with ed > E are
// redone with every block stored (full_band).
#include <mutex>

#include "kernels.cuh"

namespace phr {
namespace {

constexpr int kRecBytes = 32;  // VP, VN, HP, HN of one 64-bit block of one column

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
        int E = base + abs(m - n) + (m >> 3);
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

template <>
struct QueryBlock<SeqB> {
    uint32_t w[16];
    uint64_t mask;
    __device__ __forceinline__ void load(const uint32_t* q, int qsh, int blk, uint64_t msk) {
#pragma unroll
        for (int k = 0; k < 16; ++k) w[k] = load_window<SeqB>(q, qsh + blk * 64 + 4 * k);
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

template <class S>
__device__ __forceinline__ const uint32_t* seq_base(const ExtendParams& P, uint64_t word) {
    return (S::kBits == 2 ? P.packed2 : P.bytes) + word;
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
    const int qsh = 0, tsh = 0;

    uint8_t* recs = slot + slot_off;
    uint64_t off = align16(static_cast<uint64_t>(n) * band.W * kRecBytes);
    uint8_t* stripe_buf = recs + off;
    if (nb > G) off += align16(static_cast<uint64_t>(n));
    uint32_t* runs = reinterpret_cast<uint32_t*>(recs + off);

    const bool go = act && fits;
    const int R = go ? (nb + G - 1) / G : 0;
    const int Rmax = __reduce_max_sync(PHR_FULL_MASK, static_cast<unsigned>(R));
    const int last_lane = (nb - 1) % G;
    const uint64_t last_mask = (m & 63) ? ((1ull << (m & 63)) - 1) : ~0ull;
    const int score_bit = (m - 1) & 63;
    const int margin = m / 10 + 1;

    int score = m, best = m, best_col = 0, ncols = n;
    bool stopped = false;

    for (int r = 0; r < Rmax; ++r) {
        const int blk = r * G + gl;
        const bool blk_act = go && r < R && blk < nb;
        const bool is_last = blk_act && blk == nb - 1;
        const uint64_t bmask = (blk == nb - 1) ? last_mask : ~0ull;
        QueryBlock<S> qbk;
        if (blk_act) qbk.load(qb, qsh, blk, bmask);
        uint64_t vp = bmask, vn = 0;
        const int steps = (go && r < R) ? n + G - 1 : 0;
        const int smax = __reduce_max_sync(PHR_FULL_MASK, static_cast<unsigned>(steps));
        uint32_t payload = 0;
        bool stop_r = false;
        for (int s = 0; s < smax; ++s) {
            const uint32_t in = __shfl_up_sync(PHR_FULL_MASK, payload, 1, G);
            const int j0 = s - gl;
            const bool live = blk_act && j0 >= 0 && j0 < n && !stop_r;
            if (live) {
                uint32_t c, addc, hpc, hnc;
                if (gl == 0) {
                    c = sym_at<S>(tb, j0 + tsh);
                    if (r == 0) {
                        addc = 0;
                        hpc = 1;
                        hnc = 0;
                    } else {
                        const uint32_t cb = stripe_buf[j0];
                        addc = cb & 1;
                        hpc = (cb >> 1) & 1;
                        hnc = (cb >> 2) & 1;
                    }
                } else {
                    c = in & 0xffu;
                    addc = (in >> 8) & 1;
                    hpc = (in >> 9) & 1;
                    hnc = (in >> 10) & 1;
                }
                const uint64_t eq = qbk.eq(c);
                const uint64_t xh = eq | vn;
                const uint64_t xhvp = xh & vp;
                const uint64_t s1 = vp + xhvp;
                const uint64_t c1 = s1 < vp ? 1ull : 0ull;
                const uint64_t s2 = s1 + addc;
                const uint64_t c2 = s2 < s1 ? 1ull : 0ull;
                const uint32_t add_out = static_cast<uint32_t>(c1 | c2);
                uint64_t d0 = (s2 ^ vp) | xh;
                uint64_t hn = vp & d0;
                uint64_t hp = vn | ~(vp | d0);
                d0 &= bmask;
                hn &= bmask;
                hp &= bmask;
                const uint32_t hp_out = static_cast<uint32_t>(hp >> 63);
                const uint32_t hn_out = static_cast<uint32_t>(hn >> 63);
                const uint64_t x = (hp << 1) | hpc;
                const uint64_t hns = (hn << 1) | hnc;
                const uint64_t nvn = x & d0;
                const uint64_t nvp = (hns | ~(d0 | x)) & bmask;
                vp = nvp;
                vn = nvn;
                payload = c | (add_out << 8) | (hp_out << 9) | (hn_out << 10);
                if (r < R - 1 && gl == G - 1) stripe_buf[j0] = static_cast<uint8_t>(add_out | (hp_out << 1) | (hn_out << 2));
                // band store of column J = j0 + 1
                const int blo = band.blo(j0 + 1);
                const int slotb = blk - blo;
                if (slotb >= 0 && slotb < band.W) {
                    uint4* dst = reinterpret_cast<uint4*>(recs + (static_cast<uint64_t>(j0) * band.W + slotb) * kRecBytes);
                    dst[0] = make_uint4(static_cast<uint32_t>(vp), static_cast<uint32_t>(vp >> 32),
                                        static_cast<uint32_t>(vn), static_cast<uint32_t>(vn >> 32));
                    dst[1] = make_uint4(static_cast<uint32_t>(hp), static_cast<uint32_t>(hp >> 32),
                                        static_cast<uint32_t>(hn), static_cast<uint32_t>(hn >> 32));
                }
                if (is_last) {
                    if ((hp >> score_bit) & 1) score += 1;
                    if ((hn >> score_bit) & 1) score = score > 0 ? score - 1 : 0;
                    if (score < best) {
                        best = score;
                        best_col = j0 + 1;
                    }
                    if (fitting && score > best + margin) {
                        stopped = true;
                        ncols = j0 + 1;
                    }
                }
            }
            // the group's last lane owns the score; everyone stops when it abandons
            const uint32_t sv = __shfl_sync(PHR_FULL_MASK, stopped ? 1u : 0u, last_lane, G);
            if (fitting && r == R - 1) stop_r = sv != 0;
        }
        __syncwarp();
    }
    (void)ncols;

    // broadcast results from the lane owning the last block
    const int ed_all = __shfl_sync(PHR_FULL_MASK, fitting ? best : score, last_lane, G);
    const int end_all = __shfl_sync(PHR_FULL_MASK, fitting ? best_col : n, last_lane, G);
    const bool band_ok = ed_all <= band.E;
    const bool trace = go && band_ok;
    if (act && gl == 0 && (!fits || (go && !band_ok))) {
        const uint32_t k = atomicAdd(P.redo_count, 1u);
        P.redo_list[k] = pid;
        const uint64_t need_full = pair_need(m, n, nb, G, make_band(m, n, nb, 1, 0));
        atomicMax(P.redo_need_max, static_cast<unsigned long long>(need_full));
    }

    // ---- traceback: group-cooperative bit walk ---------------------------------
    RunWriter rw;
    rw.init(runs, static_cast<uint32_t>(m + n + 2), gl == 0);
    int i = trace ? m : 0;
    int j = trace ? end_all : 0;
    // window: lane gl holds column (jw - gl), blocks bw (lo) and bw+1 (hi) of that column
    int jw = -1, bw = -1;
    uint64_t lo_vp = 0, lo_vn = 0, lo_hp = 0, lo_hn = 0, hi_vp = 0, hi_vn = 0, hi_hp = 0, hi_hn = 0;
    for (;;) {
        const bool want = trace && i > 0 && j > 0;
        if (!__any_sync(PHR_FULL_MASK, want)) break;
        // (re)load the window when the current cell is outside it
        const int r1 = i - 1;  // query row bit of cell (i, j)
        const bool need_load =
            want && (jw < 0 || j > jw || j <= jw - G || (r1 >> 6) > bw + 1 || r1 < 64 * bw + 1);
        if (__any_sync(PHR_FULL_MASK, need_load)) {
            if (need_load) {
                jw = j;
                const int bhi = r1 >> 6;
                bw = bhi - 1;  // may be -1: then the lo block is absent
                const int col = jw - gl;
                lo_vp = lo_vn = lo_hp = lo_hn = hi_vp = hi_vn = hi_hp = hi_hn = 0;
                if (col >= 1) {
                    const int blo = band.blo(col);
                    const uint8_t* base = recs + static_cast<uint64_t>(col - 1) * band.W * kRecBytes;
                    const int sh = bhi - blo;
                    if (sh >= 0 && sh < band.W) {
                        const uint4 a = reinterpret_cast<const uint4*>(base + sh * kRecBytes)[0];
                        const uint4 b = reinterpret_cast<const uint4*>(base + sh * kRecBytes)[1];
                        hi_vp = a.x | (static_cast<uint64_t>(a.y) << 32);
                        hi_vn = a.z | (static_cast<uint64_t>(a.w) << 32);
                        hi_hp = b.x | (static_cast<uint64_t>(b.y) << 32);
                        hi_hn = b.z | (static_cast<uint64_t>(b.w) << 32);
                    }
                    const int sl = bw - blo;
                    if (bw >= 0 && sl >= 0 && sl < band.W) {
                        const uint4 a = reinterpret_cast<const uint4*>(base + sl * kRecBytes)[0];
                        const uint4 b = reinterpret_cast<const uint4*>(base + sl * kRecBytes)[1];
                        lo_vp = a.x | (static_cast<uint64_t>(a.y) << 32);
                        lo_vn = a.z | (static_cast<uint64_t>(a.w) << 32);
                        lo_hp = b.x | (static_cast<uint64_t>(b.y) << 32);
                        lo_hn = b.z | (static_cast<uint64_t>(b.w) << 32);
                    }
                }
            }
        }
        // every lane extracts the decision bits of row r1 (and r1-1) for its own column
        uint32_t bits = 0;
        if (want) {
            const int b1 = r1 >> 6, o1 = r1 & 63;
            const uint64_t vpw = (b1 == bw + 1) ? hi_vp : lo_vp;
            const uint64_t vnw = (b1 == bw + 1) ? hi_vn : lo_vn;
            const uint64_t hpw = (b1 == bw + 1) ? hi_hp : lo_hp;
            bits |= static_cast<uint32_t>((vpw >> o1) & 1);
            bits |= static_cast<uint32_t>((hpw >> o1) & 1) << 1;
            bits |= static_cast<uint32_t>((vnw >> o1) & 1) << 2;
            if (r1 >= 1) {
                const int r0 = r1 - 1;
                const int b0 = r0 >> 6, o0 = r0 & 63;
                const uint64_t hp0 = (b0 == bw + 1) ? hi_hp : lo_hp;
                const uint64_t hn0 = (b0 == bw + 1) ? hi_hn : lo_hn;
                bits |= static_cast<uint32_t>((hp0 >> o0) & 1) << 3;
                bits |= static_cast<uint32_t>((hn0 >> o0) & 1) << 4;
            }
        }
        const int src = want ? (jw - j) : gl;
        const uint32_t cb = __shfl_sync(PHR_FULL_MASK, bits, src, G);
        if (want) {
            if (cb & 1) {
                rw.push(3, 1);  // D: query-extra
                --i;
            } else if (cb & 2) {
                rw.push(2, 1);  // I: target-extra
                --j;
            } else {
                const int dh = (r1 >= 1) ? static_cast<int>((cb >> 3) & 1) - static_cast<int>((cb >> 4) & 1) : 1;
                const int cost = dh - static_cast<int>((cb >> 2) & 1);
                rw.push(cost == 0 ? 0 : 1, 1);
                --i;
                --j;
            }
        }
    }
    if (trace) {
        if (i > 0) rw.push(3, static_cast<uint32_t>(i));
        if (j > 0) rw.push(2, static_cast<uint32_t>(j));
        rw.flush();
    }
    __syncwarp();
    // every group lane tracked the same runs; lane 0's writes are the ones that landed
    const uint32_t nr = rw.n;
    const bool fmt = trace && !rw.overflow;
    uint32_t tl = 0;
    {
        const uint32_t nr_fmt = fmt ? nr : 0;
        const uint32_t nrmax = __reduce_max_sync(PHR_FULL_MASK, nr_fmt);
        (void)nrmax;
        // groups format independently; format_runs_group loops to the group's own count,
        // so keep every lane of the warp in the same loop by iterating to the warp max
        const int l = gl;
        uint32_t base = 0;
        const uint32_t rounds = (nrmax + G - 1) / G;
        char* out = act ? P.text + P.text_off[pid] : nullptr;
        for (uint32_t rr = 0; rr < rounds; ++rr) {
            const uint32_t c = rr * G + l;
            uint32_t len = 0, run = 0;
            if (c < nr_fmt) {
                run = runs[nr_fmt - 1 - c];
                len = ndigits(run >> 2) + 1;
            }
            const uint32_t incl = group_incl_scan(len, G);
            if (c < nr_fmt) {
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
        tl = base;
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
__global__ void __launch_bounds__(256) myers_kernel(ExtendParams P) {
    const int lane = lane_id();
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    uint8_t* slot = P.scratch + warp_global * P.slot_bytes;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = P.tasks.range[0] + atomicAdd(P.queue_head, 1u);
        task = __shfl_sync(PHR_FULL_MASK, task, 0);
        if (task >= P.tasks.range[1]) break;
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
        const bool fits = total <= P.slot_bytes;
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
constexpr uint64_t kNoAllocCtl = 256;
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
    uint32_t* ctl = reinterpret_cast<uint32_t*>(A.scratch);  // [0] next pair, [1] error flags
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
        if (lane == 0) i = atomicAdd(reinterpret_cast<unsigned long long*>(ctl + 2), 1ull);
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
                atomicOr(ctl + 1, 1u);
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
        myers_group<SeqB>(P, d, 0, lane < G, G, work, 0, true);
        __syncwarp();
        if (lane == 0) {
            const PairOut o = *pout;
            const bool ok = o.status == PHR_OK && *err == 0 && *rcount == 0;
            A.status[i] = ok ? PHR_OK : PHR_ERR_CUDA;
            A.ed[i] = ok ? static_cast<uint32_t>(o.ed) : 0;
            A.consumed[i] = ok ? static_cast<uint32_t>(o.t_consumed) : 0;
            A.cigar_len[i] = ok ? o.text_len : 0;
            if (!ok) atomicOr(ctl + 1, 2u);
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
    if (cudaMemcpyAsync(&flags, scratch + 4, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return PHR_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PHR_ERR_CUDA;
    if (flags & 2u) return PHR_ERR_CUDA;
    if (flags & 1u) return PHR_ERR_ARG;
    return PHR_OK;
}
