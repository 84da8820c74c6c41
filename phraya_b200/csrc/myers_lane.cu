// myers_lane.cu -- banded Myers edit distance with CIGAR, one pair per lane (sm_100a).
//
// Serves the global engine (myers_edit_distance, phraya-align/src/lib.rs:94-96 ->
// myers_edit_distance_impl, wfa_simd.rs:3657-3673) for 2-bit pairs: distance plus the
// traceback of myers_backtrace_flat (wfa_simd.rs:3702-3781: precedence D, I, diagonal).
//
// Method. Myers' block algorithm (Myers 1999, "A fast bit-vector algorithm for
// approximate string matching based on dynamic programming", section 4): a column is
// cut into 64-row blocks and the only value crossing a block boundary is the horizontal
// delta hin in {-1, 0, +1} of the row above the block. Each lane owns one pair and walks
// its columns; per column it updates a window of P consecutive blocks (registers
// vp/vn, one pair of 64-bit words per block) and passes hin down the window in
// registers. Peq (the match masks of a block for the four bases) sits in shared
// memory, [slot][base][lane], so a lane's 64-bit loads never share a bank pair.
//
// Band. Every cell of an alignment of cost ed satisfies |i-j| + |(m-i)-(n-j)| <= ed, so
// its diagonal d = j - i lies in [dmin, dmax] (lane_band, kernels.cuh) when ed <= E.
// The window at column j starts at block blo(j) = max(0, floor((j - dmax - 1) / 64)):
//  * rows above the window are replaced by hin = +1 at its top, i.e. D'[r][j] =
//    D'[r][j-1] + 1, an upper bound of the true value (an insertion step);
//  * a block entering at the bottom starts as vp = all ones, vn = 0 (D' grows by one
//    per row down from the block's top), also an upper bound (deletion steps).
// So D' >= D everywhere, and D' = D on every cell whose optimal paths stay inside
// [dmin, dmax]: P = ceil((dmax - dmin + 127) / 64) blocks keep both replaced regions
// strictly outside the band. Traceback decisions compare D'(cell) with D'(above) + 1 /
// D'(left) + 1; on a cell of the reference's path (inside the band, D' = D) the test
// holds for D' exactly when it holds for D, because D' >= D and a neighbour with
// D = cur - 1 lies on an optimal path as well. Hence, when ed <= E, the walk visits
// the reference's path and its cost (X + I + D count) is ed. When ed > E the walk
// either leaves the band (checked at every run end; the band is convex and runs are
// straight) or stays inside it, where D' obeys the DP recurrence and the cost equals
// D'(m, n) >= ed > E. Either way the pair is redone by the warp-group kernel with
// every block (myers.cu), so every reported result equals the reference's.
//
// Records. Per column and slot a 16-byte {VP, HP} record, laid out [column group][slot]
// [lane][column in group] (kLaneColGroup columns per group; with one, a warp's stores of
// one column and slot are 512 contiguous bytes). VP bit r is D[r+1][j] - D[r][j] == +1
// ("cur == above + 1"), HP bit r is D[r+1][j] - D[r+1][j-1] == +1 ("cur == left + 1").
#include "kernels.cuh"

namespace phr {
namespace {

constexpr int kLaneWarps = kLaneThreads / 32;
constexpr int kTraceCols = 16;  // columns whose records one traceback refill loads
static_assert(kTraceCols * 32 * 16 <= kLaneMaxSlots * 4 * 32 * 8, "traceback slots exceed the Peq area");

__device__ __forceinline__ uint32_t even_bits(uint32_t x) {
    x &= 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
    x = (x | (x >> 4)) & 0x00FF00FFu;
    x = (x | (x >> 8)) & 0x0000FFFFu;
    return x;
}

// Match masks of a 2-bit query block from its four words: bit r of e[c] is set when
// base r of the block equals c.
__device__ __forceinline__ void peq_words(const uint32_t qw[4], uint64_t e[4]) {
    e[0] = e[1] = e[2] = e[3] = 0;
#pragma unroll
    for (int wi = 0; wi < 4; ++wi) {
        const uint32_t w = qw[wi];
        const int sh = wi * 16;
        e[0] |= static_cast<uint64_t>(even_bits(~(w | (w >> 1)))) << sh;
        const uint32_t x1 = w ^ 0x55555555u;
        e[1] |= static_cast<uint64_t>(even_bits(~(x1 | (x1 >> 1)))) << sh;
        const uint32_t x2 = w ^ 0xAAAAAAAAu;
        e[2] |= static_cast<uint64_t>(even_bits(~(x2 | (x2 >> 1)))) << sh;
        const uint32_t x3 = ~w;
        e[3] |= static_cast<uint64_t>(even_bits(~(x3 | (x3 >> 1)))) << sh;
    }
}

__device__ __forceinline__ void load_block_words(const uint32_t* __restrict__ q, int b, uint32_t qw[4]) {
#pragma unroll
    for (int wi = 0; wi < 4; ++wi) qw[wi] = __ldg(q + b * 4 + wi);
}

__device__ __forceinline__ uint32_t lo32(uint64_t x) { return static_cast<uint32_t>(x); }
__device__ __forceinline__ uint32_t hi32(uint64_t x) { return static_cast<uint32_t>(x >> 32); }
__device__ __forceinline__ uint64_t mk64(uint32_t lo, uint32_t hi) {
    return (static_cast<uint64_t>(hi) << 32) | lo;
}

// (x << 1) | bit 31 of `above_hi` (the carry out of the block above).
__device__ __forceinline__ uint64_t shl1_in(uint64_t x, uint32_t above_hi) {
    return mk64(__funnelshift_l(above_hi, lo32(x), 1), __funnelshift_l(lo32(x), hi32(x), 1));
}

// One block, one column. pa / ma: high words of the block above's Ph / Mh (their bit 31
// is hin = +1 / -1); replaced by this block's on return. TOP: hin = +1.
template <bool TOP>
__device__ __forceinline__ uint64_t advance_block(uint64_t& vp, uint64_t& vn, uint64_t eq, uint32_t& pa,
                                                  uint32_t& ma) {
    const uint32_t a_p = TOP ? 0x80000000u : pa;
    const uint32_t a_m = TOP ? 0u : ma;
    const uint64_t xv = eq | vn;
    const uint64_t eqh = TOP ? eq : (eq | static_cast<uint64_t>(a_m >> 31));
    const uint64_t xh = (((eqh & vp) + vp) ^ vp) | eqh;
    const uint64_t ph = vn | ~(xh | vp);
    const uint64_t mh = vp & xh;
    const uint64_t phs = shl1_in(ph, a_p);
    const uint64_t mhs = shl1_in(mh, a_m);
    vp = mhs | ~(xv | phs);
    vn = phs & xv;
    pa = hi32(ph);
    ma = hi32(mh);
    return ph;
}

// Byte offset of the record of column index j0 (column j0 + 1), slot k, lane `lane`.
template <int P>
__device__ __forceinline__ uint64_t rec_off(int j0, int k, int lane) {
    return (static_cast<uint64_t>(j0 / kLaneColGroup) * P + k) * (512 * kLaneColGroup) + lane * (16 * kLaneColGroup) +
           (j0 % kLaneColGroup) * 16;
}

struct LaneGeom {
    int P;        // blocks in the window
    int dmin, dmax;
    int n_max, m_max, nb_max;
    bool slide;   // window moves (P < nb_max)
};

__device__ __forceinline__ int lane_blo(const LaneGeom& g, int j) {
    if (!g.slide) return 0;
    const int x = j - g.dmax - 1;
    return x > 0 ? (x >> 6) : 0;
}

template <int P>
__device__ __forceinline__ void lane_forward(const uint32_t* __restrict__ qb, const uint32_t* __restrict__ tb, int n,
                                             int nb, const LaneGeom& g, uint64_t* sp, uint8_t* rec) {
    const int lane = lane_id();
    uint64_t vp[P], vn[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
        uint64_t e[4] = {0, 0, 0, 0};
        if (k < nb) {
            uint32_t qw[4];
            load_block_words(qb, k, qw);
            peq_words(qw, e);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) sp[(k * 4 + c) * 32 + lane] = e[c];
        vp[k] = ~0ull;
        vn[k] = 0;
    }
    int blo = 0;
    int next_shift = g.slide ? g.dmax + 65 : 0x7fffffff;
    // words of the next block to enter the window, loaded one slide ahead
    uint32_t qn[4] = {0, 0, 0, 0};
    if (g.slide && P < nb) load_block_words(qb, P, qn);
    uint32_t tw = 0;
    uint32_t tw_next = n > 0 ? __ldg(tb) : 0u;
    uint8_t* r = rec + lane * (16 * kLaneColGroup);   // current column group of this lane
    for (int j = 1; j <= g.n_max; ++j) {
        if (j == next_shift) {  // warp-uniform: drop the top block, a new block enters
#pragma unroll
            for (int k = 0; k + 1 < P; ++k) {
                vp[k] = vp[k + 1];
                vn[k] = vn[k + 1];
#pragma unroll
                for (int c = 0; c < 4; ++c) sp[(k * 4 + c) * 32 + lane] = sp[((k + 1) * 4 + c) * 32 + lane];
            }
            vp[P - 1] = ~0ull;
            vn[P - 1] = 0;
            ++blo;
            const int b = blo + P - 1;
            uint64_t e[4] = {0, 0, 0, 0};
            if (b < nb) peq_words(qn, e);
            if (b + 1 < nb) load_block_words(qb, b + 1, qn);
#pragma unroll
            for (int c = 0; c < 4; ++c) sp[((P - 1) * 4 + c) * 32 + lane] = e[c];
            next_shift += 64;
        }
        const int jj = j - 1;
        if ((jj & 15) == 0) {
            tw = tw_next;
            const int nw = (jj >> 4) + 1;
            tw_next = nw * 16 < n ? __ldg(tb + nw) : 0u;
        }
        const uint32_t c = (tw >> ((jj & 15) * 2)) & 3u;
        const uint64_t* eqp = sp + c * 32 + lane;
        const int sub = jj % kLaneColGroup;
        uint32_t pa = 0, ma = 0;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const uint64_t eq = eqp[k * 128];
            const uint64_t ph = k == 0 ? advance_block<true>(vp[0], vn[0], eq, pa, ma)
                                       : advance_block<false>(vp[k], vn[k], eq, pa, ma);
            *reinterpret_cast<uint4*>(r + k * (512 * kLaneColGroup) + sub * 16) =
                make_uint4(lo32(vp[k]), hi32(vp[k]), lo32(ph), hi32(ph));
        }
        if (sub == kLaneColGroup - 1) r += P * (512 * kLaneColGroup);
    }
}

// Traceback of one lane's pair from (m, n). The walk moves column by column: a column's
// record holds the VP / HP bits of 64 rows, so D runs stay in one record and I or
// diagonal moves step to the next column. Records of kTraceCols columns (current
// block) are fetched together into the lane's shared-memory slots, so one memory
// latency covers up to kTraceCols columns. Returns false when the walk left the band
// or cost more than E (the pair is then redone).
template <int P>
__device__ __forceinline__ bool lane_trace(const uint32_t* __restrict__ qb, const uint32_t* __restrict__ tb, int m,
                                           int n, const LaneBand& band, const LaneGeom& g, bool act,
                                           const uint8_t* rec, uint4* srec, RunWriter& rw, int* ed_out) {
    const int lane = lane_id();
    int i = act ? m : 0, j = act ? n : 0, cost = 0;
    bool ok = act;
    int j0 = -1, bwin = -1;          // window: columns (j0 - kTraceCols, j0] of block bwin
    uint32_t valid = 0;              // bit t: record of column j0 - t is inside the window
    uint32_t twin = 0;               // target symbols [tbase, tbase + 16)
    int tbase = 0;
    uint64_t qwin = 0;               // query symbols [qbase, qbase + 32)
    int qbase = 0x7fffffff;
    for (;;) {
        const bool want = ok && i > 0 && j > 0;
        if (!__any_sync(PHR_FULL_MASK, want)) break;
        if (!want) continue;
        const int b = (i - 1) >> 6;
        if (j0 < 0 || j <= j0 - kTraceCols || b != bwin) {
            j0 = j;
            bwin = b;
            valid = 0;
            // asynchronous global -> shared copies: all columns in flight at once, no registers
#pragma unroll
            for (int t = 0; t < kTraceCols; ++t) {
                const int jt = j - t;
                if (jt > 0) {
                    const int k = b - lane_blo(g, jt);
                    if (k >= 0 && k < P) {
                        const uint8_t* src = rec + rec_off<P>(jt - 1, k, lane);
                        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(srec + t * 32));
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
                        valid |= 1u << t;
                    }
                }
            }
            asm volatile("cp.async.wait_all;\n" ::: "memory");
            tbase = j > 16 ? j - 16 : 0;
            twin = load_window<Seq2>(tb, tbase);
        }
        const int t = j0 - j;
        if (!((valid >> t) & 1u)) {
            ok = false;
            continue;
        }
        const uint4 R = srec[t * 32];
        const uint64_t vp = mk64(R.x, R.y), hp = mk64(R.z, R.w);
        const int bit = (i - 1) & 63;
        if ((vp >> bit) & 1ull) {
            // D run: consecutive VP bits upward from row i within this block
            const int run = __clzll(~(vp << (63 - bit)));
            rw.push(3, static_cast<uint32_t>(run));
            i -= run;
            cost += run;
        } else if ((hp >> bit) & 1ull) {
            rw.push(2, 1);
            j -= 1;
            cost += 1;
        } else {
            // diagonal stretch: cells (i-u, j-u) of this window and block, u < L
            const int L = min(min(kTraceCols - t, bit + 1), min(i, j));
            uint32_t stop = 0;
#pragma unroll
            for (int u = 1; u < kTraceCols; ++u) {
                if (u < L) {
                    const uint4 Q = srec[(t + u) * 32];
                    const uint64_t sv = mk64(Q.x | Q.z, Q.y | Q.w);
                    stop |= static_cast<uint32_t>((sv >> (bit - u)) & 1ull) << u;
                }
            }
            stop |= ~(valid >> t);            // a cell without a record ends the stretch
            stop |= ~0u << L;                 // L < 32
            const int run = __ffs(stop) - 1;  // diagonal moves (>= 1: cell u = 0 is one)
            // M / X per cell: query symbols i-16 .. i-1 against target symbols j-16 .. j-1
            if ((i > 16 ? i - 16 : 0) < qbase || i - 1 >= qbase + 32) {
                qbase = i > 32 ? i - 32 : 0;
                qwin = mk64(load_window<Seq2>(qb, qbase), load_window<Seq2>(qb, qbase + 16));
            }
            const int sq = 2 * (i - 16 - qbase), st = 2 * (j - 16 - tbase);
            const uint32_t qa = static_cast<uint32_t>(sq >= 0 ? (qwin >> sq) : (qwin << -sq));
            const uint32_t ta = st >= 0 ? (twin >> st) : (twin << -st);
            const uint32_t x = qa ^ ta;
            // symbol k of the aligned words is cell u = 15 - k; bit 2k of nz -> bit 2u+1 reversed
            const uint32_t nz = (x | (x >> 1)) & 0x55555555u;
            const uint32_t neq = even_bits(__brev(nz) >> 1);
            int u = 0;
            while (u < run) {
                const uint32_t cur = (neq >> u) & 1u;
                const uint32_t y = (cur ? ~neq : neq) >> u;
                int len = y ? __ffs(y) - 1 : 32 - u;
                len = min(len, run - u);
                rw.push(cur, static_cast<uint32_t>(len));
                if (cur) cost += len;
                u += len;
            }
            i -= run;
            j -= run;
        }
        const int d = j - i;
        if (d < band.dmin || d > band.dmax || cost > band.E) ok = false;
    }
    if (ok) {
        if (i > 0) {
            rw.push(3, static_cast<uint32_t>(i));
            cost += i;
        }
        if (j > 0) {
            rw.push(2, static_cast<uint32_t>(j));
            cost += j;
        }
        rw.flush();
        if (cost > band.E || rw.overflow) ok = false;
    }
    *ed_out = cost;
    return ok;
}

template <int P>
__device__ void lane_task(const ExtendParams& Pm, uint32_t pid, const PairDesc& d, bool act, const LaneBand& band,
                          const LaneGeom& g, uint64_t* sp, uint8_t* slot) {
    const int lane = lane_id();
    const int m = act ? d.qn : 0, n = act ? d.tn : 0;
    const int nb = (m + 63) >> 6;
    const uint32_t* qb = Pm.packed2 + (act ? d.q_word : 0);
    const uint32_t* tb = Pm.packed2 + (act ? d.t_word : 0);
    lane_forward<P>(qb, tb, n, nb, g, sp, slot);
    __syncwarp();  // the traceback reuses the Peq shared memory
    const uint64_t ng = static_cast<uint64_t>((g.n_max + kLaneColGroup - 1) / kLaneColGroup);
    const uint64_t rec_bytes = (ng * kLaneColGroup * P * 512 + 255) & ~255ull;
    const uint32_t cap = static_cast<uint32_t>(g.m_max + g.n_max + 2);
    uint32_t* runs = reinterpret_cast<uint32_t*>(slot + rec_bytes) + static_cast<uint64_t>(lane) * cap;
    RunWriter rw;
    rw.init(runs, static_cast<uint32_t>(m + n + 2), true);
    int ed = 0;
    const bool ok = lane_trace<P>(qb, tb, m, n, band, g, act, slot, reinterpret_cast<uint4*>(sp) + lane, rw, &ed);
    // work counters: block-columns this task evaluated for its pairs, pairs sent to redo
    const unsigned long long cols = __reduce_add_sync(PHR_FULL_MASK, act ? static_cast<unsigned>(n) * P : 0u);
    const unsigned redo = __popc(__ballot_sync(PHR_FULL_MASK, act && !ok));
    if (lane == 0) {
        atomicAdd(Pm.work, cols);
        if (redo) atomicAdd(Pm.work + 1, static_cast<unsigned long long>(redo));
    }
    if (act && !ok) {
        const uint32_t k = atomicAdd(Pm.redo_count, 1u);
        Pm.redo_list[k] = pid;
        const uint64_t need = myers_full_need(m, n);
        atomicMax(Pm.redo_need_max, static_cast<unsigned long long>(need));
        if (Pm.redo_need) Pm.redo_need[k] = need;
    }
    if (act && ok) {
        char* out = Pm.text + Pm.text_off[pid];
        uint32_t tl = 0;
        for (int r = static_cast<int>(rw.n) - 1; r >= 0; --r) {
            const uint32_t run = runs[r];
            uint32_t v = run >> 2;
            const uint32_t nd = ndigits(v);
            for (int dd = static_cast<int>(nd) - 1; dd >= 0; --dd) {
                out[tl + dd] = static_cast<char>('0' + v % 10);
                v /= 10;
            }
            out[tl + nd] = op_char(run & 3u);
            tl += nd + 1;
        }
        PairOut o;
        o.status = PHR_OK;
        o.ed = ed;
        o.t_consumed = n;
        o.affine_score = 0;
        o.n_runs = rw.n;
        o.text_len = tl;
        Pm.out[pid] = o;
    }
}

__global__ void __launch_bounds__(kLaneThreads, 2) myers_lane_kernel(ExtendParams Pm) {
    extern __shared__ uint64_t lane_smem[];
    const int lane = lane_id();
    const int wib = threadIdx.x >> 5;
    uint64_t* sp = lane_smem + static_cast<uint64_t>(wib) * kLaneMaxSlots * 4 * 32;
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    uint8_t* slot = Pm.scratch + warp_global * Pm.slot_bytes;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = Pm.tasks.range[0] + atomicAdd(Pm.queue_head, 1u);
        task = __shfl_sync(PHR_FULL_MASK, task, 0);
        if (task >= Pm.tasks.range[1]) break;
        const int count = Pm.tasks.task_count[task];
        const bool act = lane < count;
        const uint32_t pid = act ? Pm.tasks.order[Pm.tasks.task_first[task] + lane] : 0;
        PairDesc d = {};
        if (act) d = Pm.desc[pid];
        const int m = act ? d.qn : 0, n = act ? d.tn : 0;
        const LaneBand band = lane_band(m, n, Pm.band_base);
        LaneGeom g;
        g.dmin = __reduce_min_sync(PHR_FULL_MASK, act ? band.dmin : 0x7fffffff);
        g.dmax = __reduce_max_sync(PHR_FULL_MASK, act ? band.dmax : static_cast<int>(0x80000000));
        g.n_max = __reduce_max_sync(PHR_FULL_MASK, static_cast<unsigned>(n));
        g.m_max = __reduce_max_sync(PHR_FULL_MASK, static_cast<unsigned>(m));
        g.nb_max = (g.m_max + 63) >> 6;
        g.P = lane_slots(g.dmin, g.dmax, g.nb_max);
        g.slide = g.P < g.nb_max;
        const uint64_t need = lane_task_need(g.n_max, g.m_max, g.P);
        if (g.P > kLaneMaxSlots || need > Pm.slot_bytes) {
            if (lane == 0) atomicAdd(Pm.work + 1, static_cast<unsigned long long>(count));
            if (act) {
                const uint32_t k = atomicAdd(Pm.redo_count, 1u);
                Pm.redo_list[k] = pid;
                const uint64_t nf = myers_full_need(m, n);
                atomicMax(Pm.redo_need_max, static_cast<unsigned long long>(nf));
                if (Pm.redo_need) Pm.redo_need[k] = nf;
            }
            continue;
        }
        switch (g.P) {
            case 1: lane_task<1>(Pm, pid, d, act, band, g, sp, slot); break;
            case 2: lane_task<2>(Pm, pid, d, act, band, g, sp, slot); break;
            case 3: lane_task<3>(Pm, pid, d, act, band, g, sp, slot); break;
            case 4: lane_task<4>(Pm, pid, d, act, band, g, sp, slot); break;
            case 5: lane_task<5>(Pm, pid, d, act, band, g, sp, slot); break;
            case 6: lane_task<6>(Pm, pid, d, act, band, g, sp, slot); break;
            case 7: lane_task<7>(Pm, pid, d, act, band, g, sp, slot); break;
            default: lane_task<8>(Pm, pid, d, act, band, g, sp, slot); break;
        }
        __syncwarp();
    }
}

}  // namespace

void launch_myers_lane(const ExtendParams& p, int grid, cudaStream_t st) {
    const size_t smem = static_cast<size_t>(kLaneWarps) * kLaneMaxSlots * 4 * 32 * sizeof(uint64_t);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(myers_lane_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        configured = true;
    }
    myers_lane_kernel<<<grid, kLaneThreads, smem, st>>>(p);
}

}  // namespace phr
