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
constexpr int kTraceBatch = 8;  // diagonal cells whose records one traceback fetch loads
static_assert(2 * kTraceBatch * 32 * 16 <= kLaneMaxSlots * 4 * 32 * 8, "traceback slots exceed the Peq area");

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

// Byte offset of the {VP, VN} state of slot k after column (c + 1) * kSegCols.
template <int P>
__device__ __forceinline__ uint64_t ck_off(int c, int k, int lane) {
    return ((static_cast<uint64_t>(c) * P + k) * 32 + lane) * 16;
}

// Forward pass of one lane's pair. CK = false: every column's {VP, HP} records go to
// `rec`; CK = true: only the window's {VP, VN} after every kSegCols-th column below
// n_max (the traceback recomputes the columns in between).
template <int P, bool CK>
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
    // 2-bit target symbol of column index jj (called for jj = 0, 1, 2, ... in order)
    auto next_sym = [&](int jj) -> uint32_t {
        if ((jj & 15) == 0) {
            tw = tw_next;
            const int nw = (jj >> 4) + 1;
            tw_next = nw * 16 < n ? __ldg(tb + nw) : 0u;
        }
        return (tw >> ((jj & 15) * 2)) & 3u;
    };
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
        const uint32_t c = next_sym(jj);
        const uint64_t* eqp = sp + c * 32 + lane;
        const int sub = jj % kLaneColGroup;
        uint32_t pa = 0, ma = 0;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const uint64_t eq = eqp[k * 128];
            const uint64_t ph = k == 0 ? advance_block<true>(vp[0], vn[0], eq, pa, ma)
                                       : advance_block<false>(vp[k], vn[k], eq, pa, ma);
            if (!CK)
                *reinterpret_cast<uint4*>(r + k * (512 * kLaneColGroup) + sub * 16) =
                    make_uint4(lo32(vp[k]), hi32(vp[k]), lo32(ph), hi32(ph));
        }
        if (!CK && sub == kLaneColGroup - 1) r += P * (512 * kLaneColGroup);
        if (CK && (j % kSegCols) == 0 && j < g.n_max) {  // warp-uniform
            uint8_t* c = rec + ck_off<P>(j / kSegCols - 1, 0, lane);
#pragma unroll
            for (int k = 0; k < P; ++k)
                *reinterpret_cast<uint4*>(c + k * 512) = make_uint4(lo32(vp[k]), hi32(vp[k]), lo32(vn[k]), hi32(vn[k]));
        }
    }
}

// Issues asynchronous global -> shared copies of the records of the kTraceBatch cells
// (ci - t, cj - t), t < kTraceBatch, of one diagonal, each from its own block, into
// buf[t * 32] (one cp.async group). Returns the mask of cells whose record lies in the
// window (others are left unloaded).
template <int P>
__device__ __forceinline__ uint32_t fetch_diagonal(const uint8_t* rec, const LaneGeom& g, int ci, int cj, uint4* buf) {
    const int lane = lane_id();
    uint32_t valid = 0;
#pragma unroll
    for (int t = 0; t < kTraceBatch; ++t) {
        const int it = ci - t, jt = cj - t;
        if (it > 0 && jt > 0) {
            const int k = ((it - 1) >> 6) - lane_blo(g, jt);
            if (k >= 0 && k < P) {
                const uint8_t* src = rec + rec_off<P>(jt - 1, k, lane);
                const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(buf + t * 32));
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
                valid |= 1u << t;
            }
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    return valid;
}

// 2-bit symbols [pos - 8, pos + 8) of a sequence shifted so that symbol pos - 1 - t sits
// at index 7 - t (t < 8) also when pos < 8 (lower indices then hold zeros).
__device__ __forceinline__ uint32_t diag_window(const uint32_t* __restrict__ s, int pos) {
    const int p0 = pos > 8 ? pos - 8 : 0;
    return load_window<Seq2>(s, p0) << (2 * (8 - (pos - p0)));
}

// Traceback of one lane's pair from (m, n). The records the walk needs lie along
// diagonals between indels, so they are fetched kTraceBatch cells of the current
// diagonal at a time, each cell's record from its own block, and the next batch of the
// same diagonal is prefetched while this one is processed (two shared-memory buffers
// per lane). A D run is read off one record; an I move, or a D run, starts a new
// diagonal. Returns false when the walk left the band or cost more than E (the pair is
// then redone).
template <int P>
__device__ __forceinline__ bool lane_trace(const uint32_t* __restrict__ qb, const uint32_t* __restrict__ tb, int m,
                                           int n, const LaneBand& band, const LaneGeom& g, bool act,
                                           const uint8_t* rec, uint4* srec, RunWriter& rw, int* ed_out) {
    int i = act ? m : 0, j = act ? n : 0, cost = 0;
    bool ok = act;
    uint4* bufA = srec;                      // batch starting at cell (ai, aj)
    uint4* bufB = srec + kTraceBatch * 32;   // the next batch of the same diagonal
    int ai = -1, aj = -1;
    uint32_t va = 0, vb = 0;                 // loaded-cell masks
    uint32_t xa = 0, xb = 0;                 // query XOR target symbols: cell t at index 7 - t
    for (;;) {
        const bool want = ok && i > 0 && j > 0;
        if (!__any_sync(PHR_FULL_MASK, want)) break;
        if (!want) continue;
        int t = ai - i;
        if (!(ai >= 0 && ai - i == aj - j && t >= 0 && t < kTraceBatch)) {
            if (ai >= 0 && ai - i == aj - j && t >= kTraceBatch && t < 2 * kTraceBatch) {
                // the walk went on along the diagonal into the prefetched batch
                uint4* x = bufA;
                bufA = bufB;
                bufB = x;
                ai -= kTraceBatch;
                aj -= kTraceBatch;
                va = vb;
                xa = xb;
                asm volatile("cp.async.wait_all;\n" ::: "memory");
            } else {
                // a new diagonal: this batch and the next
                ai = i;
                aj = j;
                va = fetch_diagonal<P>(rec, g, ai, aj, bufA);
                xa = diag_window(qb, ai) ^ diag_window(tb, aj);
                asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            }
            vb = fetch_diagonal<P>(rec, g, ai - kTraceBatch, aj - kTraceBatch, bufB);
            xb = (ai - kTraceBatch > 0 && aj - kTraceBatch > 0)
                     ? diag_window(qb, ai - kTraceBatch) ^ diag_window(tb, aj - kTraceBatch)
                     : 0u;
            t = ai - i;
        }
        if (!((va >> t) & 1u)) {
            ok = false;
            continue;
        }
        const uint4 R = bufA[t * 32];
        const uint64_t vp = mk64(R.x, R.y), hp = mk64(R.z, R.w);
        const int bit = (i - 1) & 63;
        if ((vp >> bit) & 1ull) {
            // D run: consecutive VP bits upward from row i within this record's block
            const int run = __clzll(~(vp << (63 - bit)));
            rw.push(3, static_cast<uint32_t>(run));
            i -= run;
            cost += run;
        } else if ((hp >> bit) & 1ull) {
            rw.push(2, 1);
            j -= 1;
            cost += 1;
        } else {
            // diagonal stretch over the cells t + u of this batch: stop at the first cell
            // with a VP or HP bit, without a record, or past the batch
            const int L = min(kTraceBatch - t, min(i, j));
            uint32_t stop = 0;
#pragma unroll
            for (int u = 1; u < kTraceBatch; ++u) {
                if (u < L) {
                    const uint4 Q = bufA[(t + u) * 32];
                    const uint64_t sv = mk64(Q.x | Q.z, Q.y | Q.w);
                    stop |= static_cast<uint32_t>((sv >> ((i - 1 - u) & 63)) & 1ull) << u;
                }
            }
            stop |= ~(va >> t);
            stop |= ~0u << L;
            const int run = __ffs(stop) - 1;  // >= 1: cell u = 0 is diagonal
            // M / X: cell t + u compares symbol index 7 - (t + u) of the batch's windows
            const uint32_t nz = (xa | (xa >> 1)) & 0x55555555u;
            const uint32_t neq = even_bits(__brev(nz) >> 17) >> t;   // bit u: cell t + u differs
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
    asm volatile("cp.async.wait_all;\n" ::: "memory");
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

// Shared memory of one warp in checkpoint mode: the Peq ring (kLaneMaxSlots + 1 blocks,
// [block % (P + 1)][base][lane], 64-bit masks). The forward pass's Peq ([slot][base]
// [lane]) reuses its start. The segment's records live in the warp's scratch slot: each
// lane writes and reads back only its own, a few KB per warp that stay in L1/L2, and
// shared memory stays small enough for two blocks per SM.
constexpr int kRingBytes = (kLaneMaxSlots + 1) * 4 * 32 * 8;
constexpr int kCkWarpBytes = kRingBytes;

// Peq of query block b (zero past the query) into ring slot b % (P + 1).
template <int P>
__device__ __forceinline__ void ring_fill(uint64_t* ring, const uint32_t* __restrict__ qb, int b, int nb, int lane) {
    uint64_t e[4] = {0, 0, 0, 0};
    if (b < nb) {
        uint32_t qw[4];
        load_block_words(qb, b, qw);
        peq_words(qw, e);
    }
    uint64_t* r = ring + (b % (P + 1)) * 128 + lane;
#pragma unroll
    for (int c = 0; c < 4; ++c) r[c * 32] = e[c];
}

// Traceback of one lane's pair from (m, n) over segments of kSegCols columns, top
// segment first. For each segment the warp recomputes its columns from the forward
// pass's checkpoint (the same window, shifts and block updates, so the same bits), keeps
// their {VP, HP} records in shared memory, and every lane whose walk is inside the
// segment moves through it one event at a time (D run, I move or diagonal cell, with
// the precedence of myers_backtrace_flat) until it leaves the segment's columns. Returns
// false when the walk left the band or cost more than E (the pair is then redone).
template <int P>
__device__ __forceinline__ bool lane_trace_ck(const uint32_t* __restrict__ qb, const uint32_t* __restrict__ tb,
                                              int m, int n, int nb, const LaneBand& band, const LaneGeom& g, bool act,
                                              uint8_t* ck, uint8_t* smem, RunWriter& rw, int* ed_out) {
    const int lane = lane_id();
    uint64_t* ring = reinterpret_cast<uint64_t*>(smem);
    uint4* seg = reinterpret_cast<uint4*>(ck + lane_ckpt_bytes(g.n_max, P));
    int i = act ? m : 0, j = act ? n : 0, cost = 0;
    bool ok = act;
    int q_idx = -1;       // query word held in q_word (the walk's row moves slowly)
    uint32_t q_word = 0;
    if (g.n_max > 0) {
        const int S = (g.n_max - 1) / kSegCols;
        int ring_lo = lane_blo(g, S * kSegCols);  // the ring holds blocks [ring_lo, ring_lo + P]
#pragma unroll
        for (int k = 0; k <= P; ++k) ring_fill<P>(ring, qb, ring_lo + k, nb, lane);
        for (int sgi = S; sgi >= 0; --sgi) {
            const int j0 = sgi * kSegCols;
            const int blo0 = lane_blo(g, j0);
            if (blo0 < ring_lo) {  // one block enters the ring at the top (in the slot of ring_lo + P)
                ring_lo = blo0;
                ring_fill<P>(ring, qb, ring_lo, nb, lane);
            }
            // ---- recompute columns j0 + 1 .. min(j0 + kSegCols, n_max) ----
            uint64_t vp[P], vn[P];
            if (sgi == 0) {
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    vp[k] = ~0ull;
                    vn[k] = 0;
                }
            } else {
                const uint8_t* c = ck + ck_off<P>(sgi - 1, 0, lane);
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    const uint4 x = *reinterpret_cast<const uint4*>(c + k * 512);
                    vp[k] = mk64(x.x, x.y);
                    vn[k] = mk64(x.z, x.w);
                }
            }
            int blo = blo0;
            const int jend = min(j0 + kSegCols, g.n_max);
            // target symbols j0 .. j0 + kSegCols - 1 share one 16-symbol word (kSegCols divides 16)
            const int wj = j0 >> 4;
            const uint32_t tw = wj * 16 < n ? __ldg(tb + wj) : 0u;
            // (each lane reads back only the records it wrote: no barrier is needed)
            for (int jj = j0 + 1; jj <= jend; ++jj) {  // warp-uniform
                if (g.slide && lane_blo(g, jj) > blo) {  // the window moves down one block
#pragma unroll
                    for (int k = 0; k + 1 < P; ++k) {
                        vp[k] = vp[k + 1];
                        vn[k] = vn[k + 1];
                    }
                    vp[P - 1] = ~0ull;
                    vn[P - 1] = 0;
                    ++blo;
                }
                const uint32_t c = (tw >> (((jj - 1) & 15) * 2)) & 3u;
                uint4* out = seg + (jj - j0 - 1) * (P * 32) + lane;
                uint32_t pa = 0, ma = 0;
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    int rs = (blo + k) % (P + 1);
                    const uint64_t eq = ring[(rs * 4 + c) * 32 + lane];
                    const uint64_t ph = k == 0 ? advance_block<true>(vp[0], vn[0], eq, pa, ma)
                                               : advance_block<false>(vp[k], vn[k], eq, pa, ma);
                    out[k * 32] = make_uint4(lo32(vp[k]), hi32(vp[k]), lo32(ph), hi32(ph));
                }
            }
            __syncwarp();
            // ---- walk every lane through this segment's columns ----
            for (;;) {
                const bool want = ok && i > 0 && j > j0;
                if (!__any_sync(PHR_FULL_MASK, want)) break;
                if (!want) continue;
                const int kb = ((i - 1) >> 6) - lane_blo(g, j);
                if (kb < 0 || kb >= P) {
                    ok = false;
                    continue;
                }
                const uint4 R = seg[((j - j0 - 1) * P + kb) * 32 + lane];
                const uint64_t vpb = mk64(R.x, R.y), hpb = mk64(R.z, R.w);
                const int bit = (i - 1) & 63;
                if ((vpb >> bit) & 1ull) {
                    // D run: consecutive VP bits upward from row i within this block
                    const int run = __clzll(~(vpb << (63 - bit)));
                    rw.push(3, static_cast<uint32_t>(run));
                    i -= run;
                    cost += run;
                } else if ((hpb >> bit) & 1ull) {
                    rw.push(2, 1);
                    j -= 1;
                    cost += 1;
                } else {
                    // target symbol j - 1 from the segment's word; query word cached
                    const int qwi = (i - 1) >> 4;
                    if (qwi != q_idx) {
                        q_idx = qwi;
                        q_word = __ldg(qb + qwi);
                    }
                    const uint32_t qs = (q_word >> (((i - 1) & 15) * 2)) & 3u;
                    const uint32_t ts = (tw >> (((j - 1) & 15) * 2)) & 3u;
                    const uint32_t x = qs != ts ? 1u : 0u;
                    rw.push(x, 1);
                    cost += static_cast<int>(x);
                    i -= 1;
                    j -= 1;
                }
                const int d = j - i;
                if (d < band.dmin || d > band.dmax || cost > band.E) ok = false;
            }
        }
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

// Forward pass and traceback of one task in one warp; records in the warp's slot. (A
// separate traceback kernel with more resident warps measured slower on B200: the 32
// lanes' walks diverge, so a traceback warp executes about as many instructions as the
// forward pass whatever hides its latency.)
template <int P, bool CK>
__device__ void lane_task(const ExtendParams& Pm, uint32_t pid, const PairDesc& d, bool act, const LaneBand& band,
                          const LaneGeom& g, uint64_t* sp, uint8_t* slot) {
    const int lane = lane_id();
    const int m = act ? d.qn : 0, n = act ? d.tn : 0;
    const int nb = (m + 63) >> 6;
    const uint32_t* qb = Pm.packed2 + (act ? d.q_word : 0);
    const uint32_t* tb = Pm.packed2 + (act ? d.t_word : 0);
    lane_forward<P, CK>(qb, tb, n, nb, g, sp, slot);
    // work counter: block-columns this task evaluated for its pairs
    const unsigned long long cols = __reduce_add_sync(PHR_FULL_MASK, act ? static_cast<unsigned>(n) * P : 0u);
    if (lane == 0) atomicAdd(Pm.work, cols);
    __syncwarp();  // the traceback reuses the Peq shared memory
    const uint64_t rec_bytes = lane_rec_bytes(g.n_max, P, CK ? 1 : 0);
    const uint32_t cap = static_cast<uint32_t>(g.m_max + g.n_max + 2);
    uint32_t* runs = reinterpret_cast<uint32_t*>(slot + rec_bytes) + static_cast<uint64_t>(lane) * cap;
    RunWriter rw;
    rw.init(runs, static_cast<uint32_t>(m + n + 2), true);
    int ed = 0;
    bool ok;
    if (CK)
        ok = lane_trace_ck<P>(qb, tb, m, n, nb, band, g, act, slot, reinterpret_cast<uint8_t*>(sp), rw, &ed);
    else
        ok = lane_trace<P>(qb, tb, m, n, band, g, act, slot, reinterpret_cast<uint4*>(sp) + lane, rw, &ed);
    // work counter: pairs sent to redo
    const unsigned redo = __popc(__ballot_sync(PHR_FULL_MASK, act && !ok));
    if (lane == 0 && redo) atomicAdd(Pm.work + 1, static_cast<unsigned long long>(redo));
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

template <bool CK>
__device__ __forceinline__ void lane_tasks(const ExtendParams& Pm, uint64_t* sp) {
    const int lane = lane_id();
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = Pm.tasks.range[0] + atomicAdd(Pm.queue_head, 1u);
        task = __shfl_sync(PHR_FULL_MASK, task, 0);
        if (task >= Pm.tasks.range[1]) break;
        uint8_t* slot = Pm.scratch + warp_global * Pm.slot_bytes;
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
        const uint64_t need = lane_task_need(g.n_max, g.m_max, g.P, CK ? 1 : 0);
        // a task beyond the kernel's window or its warp slot is redone by the every-block kernel
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
            case 1: lane_task<1, CK>(Pm, pid, d, act, band, g, sp, slot); break;
            case 2: lane_task<2, CK>(Pm, pid, d, act, band, g, sp, slot); break;
            case 3: lane_task<3, CK>(Pm, pid, d, act, band, g, sp, slot); break;
            case 4: lane_task<4, CK>(Pm, pid, d, act, band, g, sp, slot); break;
            case 5: lane_task<5, CK>(Pm, pid, d, act, band, g, sp, slot); break;
            case 6: lane_task<6, CK>(Pm, pid, d, act, band, g, sp, slot); break;
            case 7: lane_task<7, CK>(Pm, pid, d, act, band, g, sp, slot); break;
            default: lane_task<8, CK>(Pm, pid, d, act, band, g, sp, slot); break;
        }
        __syncwarp();
    }
}

constexpr int kLanePeqWarpBytes = kLaneMaxSlots * 4 * 32 * 8;  // Peq (and traceback buffers) per warp
static_assert(kLanePeqWarpBytes <= kCkWarpBytes, "the forward pass's Peq must fit the checkpoint-mode area");

__global__ void __launch_bounds__(kLaneThreads, 2) myers_lane_kernel(ExtendParams Pm) {
    extern __shared__ uint64_t lane_smem[];
    lane_tasks<false>(Pm, lane_smem + static_cast<uint64_t>(threadIdx.x >> 5) * (kLanePeqWarpBytes / 8));
}

// Checkpoint mode: kCkWarpBytes of shared memory per warp, two blocks per SM.
__global__ void __launch_bounds__(kLaneThreads, 2) myers_lane_ck_kernel(ExtendParams Pm) {
    extern __shared__ uint64_t lane_smem[];
    lane_tasks<true>(Pm, lane_smem + static_cast<uint64_t>(threadIdx.x >> 5) * (kCkWarpBytes / 8));
}

}  // namespace

int myers_lane_blocks_per_sm(int) { return 2; }

void launch_myers_lane(const ExtendParams& p, int grid, cudaStream_t st) {
    if (p.lane_ckpt) {
        const int smem = kLaneWarps * kCkWarpBytes;
        cudaFuncSetAttribute(myers_lane_ck_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        myers_lane_ck_kernel<<<grid, kLaneThreads, smem, st>>>(p);
        return;
    }
    const int smem = kLaneWarps * kLanePeqWarpBytes;
    cudaFuncSetAttribute(myers_lane_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    myers_lane_kernel<<<grid, kLaneThreads, smem, st>>>(p);
}

}  // namespace phr
