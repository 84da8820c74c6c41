// pipeline.cu -- align_read on the device: sketch -> seed -> chain -> anchor gating ->
// extension (engine.cu) -> score/select, plus the target index (TargetContext).
//
// Semantics restated from phraya-align:
//   seeding   build_minimizer_index seeding.rs:31-37, find_seeds_indexed_capped :58-80,
//             seed_occurrence_cap :94-102
//   chaining  chain_score chaining.rs:96-117, chain_seeds :134-226, Chain::target_start :32-35
//   executor  align_read executor.rs:573-733, extend_chains :528-567, anchors_from_chains
//             :347-362, chain_cap :330-336, extend_anchor :379-404, MYERS_MAX_QUERY_LEN :248
//   scoring   score_alignments lib.rs:170-199
//   types     reverse_complement phraya-core/src/types.rs:91-107
// The sketcher restates simd-minimizers 2.3.1's random minimizers
// (phraya-core/src/types.rs:1848-1869; the crate's source is not in the reference tree)
// from their published description: characters as packed-seq's AsciiSeq 2-bit codes
// ((b >> 1) & 3), 32-bit ntHash order hashes (canonical: min of forward and reverse
// complement), w-k-mer windows with the leftmost minimum, or for canonical minimizers
// the rightmost one in windows with more A/C than T/G, each selected k-mer emitted once
// per run of windows; pairs are (2-bit k-mer value, canonical min for DNA; position).
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pipeline.cuh"

namespace phr {

__constant__ int32_t c_chain_pen[101];

namespace {

inline unsigned blocks_for(uint64_t n, unsigned t) { return static_cast<unsigned>((n + t - 1) / t); }

// ntHash base seeds (Mohamadi et al. 2016), low 32 bits, indexed by the 2-bit code
// A = 0, C = 1, T = 2, G = 3 (the complement of code c is c ^ 2).
__constant__ uint32_t c_nt_seed[4] = {0x95c60474u, 0x62a02b4cu, 0x4be24456u, 0x82572324u};

// ---------------------------------------------------------------------------
// Sketching
// ---------------------------------------------------------------------------
struct SketchArgs {
    const uint8_t* seq;
    const uint64_t* off;
    const uint32_t* len;
    uint64_t n;
    const uint64_t* kbase;   // exclusive scan of k-mer counts, n+1 entries
    const uint64_t* wbase;   // exclusive scan of window counts, n+1 entries
    uint64_t total_k, total_w;
    int k, w, alphabet;
    uint64_t* key;
    uint32_t* flag;
    uint32_t* sel;
};

__device__ __forceinline__ uint64_t find_seq(const uint64_t* base, uint64_t n, uint64_t g) {
    uint64_t lo = 0, hi = n;  // largest s with base[s] <= g
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) / 2;
        if (base[mid] <= g) lo = mid; else hi = mid;
    }
    return lo;
}

constexpr int kSketchRun = 8;  // consecutive k-mer positions (windows) per thread, rolled

__device__ __forceinline__ uint32_t nt_seed(uint32_t c) {
    return c < 2u ? (c ? c_nt_seed[1] : c_nt_seed[0]) : (c == 2u ? c_nt_seed[2] : c_nt_seed[3]);
}
__device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) { return __funnelshift_l(x, x, r & 31); }

// Order hash of every k-mer: 32-bit ntHash over 2-bit codes, canonical = min(forward,
// reverse complement) for DNA, forward for protein. A thread takes kSketchRun consecutive
// positions: the first of a sequence is hashed whole, the next ones rolled,
//   f(p + 1) = rotl(f(p), 1) ^ rotl(seed[c_p], k) ^ seed[c_{p+k}]
//   r(p + 1) = rotr(r(p) ^ seed[~c_p], 1) ^ rotl(seed[~c_{p+k}], k - 1)
// (XOR and rotations are exact, so the rolled hash equals the direct one). The four
// seeds are picked by selects from uniform constant reads: an index per lane would
// serialise the constant cache.
__global__ void sketch_key_kernel(SketchArgs A) {
    const uint64_t runs = (A.total_k + kSketchRun - 1) / kSketchRun;
    const int k = A.k;
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < runs;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t g0 = r * kSketchRun;
        const uint64_t g1 = g0 + kSketchRun < A.total_k ? g0 + kSketchRun : A.total_k;
        uint64_t s = find_seq(A.kbase, A.n, g0);
        uint64_t s_end = A.kbase[s + 1];
        uint32_t hf = 0, hr = 0;
        bool fresh = true;
        for (uint64_t g = g0; g < g1; ++g) {
            while (g >= s_end) {  // next sequence (skipping those shorter than k)
                ++s;
                s_end = A.kbase[s + 1];
                fresh = true;
            }
            const uint8_t* b = A.seq + A.off[s] + (g - A.kbase[s]);
            if (fresh) {
                hf = hr = 0;
                for (int i = 0; i < k; ++i) {
                    const uint32_t c = (b[i] >> 1) & 3u;
                    hf ^= rotl32(nt_seed(c), k - 1 - i);
                    hr ^= rotl32(nt_seed(c ^ 2u), i);
                }
                fresh = false;
            } else {
                const uint32_t co = (b[-1] >> 1) & 3u, ci = (b[k - 1] >> 1) & 3u;
                hf = rotl32(hf, 1) ^ rotl32(nt_seed(co), k) ^ nt_seed(ci);
                hr = rotl32(hr ^ nt_seed(co ^ 2u), 31) ^ rotl32(nt_seed(ci ^ 2u), k - 1);
            }
            A.key[g] = (A.alphabet == PHR_ALPHABET_DNA && hr < hf) ? hr : hf;
        }
    }
}

// Selected k-mer of every window: the leftmost minimum hash, or for canonical (DNA)
// minimizers the rightmost one when the window's l = w + k - 1 characters hold no more
// T/G (codes 2, 3) than A/C. And flag = the window selects another k-mer than the
// window before it (first window of a sequence: 1), so each selected k-mer is emitted
// once per run of windows.
// A thread takes kSketchRun consecutive windows of one sequence (plus the window before
// the first, for its flag): the T/G count rolls by one character per window, and the
// leftmost and rightmost positions of the window minimum roll by one key unless one of
// them leaves the window, when the window is scanned again.
__global__ void sketch_window_kernel(SketchArgs A) {
    const int l = A.w + A.k - 1;
    const int w = A.w;
    const bool dna = A.alphabet == PHR_ALPHABET_DNA;
    const uint64_t runs = (A.total_w + kSketchRun - 1) / kSketchRun;
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < runs;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t g0 = r * kSketchRun;
        const uint64_t g1 = g0 + kSketchRun < A.total_w ? g0 + kSketchRun : A.total_w;
        uint64_t s = find_seq(A.wbase, A.n, g0);
        uint64_t s_end = A.wbase[s + 1];
        const uint8_t* bs = nullptr;
        const uint64_t* kk = nullptr;
        int tg = 0;
        uint64_t lm = 0, rm = 0, bk = 0;  // leftmost / rightmost position of the window minimum, its key
        uint32_t prev = 0;
        auto scan_min = [&](uint64_t p) {  // minimum of window p from scratch
            lm = rm = p;
            bk = kk[p];
            for (uint64_t q = p + 1; q < p + w; ++q) {
                const uint64_t v = kk[q];
                if (v < bk) {
                    lm = rm = q;
                    bk = v;
                } else if (v == bk) {
                    rm = q;
                }
            }
        };
        auto roll = [&](uint64_t p) {  // window p from window p - 1
            if (dna) tg += static_cast<int>((bs[p + l - 1] >> 2) & 1) - static_cast<int>((bs[p - 1] >> 2) & 1);
            if (lm < p) {  // the leftmost minimum left the window (lm <= rm)
                scan_min(p);
                return;
            }
            const uint64_t v = kk[p + w - 1];
            if (v < bk) {
                lm = rm = p + w - 1;
                bk = v;
            } else if (v == bk) {
                rm = p + w - 1;
            }
        };
        auto pick = [&]() { return static_cast<uint32_t>((!dna || 2 * tg > l) ? lm : rm); };
        bool fresh = true;
        for (uint64_t g = g0; g < g1; ++g) {
            while (g >= s_end) {  // next sequence (skipping those without a window)
                ++s;
                s_end = A.wbase[s + 1];
                fresh = true;
            }
            const uint64_t p = g - A.wbase[s];
            if (fresh) {
                bs = A.seq + A.off[s];
                kk = A.key + A.kbase[s];
                // start at the window before the run (for this window's flag) if there is one
                const uint64_t p0 = p > 0 ? p - 1 : 0;
                tg = 0;
                if (dna)
                    for (int i = 0; i < l; ++i) tg += (bs[p0 + i] >> 2) & 1;  // bit 1 of the code (b >> 1) & 3
                scan_min(p0);
                if (p > 0) {
                    prev = pick();
                    roll(p);
                }
                fresh = false;
            } else {
                roll(p);
            }
            const uint32_t sel = pick();
            A.sel[g] = sel;
            A.flag[g] = (p == 0 || sel != prev) ? 1u : 0u;
            prev = sel;
        }
    }
}

// 2-bit value of the k-mer at b, first character in the low bits; DNA: the smaller of
// it and its reverse complement's.
__device__ __forceinline__ uint64_t kmer_value(const uint8_t* b, int k, int alphabet) {
    uint64_t vf = 0, vr = 0;
    for (int i = 0; i < k; ++i) {
        const uint64_t c = (b[i] >> 1) & 3u;
        vf |= c << (2 * i);
        vr |= (c ^ 2ull) << (2 * (k - 1 - i));
    }
    return (alphabet == PHR_ALPHABET_DNA && vr < vf) ? vr : vf;
}

struct SketchOut {
    uint64_t* values;
    uint32_t* positions;
    uint64_t* sk_off;       // per sequence: first output index (compact layout)
    uint32_t* sk_n;
    const uint64_t* remap_off;  // optional caller layout: output at remap_off[s] + local index
};

__global__ void sketch_scatter_kernel(SketchArgs A, const uint32_t* scan, SketchOut O) {
    for (uint64_t g = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; g < A.total_w;
         g += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (!A.flag[g]) continue;
        const uint64_t s = find_seq(A.wbase, A.n, g);
        const uint64_t first = A.wbase[s];
        const uint64_t local = scan[g] - scan[first];
        const uint64_t dst = O.remap_off ? O.remap_off[s] + local : static_cast<uint64_t>(scan[g]);
        const uint32_t b = A.sel[g];
        O.values[dst] = kmer_value(A.seq + A.off[s] + b, A.k, A.alphabet);
        O.positions[dst] = b;
    }
}

__global__ void sketch_count_kernel(SketchArgs A, const uint32_t* scan, SketchOut O) {
    const uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (s >= A.n) return;
    const uint64_t a = A.wbase[s], b = A.wbase[s + 1];
    uint32_t cnt = 0;
    uint64_t start = 0;
    if (b > a) {
        start = scan[a];
        cnt = scan[b - 1] + A.flag[b - 1] - scan[a];
    } else {
        start = (a < A.total_w) ? scan[a] : (A.total_w ? scan[A.total_w - 1] + A.flag[A.total_w - 1] : 0);
    }
    O.sk_n[s] = cnt;
    if (O.sk_off) O.sk_off[s] = start;
}

__global__ void count_bases_kernel(const uint32_t* len, uint64_t n, int k, int w, uint64_t* nk, uint64_t* nw) {
    const uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (s > n) return;
    if (s == n) {
        nk[s] = 0;
        nw[s] = 0;
        return;
    }
    const int64_t L = len[s];
    const int64_t kc = L >= k ? L - k + 1 : 0;
    nk[s] = static_cast<uint64_t>(kc);
    nw[s] = static_cast<uint64_t>(kc >= w ? kc - w + 1 : 0);
}

// ---------------------------------------------------------------------------
// Reverse complement (types.rs:91-107)
// ---------------------------------------------------------------------------
__global__ void revcomp_kernel(const uint8_t* seq, const uint64_t* off, const uint32_t* len, uint64_t n,
                               uint8_t* out, const uint64_t* out_off) {
    const uint64_t r = blockIdx.x;
    if (r >= n) return;
    const uint8_t* src = seq + off[r];
    uint8_t* dst = out + out_off[r];
    const uint32_t L = len[r];
    for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) {
        uint8_t b = src[L - 1 - i];
        switch (b) {
            case 'A': b = 'T'; break;
            case 'T': b = 'A'; break;
            case 'C': b = 'G'; break;
            case 'G': b = 'C'; break;
            case 'a': b = 't'; break;
            case 't': b = 'a'; break;
            case 'c': b = 'g'; break;
            case 'g': b = 'c'; break;
            default: break;
        }
        dst[i] = b;
    }
}

// ---------------------------------------------------------------------------
// Index lookup
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool idx_lookup(const IndexView& I, uint64_t key, uint32_t* off, uint32_t* cnt) {
    uint64_t slot = key & I.mask;
    for (uint64_t probe = 0; probe <= I.mask; ++probe) {
        const uint32_t c = I.cnt[slot];
        if (c == 0) return false;
        if (I.keys[slot] == key) {
            *off = I.off[slot];
            *cnt = c;
            return true;
        }
        slot = (slot + 1) & I.mask;
    }
    return false;
}

// ---------------------------------------------------------------------------
// Seeding: count, then emit as (tpos << 32 | qpos) keys (chain order is re-sorted by
// (tpos, qpos) anyway, so the query-position sort of find_seeds_indexed_capped is not
// materialised; the count it returns is).
// ---------------------------------------------------------------------------
struct SeedArgs {
    IndexView I;
    const uint64_t* sk_val;
    const uint32_t* sk_pos;
    const uint64_t* sk_off;
    const uint32_t* sk_n;
    uint64_t n_units;
    uint32_t* nseeds;
    const uint64_t* seed_off;
    uint64_t* skey;
    uint32_t* sidx;
    uint64_t* smin;
};

__global__ void seed_count_kernel(SeedArgs S) {
    const uint64_t u = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (u >= S.n_units) return;
    const uint64_t o = S.sk_off[u];
    const uint32_t n = S.sk_n[u];
    uint32_t total = 0;
    for (uint32_t i = lane; i < n; i += 32) {
        uint32_t off, cnt;
        if (idx_lookup(S.I, S.sk_val[o + i], &off, &cnt) && cnt <= S.I.occ_cap) total += cnt;
    }
    for (int d = 16; d; d >>= 1) total += __shfl_xor_sync(PHR_FULL_MASK, total, d);
    if (lane == 0) S.nseeds[u] = total;
}

__global__ void seed_emit_kernel(SeedArgs S) {
    const uint64_t u = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (u >= S.n_units) return;
    const uint64_t o = S.sk_off[u];
    const uint32_t n = S.sk_n[u];
    uint64_t w = S.seed_off[u];
    for (uint32_t c0 = 0; c0 < n; c0 += 32) {
        const uint32_t i = c0 + lane;
        uint32_t off = 0, cnt = 0;
        uint64_t val = 0;
        uint32_t qp = 0;
        if (i < n) {
            val = S.sk_val[o + i];
            qp = S.sk_pos[o + i];
            if (!idx_lookup(S.I, val, &off, &cnt) || cnt > S.I.occ_cap) cnt = 0;
        }
        uint32_t incl = cnt;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(PHR_FULL_MASK, incl, d);
            if (lane >= d) incl += v;
        }
        const uint64_t dst = w + incl - cnt;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t tp = S.I.pos[off + k];
            S.skey[dst + k] = (static_cast<uint64_t>(tp) << 32) | qp;
            S.sidx[dst + k] = static_cast<uint32_t>(dst + k);
            S.smin[dst + k] = val;
        }
        w += __shfl_sync(PHR_FULL_MASK, incl, 31);
    }
}

// ---------------------------------------------------------------------------
// Chaining DP (chaining.rs:134-187). One warp per unit; the predecessor scan of seed i
// runs 32 candidates per step. The reference's sequential bookkeeping (running best,
// dominated_count, n_skip and its early break) is reproduced with warp scans:
//   * running best before candidate j = max(seed_len, totals of earlier valid j)
//   * n_skip evolves by x -> max(x-1, 0) (improvement) or x -> x+1 (dominated past
//     max_skip); both are x -> max(x + a, b), closed under composition, so a
//     Hillis-Steele scan gives n_skip after every candidate; the first candidate that
//     takes it past max_skip ends the scan (its dominated_count increment included).
// ---------------------------------------------------------------------------
struct ChainArgs {
    uint64_t n_units;
    const uint32_t* nseeds;
    const uint64_t* seed_off;
    const uint64_t* skey_sorted;   // (tpos << 32 | qpos) sorted per unit
    int32_t* f;
    int32_t* pred;
    uint32_t* dominated;
};

constexpr int kSeedLen = 21, kMaxBand = 100, kMaxDistX = 100, kMaxIter = 5000, kMaxSkip = 25, kMinChainScore = 25;
constexpr int NEG_INF = -(1 << 29);

__global__ void chain_dp_kernel(ChainArgs C) {
    const uint64_t u = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (u >= C.n_units) return;
    const uint32_t n = C.nseeds[u];
    const uint64_t base = C.seed_off[u];
    const uint64_t* key = C.skey_sorted + base;
    int32_t* f = C.f + base;
    int32_t* pred = C.pred + base;
    uint32_t* dom = C.dominated + base;
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t ki = key[i];
        const int64_t ti = static_cast<int64_t>(ki >> 32), qi = static_cast<int64_t>(ki & 0xffffffffu);
        int best = kSeedLen;
        int best_pred = -1;
        int nskip = 0;
        const int64_t floor = i > static_cast<uint32_t>(kMaxIter) ? static_cast<int64_t>(i) - kMaxIter : 0;
        bool stop = false;
        for (int64_t jb = static_cast<int64_t>(i) - 1; jb >= floor && !stop; jb -= 32) {
            const int64_t j = jb - lane;
            const bool inb = j >= floor;
            int64_t tj = 0, qj = 0;
            if (inb) {
                const uint64_t kj = key[j];
                tj = static_cast<int64_t>(kj >> 32);
                qj = static_cast<int64_t>(kj & 0xffffffffu);
            }
            // positional cutoff (chaining.rs:159-163): ends the scan at the first such j
            const bool brk = inb && (ti - tj >= kMaxDistX + kSeedLen);
            const unsigned brk_mask = __ballot_sync(PHR_FULL_MASK, brk);
            const int brk_lane = brk_mask ? __ffs(brk_mask) - 1 : 32;
            const bool proc = inb && lane < brk_lane;
            // chain_score (chaining.rs:96-117)
            bool valid = false;
            int total = NEG_INF;
            if (proc) {
                const int64_t dq = qi - qj, dr = ti - tj;
                if (dq > 0 && dr > 0 && dr <= kMaxDistX + kSeedLen) {
                    const int64_t dd = dr > dq ? dr - dq : dq - dr;
                    if (dd <= kMaxBand) {
                        const int64_t dg = dr < dq ? dr : dq;
                        int sc = static_cast<int>(dg < kSeedLen ? dg : kSeedLen);
                        if (dd > 0) sc -= c_chain_pen[dd];
                        valid = true;
                        total = sc + f[j];
                    }
                }
            }
            // running best before this lane
            int pre = valid ? total : NEG_INF;
            int excl = NEG_INF;
            {
                int incl = pre;
                for (int d = 1; d < 32; d <<= 1) {
                    const int v = __shfl_up_sync(PHR_FULL_MASK, incl, d);
                    if (lane >= d) incl = max(incl, v);
                }
                excl = __shfl_up_sync(PHR_FULL_MASK, incl, 1);
                if (lane == 0) excl = NEG_INF;
            }
            const int run_best = max(best, excl);
            const bool improved = valid && total > run_best;
            const bool dominated = valid && !improved;
            const uint32_t dcnt = dominated ? dom[j] + 1 : 0;
            const bool incr = dominated && dcnt > static_cast<uint32_t>(kMaxSkip);
            // n_skip as composition of x -> max(x + a, b)
            int a = improved ? -1 : (incr ? 1 : 0);
            int b = improved ? 0 : NEG_INF;
            for (int d = 1; d < 32; d <<= 1) {
                const int pa = __shfl_up_sync(PHR_FULL_MASK, a, d);
                const int pb = __shfl_up_sync(PHR_FULL_MASK, b, d);
                if (lane >= d) {  // this = this o prev: max(max(x + pa, pb) + a, b)
                    b = max(pb + a, b);
                    a = pa + a;
                }
            }
            const int after = max(nskip + a, b);
            const bool over = incr && after > kMaxSkip;
            const unsigned over_mask = __ballot_sync(PHR_FULL_MASK, over);
            const int cut = over_mask ? __ffs(over_mask) - 1 : 31;  // last processed lane
            if (dominated && lane <= cut) dom[j] = dcnt;
            const unsigned imp_mask = __ballot_sync(PHR_FULL_MASK, improved && lane <= cut);
            if (imp_mask) {
                const int il = 31 - __clz(imp_mask);  // last improvement holds the maximum
                best = __shfl_sync(PHR_FULL_MASK, total, il);
                best_pred = static_cast<int>(__shfl_sync(PHR_FULL_MASK, static_cast<int>(j), il));
            }
            // n_skip after the last processed lane of this chunk
            const int last_proc = min(cut, brk_lane - 1);
            if (last_proc >= 0) nskip = __shfl_sync(PHR_FULL_MASK, after, last_proc);
            stop = (over_mask != 0) || (brk_mask != 0);
        }
        if (lane == 0) {
            f[i] = best;
            pred[i] = best_pred;
        }
        __syncwarp();
    }
}

// Backtrack (chaining.rs:189-225): ends in order of descending f (stable), one walk per
// unit on lane 0. Chains are produced in non-increasing score order, so the final
// stable sort by score is the identity.
struct BacktrackArgs {
    uint64_t n_units;
    const uint32_t* nseeds;
    const uint64_t* seed_off;
    const uint64_t* skey_sorted;
    const uint32_t* sidx_sorted;   // original seed index of each sorted position
    const uint64_t* smin;          // minimizer value by original seed index
    const int32_t* f;
    const int32_t* pred;
    const uint32_t* order;         // per unit, local indices by (f desc, index asc)
    uint8_t* used;
    uint32_t* nchains;
    // chain records (capacity = seeds of the unit)
    int64_t* ch_score;
    uint32_t* ch_first;            // first seed slot (unit-relative)
    uint32_t* ch_len;
    uint32_t* ch_tstart;
    uint64_t* ch_seed_key;         // chain seeds in query order (t << 32 | q)
    uint64_t* ch_seed_min;
};

__global__ void chain_backtrack_kernel(BacktrackArgs B) {
    const uint64_t u = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (u >= B.n_units) return;
    const uint32_t n = B.nseeds[u];
    const uint64_t base = B.seed_off[u];
    uint32_t nch = 0, slot = 0;
    for (uint32_t e = 0; e < n; ++e) {
        const uint32_t end = B.order[base + e];
        if (B.used[base + end] || B.f[base + end] < kMinChainScore) continue;
        uint32_t len = 0;
        int32_t cur = static_cast<int32_t>(end);
        while (cur >= 0 && !B.used[base + cur]) {
            B.used[base + cur] = 1;
            ++len;
            cur = B.pred[base + cur];
        }
        if (len == 0) continue;
        // second walk writes the seeds in query order (reverse of the walk)
        cur = static_cast<int32_t>(end);
        uint64_t first_key = 0;
        for (uint32_t k = 0; k < len; ++k) {
            const uint64_t key = B.skey_sorted[base + cur];
            B.ch_seed_key[base + slot + len - 1 - k] = key;
            B.ch_seed_min[base + slot + len - 1 - k] = B.smin[B.sidx_sorted[base + cur]];
            first_key = key;
            cur = B.pred[base + cur];
        }
        const int64_t t0 = static_cast<int64_t>(first_key >> 32), q0 = static_cast<int64_t>(first_key & 0xffffffffu);
        B.ch_score[base + nch] = B.f[base + end];
        B.ch_first[base + nch] = slot;
        B.ch_len[base + nch] = len;
        B.ch_tstart[base + nch] = static_cast<uint32_t>(t0 - q0 > 0 ? t0 - q0 : 0);
        ++nch;
        slot += len;
    }
    B.nchains[u] = nch;
}

__global__ void order_key_kernel(uint64_t n_units, const uint32_t* nseeds, const uint64_t* seed_off, const int32_t* f,
                                 uint64_t* okey, uint32_t* oval) {
    const uint64_t u = blockIdx.x;
    if (u >= n_units) return;
    const uint32_t n = nseeds[u];
    const uint64_t base = seed_off[u];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        okey[base + i] = (static_cast<uint64_t>(0x7FFFFFFF - f[base + i]) << 32) | i;
        oval[base + i] = i;
    }
}

__global__ void seg_bounds_kernel(uint64_t n_units, const uint64_t* seed_off, const uint32_t* nseeds, int* beg,
                                  int* end) {
    const uint64_t u = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (u >= n_units) return;
    beg[u] = static_cast<int>(seed_off[u]);
    end[u] = static_cast<int>(seed_off[u] + nseeds[u]);
}

// ---------------------------------------------------------------------------
// Anchor gating and pair lists (executor.rs:625-698, 528-567)
// ---------------------------------------------------------------------------
struct GateArgs {
    uint64_t n_reads;
    int alphabet;
    int strategy, gap_model;
    uint32_t chain_cap;
    const uint32_t* len;           // read lengths
    const uint8_t* has_stored;
    const uint32_t* sk_n;          // per unit sketch length
    const uint32_t* nseeds;        // per unit
    const uint32_t* nchains;
    const uint64_t* seed_off;      // chain arrays are unit-relative at seed_off
    const uint32_t* ch_tstart;
    uint64_t target_len;
    // per (read, orientation): engine, number of anchors; per read: early outcome
    int8_t* ou_engine;             // -1: not extended
    uint32_t* ou_count;
    int32_t* read_early;           // -1 none, else outcome (NoSeed for stored-empty)
    uint8_t* had_seeds;            // per read: a seed in either searched orientation
    uint8_t* rev_searched;         // per read: reverse orientation seeded and chained
    uint32_t* eng_count;           // [slot * (n_reads + 1) + read] pair counts, for the scans
};

__device__ __forceinline__ int pick_engine(int strategy, int gap_model, uint32_t qlen) {
    if (strategy == PHR_SENSITIVE) return gap_model == PHR_GAP_AFFINE ? PHR_ENGINE_WFA_AFFINE : PHR_ENGINE_WFA_LINEAR;
    return qlen <= 500 ? PHR_ENGINE_MYERS_FIT : PHR_ENGINE_WFA_LINEAR;
}

// engine id -> slot 0..2 (Myers fit, WFA linear, WFA affine)
__device__ __forceinline__ int eng_slot(int e) { return e == PHR_ENGINE_MYERS_FIT ? 0 : e == PHR_ENGINE_WFA_LINEAR ? 1 : 2; }

__global__ void gate_kernel(GateArgs G) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (r >= G.n_reads) return;
    const bool dna = G.alphabet == PHR_ALPHABET_DNA;
    const uint64_t uf = r, ur = G.n_reads + r;
    const uint32_t fs = G.nseeds[uf];
    // executor.rs:641-643: an empty forward sketch that found no seeds skips the
    // reverse orientation entirely (no reverse seeds, no reverse chains)
    const bool rev_searched = dna && !(fs == 0 && G.sk_n[uf] == 0);
    const uint32_t rs = rev_searched ? G.nseeds[ur] : 0;
    const bool had_seeds = fs > 0 || rs > 0;
    G.had_seeds[r] = had_seeds ? 1 : 0;
    G.rev_searched[r] = rev_searched ? 1 : 0;
    const bool stored = G.has_stored && G.has_stored[r];
    const uint64_t stride = G.n_reads + 1;
    G.eng_count[r] = G.eng_count[stride + r] = G.eng_count[2 * stride + r] = 0;
    G.ou_engine[2 * r] = G.ou_engine[2 * r + 1] = -1;
    G.ou_count[2 * r] = G.ou_count[2 * r + 1] = 0;
    G.read_early[r] = -1;
    if (stored && G.sk_n[uf] == 0 && !had_seeds) {  // executor.rs:671-674
        G.read_early[r] = PHR_OUT_NO_SEED;
        return;
    }
    const uint32_t fc = G.nchains[uf];
    const uint32_t rc = rev_searched ? G.nchains[ur] : 0;
    const bool ext_f = !(fc == 0 && rc > 0);
    const bool ext_r = !(fc > 0 && rc == 0);
    const uint32_t len_o[2] = {G.len[r], dna ? G.len[r] : 0u};
    const bool ext[2] = {ext_f, ext_r};
    const uint32_t nc[2] = {fc, rc};
    for (int o = 0; o < 2; ++o) {
        if (!ext[o]) continue;
        const int e = pick_engine(G.strategy, G.gap_model, len_o[o]);
        const uint32_t cnt = nc[o] == 0 ? 1u : min(nc[o], G.chain_cap);
        G.ou_engine[2 * r + o] = static_cast<int8_t>(e);
        G.ou_count[2 * r + o] = cnt;
        G.eng_count[eng_slot(e) * stride + r] += cnt;
    }
}

struct PairBuildArgs {
    uint64_t n_reads;
    const int8_t* ou_engine;
    const uint32_t* ou_count;
    const uint64_t* eng_first;     // [slot * (n_reads + 1) + read]: first pair index in the slot's list
    const uint32_t* nchains;
    const uint64_t* seed_off;
    const uint32_t* ch_tstart;
    const uint64_t* read_off;      // fwd reads in the query arena
    const uint64_t* rc_off;        // rc reads in the query arena
    const uint32_t* len;
    const uint8_t* rev_searched;   // per read
    int alphabet;
    uint64_t target_len;
    // per engine slot pair arrays
    uint64_t* q_off[3];
    uint32_t* q_len[3];
    uint64_t* t_off[3];
    uint32_t* t_len[3];
    uint32_t* t_seed[3];
    uint64_t* ou_first;            // per (read, orientation): first pair index in its engine list
};

__global__ void pair_build_kernel(PairBuildArgs B) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (r >= B.n_reads) return;
    const uint64_t stride = B.n_reads + 1;
    uint64_t next[3] = {B.eng_first[r], B.eng_first[stride + r], B.eng_first[2 * stride + r]};
    const bool dna = B.alphabet == PHR_ALPHABET_DNA;
    for (int o = 0; o < 2; ++o) {
        const int e = B.ou_engine[2 * r + o];
        if (e < 0) continue;
        const int es = eng_slot(e);
        const uint64_t u = o == 0 ? r : B.n_reads + r;
        const uint32_t nc = (o == 1 && !B.rev_searched[r]) ? 0u : B.nchains[u];
        const uint32_t cnt = B.ou_count[2 * r + o];
        const uint32_t qlen = (o == 1 && !dna) ? 0u : B.len[r];
        const uint64_t qo = o == 0 ? B.read_off[r] : B.rc_off[r];
        B.ou_first[2 * r + o] = next[es];
        for (uint32_t a = 0; a < cnt; ++a) {
            const uint32_t ts = nc == 0 ? 0u : B.ch_tstart[B.seed_off[u] + a];
            const uint64_t wend = ::min(static_cast<unsigned long long>(ts) + 2ull * qlen, static_cast<unsigned long long>(B.target_len));
            const uint64_t k = next[es]++;
            B.q_off[es][k] = qo;
            B.q_len[es][k] = qlen;
            B.t_off[es][k] = 0;
            B.t_len[es][k] = static_cast<uint32_t>(wend);
            B.t_seed[es][k] = ts;
        }
    }
}

// ---------------------------------------------------------------------------
// score_alignments + orientation choice (lib.rs:170-199, executor.rs:701-733)
// ---------------------------------------------------------------------------
struct SelectArgs {
    uint64_t n_reads;
    int alphabet, strategy;
    const uint32_t* len;
    const uint8_t* had_seeds;
    const int32_t* read_early;
    const int8_t* ou_engine;
    const uint32_t* ou_count;
    const uint64_t* ou_first;
    const phr_alignment* aln[3];
    const char* cigar[3];
    phr_read_result* res;          // per read
    uint64_t* sel_pair;            // per read list of (engine slot << 56 | pair index)
    uint32_t sel_cap;              // max alignments per read (= 2 * chain_cap)
    uint64_t* stats;               // 5 counters (atomic)
};

__device__ bool aln_equal(const phr_alignment& a, const char* ca, const phr_alignment& b, const char* cb) {
    if (a.edit_distance != b.edit_distance || a.query_start != b.query_start || a.query_end != b.query_end ||
        a.target_start != b.target_start || a.target_end != b.target_end || a.cigar_len != b.cigar_len)
        return false;
    for (uint32_t i = 0; i < a.cigar_len; ++i)
        if (ca[a.cigar_off + i] != cb[b.cigar_off + i]) return false;
    return true;
}

__global__ void select_kernel(SelectArgs S) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (r >= S.n_reads) return;
    phr_read_result out;
    memset(&out, 0, sizeof(out));
    const bool dna = S.alphabet == PHR_ALPHABET_DNA;
    const bool had_seeds = S.had_seeds[r] != 0;
    uint64_t* list = S.sel_pair + r * S.sel_cap;
    if (S.read_early[r] >= 0) {
        out.outcome = S.read_early[r];
        S.res[r] = out;
        atomicAdd(reinterpret_cast<unsigned long long*>(&S.stats[out.outcome]), 1ull);
        return;
    }
    // per orientation: primary index (first minimum edit distance among OK alignments)
    int prim[2] = {-1, -1};
    uint32_t prim_ed[2] = {0, 0};
    for (int o = 0; o < 2; ++o) {
        const int e = S.ou_engine[2 * r + o];
        if (e < 0) continue;
        const int es = eng_slot(e);
        const uint64_t first = S.ou_first[2 * r + o];
        for (uint32_t a = 0; a < S.ou_count[2 * r + o]; ++a) {
            const phr_alignment& x = S.aln[es][first + a];
            if (x.status != PHR_OK) continue;
            if (prim[o] < 0 || x.edit_distance < prim_ed[o]) {
                prim[o] = static_cast<int>(a);
                prim_ed[o] = x.edit_distance;
            }
        }
    }
    int win;
    if (prim[0] >= 0 && prim[1] >= 0 && prim_ed[1] < prim_ed[0]) win = 1;
    else if (prim[0] >= 0) win = 0;
    else if (prim[1] >= 0) win = 1;
    else {
        out.outcome = PHR_OUT_NO_ALIGNMENT;
        S.res[r] = out;
        atomicAdd(reinterpret_cast<unsigned long long*>(&S.stats[out.outcome]), 1ull);
        return;
    }
    const double qlen1 = static_cast<double>(S.len[r] > 0 ? S.len[r] : 1);
    const double primary_score = 1.0 - static_cast<double>(prim_ed[win]) / qlen1;
    if (S.strategy == PHR_FAST && static_cast<double>(prim_ed[win]) / qlen1 > 0.20) {
        out.outcome = PHR_OUT_FAST_CUTOFF;
        S.res[r] = out;
        atomicAdd(reinterpret_cast<unsigned long long*>(&S.stats[out.outcome]), 1ull);
        return;
    }
    out.outcome = primary_score >= 0.95 ? PHR_OUT_PLACED : (had_seeds ? PHR_OUT_BELOW_THRESHOLD : PHR_OUT_NO_SEED);
    out.has_result = 1;
    out.reverse = static_cast<uint8_t>(win);
    const int e = S.ou_engine[2 * r + win];
    const int es = eng_slot(e);
    const uint64_t first = S.ou_first[2 * r + win];
    const phr_alignment& P = S.aln[es][first + prim[win]];
    const char* cg = S.cigar[es];
    // score_alignments uses the length of the orientation's query bytes
    const double L = static_cast<double>((win == 1 && !dna) ? 0u : S.len[r]);
    uint32_t n = 0;
    list[n++] = (static_cast<uint64_t>(es) << 56) | (first + prim[win]);
    for (uint32_t a = 0; a < S.ou_count[2 * r + win]; ++a) {
        const phr_alignment& x = S.aln[es][first + a];
        if (x.status != PHR_OK) continue;
        if (aln_equal(x, cg, P, cg)) continue;
        const double pn = 1.0 - (static_cast<double>(P.edit_distance) / L);
        const double an = 1.0 - (static_cast<double>(x.edit_distance) / L);
        if (an / pn >= 0.95 && n < S.sel_cap) list[n++] = (static_cast<uint64_t>(es) << 56) | (first + a);
    }
    out.n_aln = n;
    S.res[r] = out;
    atomicAdd(reinterpret_cast<unsigned long long*>(&S.stats[out.outcome]), 1ull);
}

// Output packing: per read its alignments (primary first) with CIGAR text.
struct PackOutArgs {
    uint64_t n_reads;
    const phr_read_result* res;
    const uint64_t* sel_pair;
    uint32_t sel_cap;
    const uint64_t* aln_off;       // per read exclusive scan of n_aln
    const uint64_t* cig_off;       // per read exclusive scan of total cigar bytes
    const phr_alignment* aln[3];
    const char* cigar[3];
    phr_read_result* out_res;
    phr_alignment* out_aln;
    char* out_cigar;
};

__global__ void read_cigar_len_kernel(uint64_t n_reads, const phr_read_result* res, const uint64_t* sel_pair,
                                      uint32_t sel_cap, const phr_alignment* a0, const phr_alignment* a1,
                                      const phr_alignment* a2, uint64_t* n_aln, uint64_t* cig_len) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (r >= n_reads) return;
    const phr_alignment* A[3] = {a0, a1, a2};
    uint64_t c = 0;
    const uint32_t n = res[r].has_result ? res[r].n_aln : 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t sp = sel_pair[r * sel_cap + i];
        c += A[sp >> 56][sp & ((1ull << 56) - 1)].cigar_len;
    }
    n_aln[r] = n;
    cig_len[r] = c;
}

__global__ void pack_out_kernel(PackOutArgs P) {
    const uint64_t r = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= P.n_reads) return;
    phr_read_result rr = P.res[r];
    rr.aln_off = P.aln_off[r];
    const uint32_t n = rr.has_result ? rr.n_aln : 0;
    rr.n_aln = n;
    if (lane == 0) P.out_res[r] = rr;
    uint64_t co = P.cig_off[r];
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t sp = P.sel_pair[r * P.sel_cap + i];
        const int es = static_cast<int>(sp >> 56);
        const phr_alignment a = P.aln[es][sp & ((1ull << 56) - 1)];
        const char* src = P.cigar[es] + a.cigar_off;
        for (uint32_t c = lane; c < a.cigar_len; c += 32) P.out_cigar[co + c] = src[c];
        if (lane == 0) {
            phr_alignment o = a;
            o.cigar_off = co;
            P.out_aln[rr.aln_off + i] = o;
        }
        co += a.cigar_len;
    }
}



// ---------------------------------------------------------------------------
// Tandem repeats (detect_tandem_repeats, phraya-core/src/lib.rs:79-135)
// ---------------------------------------------------------------------------
__device__ __host__ __forceinline__ uint8_t upper_ascii(uint8_t c) {
    return (c >= 'a' && c <= 'z') ? static_cast<uint8_t>(c - 32) : c;
}

// The detector walks left to right; at a walk position p it takes the first period P in
// 4, 3, 2 with p + 3P <= n whose unit occurs three times in a row, i.e. s[i] == s[i + P]
// for every i in [p, p + 2P) (upper-cased bytes), and jumps past the repeat. Whether p
// passes that test does not depend on the walk, so every position is tested here in
// parallel; the walk itself then only visits the flagged positions (host, in order).
__global__ void repeat_candidate_kernel(const uint8_t* s, uint64_t base, uint64_t cnt, uint64_t n, uint8_t* flag) {
    const uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (j >= cnt) return;
    const uint64_t p = base + j;
    uint8_t f = 0;
    if (p + 6 <= n) {
        for (int P = 4; P >= 2 && !f; --P) {
            if (p + 3 * static_cast<uint64_t>(P) > n) continue;
            bool ok = true;
            for (int i = 0; i < 2 * P && ok; ++i) ok = upper_ascii(s[p + i]) == upper_ascii(s[p + i + P]);
            if (ok) f = static_cast<uint8_t>(P);
        }
    }
    flag[j] = f;
}

// ---------------------------------------------------------------------------
// Variant observations (extract_variants_from_cigar, phraya-align/src/executor.rs:814-1046)
// ---------------------------------------------------------------------------
struct VariantArgs {
    uint64_t n;
    const phr_read_result* res;     // packed results: read r's alignments at aln[aln_off ..], primary first
    const phr_alignment* aln;
    const char* cigar;
    const uint8_t* qarena;          // read r forward at rd_off[r], reverse complement at rd_off[n + r]
    const uint64_t* rd_off;
    const uint32_t* rd_len;
    const uint8_t* target;
    uint64_t tlen;
    const uint32_t* rep_start;      // tandem-repeat regions, sorted, end inclusive
    const uint32_t* rep_end;
    uint64_t n_rep;
    const uint32_t* hs_start;       // hotspot intervals [start, end), sorted
    const uint32_t* hs_end;
    uint64_t n_hs;
    uint64_t radius;
    uint64_t* cnt;                  // count pass: per read variants [r], coverage cells [n+1+r], alleles [2(n+1)+r]
    const uint64_t* off;            // write pass: exclusive scans of cnt, same layout
    phr_variant* var;
    uint32_t* cov;
    phr_allele* al;
};

// partition_point(start <= pos) over a sorted array: the number of entries <= pos.
__device__ __forceinline__ uint64_t upper_bound_u32(const uint32_t* a, uint64_t n, uint64_t pos) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (a[mid] <= pos) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// One warp per read. Every lane parses the primary CIGAR (the same bytes, so the loads
// broadcast and control flow stays warp-uniform); the lanes split each variant's
// coverage cells and the insertion allele counts. WRITE = false counts the read's
// outputs, WRITE = true writes them at the scanned offsets.
template <bool WRITE>
__global__ void variant_kernel(VariantArgs V) {
    const uint64_t r = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= V.n) return;
    const uint64_t n1 = V.n + 1;
    uint64_t nv = 0, nc = 0, na = 0;
    if (WRITE) {
        nv = V.off[r];
        nc = V.off[n1 + r];
        na = V.off[2 * n1 + r];
    }
    const phr_read_result rr = V.res[r];
    if (rr.has_result && rr.n_aln) {
        const phr_alignment pa = V.aln[rr.aln_off];
        const uint8_t* q = V.qarena + V.rd_off[rr.reverse ? V.n + r : r];
        const uint64_t qlen = V.rd_len[r];
        const uint64_t tlen = V.tlen;
        // primary_score (executor.rs:713) times kmer_uniqueness is the confidence.
        const double score =
            1.0 - static_cast<double>(pa.edit_distance) / static_cast<double>(qlen > 1 ? qlen : 1);
        const char* c = V.cigar + pa.cigar_off;
        const uint32_t clen = pa.cigar_len;
        auto emit = [&](uint64_t tp, uint8_t ref, uint8_t type, uint64_t ins_lo, uint64_t ins_hi, uint8_t allele) {
            const uint64_t ws = tp >= V.radius ? tp - V.radius : 0;
            const uint64_t we = min(tp + V.radius + 1, tlen);
            const uint64_t cl = we - ws;
            // alleles: one for a SNP / deletion, the distinct inserted bytes for an insertion
            uint32_t bm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint32_t nal = 1;
            if (type == 1) {
                for (uint64_t k = ins_lo + lane; k < ins_hi; k += 32) {
                    const uint32_t b = q[k];
#pragma unroll
                    for (int w = 0; w < 8; ++w)
                        if ((b >> 5) == static_cast<uint32_t>(w)) bm[w] |= 1u << (b & 31);
                }
                nal = 0;
#pragma unroll
                for (int w = 0; w < 8; ++w) {
                    bm[w] = __reduce_or_sync(0xffffffffu, bm[w]);
                    nal += __popc(bm[w]);
                }
            }
            if (WRITE) {
                for (uint64_t j = lane; j < cl; j += 32) {  // get_abs_multi over the read's windows
                    const uint64_t pos = ws + j;
                    uint32_t cv = 0;
                    for (uint32_t a = 0; a < rr.n_aln; ++a) {
                        const phr_alignment& x = V.aln[rr.aln_off + a];
                        const uint64_t s0 = min(static_cast<uint64_t>(x.target_start), tlen);
                        const uint64_t e0 = min(static_cast<uint64_t>(x.target_end), tlen);
                        cv += (pos >= s0 && pos < e0) ? 1u : 0u;
                    }
                    V.cov[nc + j] = cv;
                }
                if (type == 1) {
                    uint32_t k_out = 0;
#pragma unroll
                    for (int w = 0; w < 8; ++w) {
                        uint32_t bits = bm[w];
                        while (bits) {
                            const uint32_t b = static_cast<uint32_t>(w) * 32 + (__ffs(bits) - 1);
                            bits &= bits - 1;
                            uint32_t cntb = 0;
                            for (uint64_t k = ins_lo + lane; k < ins_hi; k += 32) cntb += q[k] == b ? 1u : 0u;
                            cntb = __reduce_add_sync(0xffffffffu, cntb);
                            if (lane == 0) {
                                phr_allele o;
                                o.base = static_cast<uint8_t>(b);
                                o._pad[0] = o._pad[1] = o._pad[2] = 0;
                                o.count = cntb;
                                V.al[na + k_out] = o;
                            }
                            ++k_out;
                        }
                    }
                } else if (lane == 0) {
                    phr_allele o;
                    o.base = allele;
                    o._pad[0] = o._pad[1] = o._pad[2] = 0;
                    o.count = 1;
                    V.al[na] = o;
                }
                if (lane == 0) {
                    phr_variant v;
                    v.position = static_cast<uint32_t>(tp);
                    v.ref_base = ref;
                    v.variant_type = type;
                    const uint64_t ri = upper_bound_u32(V.rep_start, V.n_rep, tp);
                    v.in_tandem_repeat = (ri > 0 && tp < V.rep_end[ri - 1]) ? 1 : 0;
                    v.strand = rr.reverse;
                    v.read = static_cast<uint32_t>(r);
                    v.edit_distance = pa.edit_distance;
                    const uint64_t hi = upper_bound_u32(V.hs_start, V.n_hs, static_cast<uint32_t>(tp));
                    v.kmer_uniqueness = (hi > 0 && static_cast<uint32_t>(tp) < V.hs_end[hi - 1]) ? 0.0 : 1.0;
                    v.confidence = v.kmer_uniqueness * score;
                    v.coverage_off = nc;
                    v.coverage_len = static_cast<uint32_t>(cl);
                    v.coverage_variant_offset = static_cast<uint32_t>(tp - ws);
                    v.allele_off = na;
                    v.n_alleles = nal;
                    v._pad = 0;
                    V.var[nv] = v;
                }
            }
            nv += 1;
            nc += cl;
            na += nal;
        };
        uint64_t qp = 0, tp = pa.target_start;
        uint32_t i = 0;
        while (i < clen) {
            uint64_t count = 0;
            bool digits = false;
            while (i < clen && c[i] >= '0' && c[i] <= '9') {
                count = count * 10 + static_cast<uint64_t>(c[i] - '0');
                ++i;
                digits = true;
            }
            if (i >= clen) break;
            const char op = c[i++];
            if (!digits) count = 1;  // parse_cigar: an empty count reads as 1
            if (op == 'M') {
                qp += count;
                tp += count;
            } else if (op == 'X') {
                for (uint64_t k = 0; k < count; ++k)
                    if (qp + k < qlen && tp + k < tlen) emit(tp + k, V.target[tp + k], 0, 0, 0, q[qp + k]);
                qp += count;
                tp += count;
            } else if (op == 'I') {  // target bases absent from the read: a deletion at tp
                if (tp < tlen && qp < qlen) emit(tp, V.target[tp], 2, 0, 0, '.');
                tp += count;
            } else if (op == 'D') {  // read bases absent from the target: an insertion at tp
                if (qp < qlen && tp < tlen) emit(tp, '.', 1, qp, min(qp + count, qlen), 0);
                qp += count;
            }
        }
    }
    if (!WRITE && lane == 0) {
        V.cnt[r] = nv;
        V.cnt[n1 + r] = nc;
        V.cnt[2 * n1 + r] = na;
    }
}

// Coverage merge (phraya-cli/src/main.rs:556-572): one warp per alignment adds its
// window's quantized count to the resident track. The window count is 1 everywhere
// (compute_windowed_coverage, executor.rs:1071-1090), quantized per window
// (quantize_coverage, executor.rs:1092-1096) unless `depth` asks for the raw count.
__global__ void coverage_add_kernel(const phr_alignment* aln, uint64_t n_aln, uint64_t tlen, int depth,
                                    uint32_t* track) {
    const uint64_t a = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (a >= n_aln) return;
    const uint32_t c = 1;
    const uint32_t w = depth ? c : ((c + 2) / 5) * 5;
    if (w == 0) return;
    const uint64_t s0 = min(static_cast<uint64_t>(aln[a].target_start), tlen);
    const uint64_t e0 = min(static_cast<uint64_t>(aln[a].target_end), tlen);
    for (uint64_t p = s0 + lane; p < e0; p += 32) atomicAdd(track + p, w);
}

// ---------------------------------------------------------------------------
// Minimizer index build (build_minimizer_index, seeding.rs:31-37)
// ---------------------------------------------------------------------------
__global__ void iota_u32_kernel(uint32_t* out, uint64_t n) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = static_cast<uint32_t>(i);
}

// Positions grouped by value: the stable sort by value kept each value's entries in
// sketch order, which is the order of its position list.
__global__ void gather_pos_kernel(const uint32_t* pos, const uint32_t* order, uint64_t n, uint32_t* out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = pos[order[i]];
}

// Open addressing, linear probing from value & mask (the lookup's probe sequence). A slot
// is claimed by swapping its count from 0 (counts are at least 1); the table has at least
// twice as many slots as values, so the probe ends; it is bounded by the table size.
__global__ void index_insert_kernel(const uint64_t* uniq, const uint32_t* run_cnt, const uint32_t* run_off,
                                    const int* n_runs, uint64_t mask, uint64_t* keys, uint32_t* off, uint32_t* cnt) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (r >= static_cast<uint64_t>(*n_runs)) return;
    const uint64_t v = uniq[r];
    uint64_t s = v & mask;
    for (uint64_t probe = 0; probe <= mask; ++probe) {
        if (atomicCAS(cnt + s, 0u, run_cnt[r]) == 0u) {
            keys[s] = v;
            off[s] = run_off[r];
            return;
        }
        s = (s + 1) & mask;
    }
}

__global__ void offset_add_kernel(const uint64_t* in, uint64_t* out, uint64_t n, uint64_t add) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = in[i] + add;
}

// Stored forward sketches (plan.get_read_sketch, executor.rs:615-624) replace the
// computed ones: their entries are appended after the computed ones and the unit's
// (offset, count) re-pointed.
__global__ void stored_patch_kernel(uint64_t n, const uint8_t* has_stored, const uint64_t* s_off, const uint32_t* s_n,
                                    uint64_t base, uint64_t* sk_off, uint32_t* sk_n) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (r >= n || !has_stored[r]) return;
    sk_off[r] = base + s_off[r];
    sk_n[r] = s_n[r];
}

__global__ void u32_to_u64_kernel(const uint32_t* in, uint64_t* out, uint64_t n) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = in[i];
}

}  // namespace

// ===========================================================================
// Host side
// ===========================================================================
static void init_penalty_table(int device) {
    static bool done[64] = {false};
    if (device >= 0 && device < 64 && done[device]) return;
    int32_t pen[101];
    pen[0] = 0;
    for (int dd = 1; dd <= 100; ++dd) {
        // chaining.rs:111-115: (0.21 * dd + 0.5 * log2(dd + 1)).round(), half away from zero
        const double lin = 0.21 * static_cast<double>(dd);
        const double lg = 0.5 * std::log2(static_cast<double>(dd) + 1.0);
        pen[dd] = static_cast<int32_t>(std::round(lin + lg));
    }
    cudaMemcpyToSymbol(c_chain_pen, pen, sizeof(pen));
    if (device >= 0 && device < 64) done[device] = true;
}

phr_status sketch_device(Ctx* ctx, DeviceArena& A, const uint8_t* seq, const uint64_t* off, const uint32_t* len,
                         uint64_t n, int k, int w, int alphabet, uint64_t** values, uint32_t** positions,
                         uint64_t** sk_off, uint32_t** sk_n, uint64_t* total, const uint64_t* remap_off) {
    cudaStream_t st = ctx->stream;
    const unsigned T = 256;
    uint64_t* nk = static_cast<uint64_t*>(A.take((n + 1) * 8));
    uint64_t* nw = static_cast<uint64_t*>(A.take((n + 1) * 8));
    uint64_t* kb = static_cast<uint64_t*>(A.take((n + 1) * 8));
    uint64_t* wb = static_cast<uint64_t*>(A.take((n + 1) * 8));
    if (!wb) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (sketch)");
    {
        KernelScope ks(ctx, "sketch_sizes");
        count_bases_kernel<<<blocks_for(n + 1, T), T, 0, st>>>(len, n, k, w, nk, nw);
    }
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, nk, kb, static_cast<int>(n + 1), st);
    void* tmp = A.take(tb + 256);
    if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (sketch scan)");
    size_t t2 = tb;
    cub::DeviceScan::ExclusiveSum(tmp, t2, nk, kb, static_cast<int>(n + 1), st);
    t2 = tb;
    cub::DeviceScan::ExclusiveSum(tmp, t2, nw, wb, static_cast<int>(n + 1), st);
    uint64_t tot[2] = {0, 0};
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[0], kb + n, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[1], wb + n, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    const uint64_t TK = tot[0], TW = tot[1];
    SketchArgs S{seq, off, len, n, kb, wb, TK, TW, k, w, alphabet, nullptr, nullptr, nullptr};
    S.key = static_cast<uint64_t*>(A.take(TK * 8 + 8));
    S.flag = static_cast<uint32_t*>(A.take(TW * 4 + 8));
    S.sel = static_cast<uint32_t*>(A.take(TW * 4 + 8));
    uint32_t* scan = static_cast<uint32_t*>(A.take(TW * 4 + 8));
    SketchOut O{};
    if (!remap_off) {
        *values = static_cast<uint64_t*>(A.take(TW * 8 + 8));
        *positions = static_cast<uint32_t*>(A.take(TW * 4 + 8));
        *sk_off = static_cast<uint64_t*>(A.take(n * 8 + 8));
    }
    if (!*sk_n) *sk_n = static_cast<uint32_t*>(A.take(n * 4 + 8));
    if (!*sk_n || !*values || !scan) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (sketch outputs)");
    O.values = *values;
    O.positions = *positions;
    O.sk_off = remap_off ? nullptr : *sk_off;
    O.sk_n = *sk_n;
    O.remap_off = remap_off;
    const unsigned grid = std::max<unsigned>(1, std::min<unsigned>(blocks_for(std::max<uint64_t>(TK, 1), T),
                                                                    static_cast<unsigned>(ctx->sm_count * 16)));
    // the key and window kernels take kSketchRun positions per thread
    const auto run_grid = [&](uint64_t total) {
        return std::max<unsigned>(1, std::min<unsigned>(blocks_for(std::max<uint64_t>((total + kSketchRun - 1) /
                                                                                      kSketchRun, 1), T),
                                                        static_cast<unsigned>(ctx->sm_count * 16)));
    };
    const unsigned grid_w = run_grid(TW);
    if (TK) {
        KernelScope ks(ctx, "sketch_key");
        sketch_key_kernel<<<run_grid(TK), T, 0, st>>>(S);
    }
    if (TW) {
        {
            KernelScope ks(ctx, "sketch_window");
            sketch_window_kernel<<<grid_w, T, 0, st>>>(S);
        }
        size_t ts = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, ts, S.flag, scan, static_cast<int>(TW), st);
        void* t3 = A.take(ts + 256);
        if (!t3) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (sketch flags)");
        cub::DeviceScan::ExclusiveSum(t3, ts, S.flag, scan, static_cast<int>(TW), st);
        KernelScope ks(ctx, "sketch_scatter");
        sketch_scatter_kernel<<<grid, T, 0, st>>>(S, scan, O);
    }
    if (n) {
        KernelScope ks(ctx, "sketch_count");
        sketch_count_kernel<<<blocks_for(n, T), T, 0, st>>>(S, scan, O);
    }
    uint64_t t_last = 0;
    if (TW) {
        uint32_t a = 0, b = 0;
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&a, scan + TW - 1, 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&b, S.flag + TW - 1, 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        t_last = static_cast<uint64_t>(a) + b;
    }
    *total = t_last;
    PHR_CUDA_TRY(ctx, cudaGetLastError());
    return PHR_OK;
}

// Builds the device index from a host sketch (build_minimizer_index + occurrence cap).
// build_minimizer_index (seeding.rs:31-37) and seed_occurrence_cap (seeding.rs:94-102,
// floor 256, executor.rs:258) on the device from a sketch already on the device: a stable
// radix sort of (value, entry) pairs groups each value's positions in sketch order, a
// run-length encoding gives the distinct values and their counts, the median count sets
// the cap, and the values go into an open-addressing table. Temporaries live in the
// context's extension arena; the index itself is one allocation kept by `idx`.
static phr_status build_index_device(Ctx* ctx, phr_index* idx, const uint64_t* vals, const uint32_t* pos, uint64_t n) {
    cudaStream_t st = ctx->stream;
    const unsigned T = 256;
    if (n > 0x7FFFFFF0ull) return set_error(ctx, PHR_ERR_ARG, "sketch of more than 2^31 - 16 minimizers");
    const int ni = static_cast<int>(n);
    DeviceArena& A = ctx->arena;
    A.reset();
    size_t t_sort = 0, t_rle = 0, t_scan = 0, t_csort = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t_sort, static_cast<const uint64_t*>(nullptr),
                                    static_cast<uint64_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
                                    static_cast<uint32_t*>(nullptr), ni, 0, 64, st);
    cub::DeviceRunLengthEncode::Encode(nullptr, t_rle, static_cast<const uint64_t*>(nullptr),
                                       static_cast<uint64_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                       static_cast<int*>(nullptr), ni, st);
    cub::DeviceScan::ExclusiveSum(nullptr, t_scan, static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), ni, st);
    cub::DeviceRadixSort::SortKeys(nullptr, t_csort, static_cast<const uint32_t*>(nullptr),
                                   static_cast<uint32_t*>(nullptr), ni, 0, 32, st);
    const size_t t_need = std::max({t_sort, t_rle, t_scan, t_csort}) + 256;
    auto al = [](size_t b) { return (b + 511) / 256 * 256; };
    PHR_CUDA_TRY(ctx, A.reserve(al(n * 8) * 2 + al(n * 4) * 6 + al(64) + al(t_need) + 4096));
    uint64_t* skeys = static_cast<uint64_t*>(A.take(n * 8 + 8));
    uint64_t* uniq = static_cast<uint64_t*>(A.take(n * 8 + 8));
    uint32_t* ent = static_cast<uint32_t*>(A.take(n * 4 + 8));
    uint32_t* order = static_cast<uint32_t*>(A.take(n * 4 + 8));
    uint32_t* run_cnt = static_cast<uint32_t*>(A.take(n * 4 + 8));
    uint32_t* run_off = static_cast<uint32_t*>(A.take(n * 4 + 8));
    uint32_t* cnt_sorted = static_cast<uint32_t*>(A.take(n * 4 + 8));
    int* d_runs = static_cast<int*>(A.take(64));
    void* tmp = A.take(t_need);
    if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (index build)");
    int h_runs = 0;
    uint32_t h_median = 0;
    if (n) {
        {
            KernelScope ks(ctx, "index_iota");
            iota_u32_kernel<<<blocks_for(n, T), T, 0, st>>>(ent, n);
        }
        size_t t = t_need;
        cub::DeviceRadixSort::SortPairs(tmp, t, vals, skeys, ent, order, ni, 0, 64, st);
        t = t_need;
        cub::DeviceRunLengthEncode::Encode(tmp, t, skeys, uniq, run_cnt, d_runs, ni, st);
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&h_runs, d_runs, sizeof(int), cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        t = t_need;
        cub::DeviceScan::ExclusiveSum(tmp, t, run_cnt, run_off, h_runs, st);
        t = t_need;
        cub::DeviceRadixSort::SortKeys(tmp, t, run_cnt, cnt_sorted, h_runs, 0, 32, st);
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&h_median, cnt_sorted + h_runs / 2, 4, cudaMemcpyDeviceToHost, st));
    }
    const uint64_t distinct = static_cast<uint64_t>(h_runs);
    uint64_t slots = 16;
    while (slots < 2 * distinct + 16) slots <<= 1;
    const size_t bytes = slots * (8 + 4 + 4) + n * 4 + 256;
    void* blk = nullptr;
    PHR_CUDA_TRY(ctx, cudaMalloc(&blk, bytes));
    idx->d_block = blk;
    char* p = static_cast<char*>(blk);
    uint64_t* keys = reinterpret_cast<uint64_t*>(p);
    uint32_t* off = reinterpret_cast<uint32_t*>(p + slots * 8);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(p + slots * 12);
    uint32_t* dpos = reinterpret_cast<uint32_t*>(p + slots * 16);
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(keys, 0, slots * 8, st));
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(off, 0, slots * 4, st));
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt, 0, slots * 4, st));
    if (n) {
        {
            KernelScope ks(ctx, "index_gather");
            gather_pos_kernel<<<blocks_for(n, T), T, 0, st>>>(pos, order, n, dpos);
        }
        KernelScope ks(ctx, "index_insert");
        index_insert_kernel<<<blocks_for(distinct, T), T, 0, st>>>(uniq, run_cnt, run_off, d_runs, slots - 1, keys, off,
                                                                  cnt);
    }
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    PHR_CUDA_TRY(ctx, cudaGetLastError());
    const uint64_t cap = distinct ? std::max<uint64_t>(256, static_cast<uint64_t>(h_median) * 8) : 256;
    idx->view.keys = keys;
    idx->view.off = off;
    idx->view.cnt = cnt;
    idx->view.pos = dpos;
    idx->view.mask = slots - 1;
    idx->view.occ_cap = static_cast<uint32_t>(std::min<uint64_t>(cap, 0xFFFFFFFFu));
    idx->n_min = n;
    idx->n_distinct = distinct;
    idx->device_bytes = bytes + idx->target_len + 64;
    return PHR_OK;
}

// detect_tandem_repeats (phraya-core/src/lib.rs:79-135, min_repeat_count 3) over the
// index's target: the device flags every position that passes the walk's test, the host
// walks the flagged positions in order (skipping those inside an accepted repeat) and
// extends each accepted repeat unit by unit. `target` is the caller's host copy.
static phr_status detect_repeats(Ctx* ctx, phr_index* idx, const uint8_t* target) {
    const uint64_t n = idx->target_len;
    idx->rep_start.clear();
    idx->rep_end.clear();
    cudaStream_t st = ctx->stream;
    if (n >= 6) {
        const uint64_t chunk = std::min<uint64_t>(n, 1ull << 28);
        DeviceArena& A = ctx->pipe;
        A.reset();
        size_t tb = 0;
        thrust::counting_iterator<uint32_t> it(0);
        cub::DeviceSelect::Flagged(nullptr, tb, it, static_cast<const uint8_t*>(nullptr),
                                   static_cast<uint32_t*>(nullptr), static_cast<int*>(nullptr),
                                   static_cast<int>(chunk), st);
        PHR_CUDA_TRY(ctx, A.reserve(chunk * 5 + tb + (4 << 20)));
        uint8_t* flag = static_cast<uint8_t*>(A.take(chunk + 64));
        uint32_t* cand = static_cast<uint32_t*>(A.take(chunk * 4 + 64));
        int* d_cnt = static_cast<int*>(A.take(64));
        void* tmp = A.take(tb + 256);
        if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (repeat scan)");
        std::vector<uint32_t> h;
        uint64_t cur = 0;
        for (uint64_t base = 0; base < n; base += chunk) {
            const uint64_t cnt = std::min<uint64_t>(chunk, n - base);
            {
                KernelScope ks(ctx, "repeat_candidates");
                repeat_candidate_kernel<<<blocks_for(cnt, 256), 256, 0, st>>>(idx->d_target, base, cnt, n, flag);
            }
            size_t t2 = tb;
            cub::DeviceSelect::Flagged(tmp, t2, thrust::counting_iterator<uint32_t>(static_cast<uint32_t>(base)),
                                       flag, cand, d_cnt, static_cast<int>(cnt), st);
            int hc = 0;
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&hc, d_cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
            PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
            h.resize(static_cast<size_t>(hc));
            if (hc) PHR_CUDA_TRY(ctx, cudaMemcpy(h.data(), cand, static_cast<size_t>(hc) * 4, cudaMemcpyDeviceToHost));
            for (uint32_t p : h) {
                if (p < cur) continue;
                int P = 4;
                for (; P >= 2; --P) {  // the same test the device applied; the first period wins
                    if (p + 3ull * P > n) continue;
                    bool ok = true;
                    for (int i = 0; i < 2 * P && ok; ++i) ok = upper_ascii(target[p + i]) == upper_ascii(target[p + i + P]);
                    if (ok) break;
                }
                if (P < 2) continue;
                uint64_t end = p + static_cast<uint64_t>(P);
                while (end + P <= n) {
                    bool eq = true;
                    for (int i = 0; i < P && eq; ++i) eq = upper_ascii(target[p + i]) == upper_ascii(target[end + i]);
                    if (!eq) break;
                    end += P;
                }
                idx->rep_start.push_back(p);
                idx->rep_end.push_back(static_cast<uint32_t>(end - 1));
                cur = end;
            }
        }
    }
    const uint64_t nr = idx->rep_start.size();
    if (nr) {
        PHR_CUDA_TRY(ctx, cudaMalloc(&idx->d_rep, nr * 8));
        PHR_CUDA_TRY(ctx, cudaMemcpy(idx->d_rep, idx->rep_start.data(), nr * 4, cudaMemcpyHostToDevice));
        PHR_CUDA_TRY(ctx, cudaMemcpy(idx->d_rep + nr, idx->rep_end.data(), nr * 4, cudaMemcpyHostToDevice));
        idx->device_bytes += nr * 8;
    }
    return PHR_OK;
}

phr_status index_create(Ctx* ctx, const uint8_t* target, uint64_t tlen, const phr_sketch* sketch, int alphabet,
                        phr_index** out) {
    init_penalty_table(ctx->device);
    if (tlen > 0xFFFFFFF0ull) return set_error(ctx, PHR_ERR_ARG, "target longer than 2^32 - 16 bases");
    phr_index* idx = new phr_index();
    idx->ctx = ctx;
    idx->alphabet = alphabet;
    idx->target_len = tlen;
    idx->k = alphabet == PHR_ALPHABET_DNA ? 21 : 6;
    idx->w = alphabet == PHR_ALPHABET_DNA ? 11 : 5;
    cudaError_t e = cudaMalloc(&idx->d_target, tlen + 64);
    if (e != cudaSuccess) {
        delete idx;
        return cuda_status(ctx, e, "cudaMalloc(target)");
    }
    if (tlen) {
        e = cudaMemcpy(idx->d_target, target, tlen, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            delete idx;
            return cuda_status(ctx, e, "cudaMemcpy(target)");
        }
    }
    DeviceArena& A = ctx->pipe;
    A.reset();
    const uint64_t* d_vals = nullptr;
    const uint32_t* d_pos = nullptr;
    uint64_t total = 0;
    if (sketch) {
        if (sketch->n && (!sketch->values || !sketch->positions)) {
            delete idx;
            return set_error(ctx, PHR_ERR_ARG, "sketch arrays are NULL");
        }
        if (sketch->k > 0) idx->k = sketch->k;
        if (sketch->w > 0) idx->w = sketch->w;
        total = sketch->n;
        e = A.reserve(total * 12 + 4096);
        uint64_t* v = static_cast<uint64_t*>(A.take(total * 8 + 8));
        uint32_t* q = static_cast<uint32_t*>(A.take(total * 4 + 8));
        if (e != cudaSuccess || !q) {
            delete idx;
            return e != cudaSuccess ? cuda_status(ctx, e, "arena reserve (sketch upload)")
                                    : set_error(ctx, PHR_ERR_OOM, "arena exhausted (sketch upload)");
        }
        if (total) {
            e = cudaMemcpyAsync(v, sketch->values, total * 8, cudaMemcpyHostToDevice, ctx->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(q, sketch->positions, total * 4, cudaMemcpyHostToDevice, ctx->stream);
            if (e != cudaSuccess) {
                delete idx;
                return cuda_status(ctx, e, "sketch upload");
            }
        }
        d_vals = v;
        d_pos = q;
    } else {
        e = A.reserve(tlen * 40 + (64 << 20));
        if (e != cudaSuccess) {
            delete idx;
            return cuda_status(ctx, e, "arena reserve (target sketch)");
        }
        uint64_t* off = static_cast<uint64_t*>(A.take(8));
        uint32_t* len = static_cast<uint32_t*>(A.take(4));
        const uint64_t zero = 0;
        const uint32_t l32 = static_cast<uint32_t>(tlen);
        cudaMemcpy(off, &zero, 8, cudaMemcpyHostToDevice);
        cudaMemcpy(len, &l32, 4, cudaMemcpyHostToDevice);
        uint64_t *vals = nullptr, *sk_off = nullptr;
        uint32_t *poss = nullptr, *sk_n = nullptr;
        phr_status s = sketch_device(ctx, A, idx->d_target, off, len, 1, idx->k, idx->w, alphabet, &vals, &poss,
                                     &sk_off, &sk_n, &total, nullptr);
        if (s != PHR_OK) {
            delete idx;
            return s;
        }
        d_vals = vals;
        d_pos = poss;
    }
    phr_status s = build_index_device(ctx, idx, d_vals, d_pos, total);
    if (s == PHR_OK) s = detect_repeats(ctx, idx, target);
    if (s != PHR_OK) {
        delete idx;
        return s;
    }
    *out = idx;
    return PHR_OK;
}

phr_status seed_chain_device(Ctx* ctx, DeviceArena& A, const phr_index* idx, const uint64_t* sk_val,
                             const uint32_t* sk_pos, const uint64_t* sk_off, const uint32_t* sk_n, uint64_t n_units,
                             ChainResult* C) {
    cudaStream_t st = ctx->stream;
    const unsigned T = 256;
    C->n_units = n_units;
    C->nseeds = static_cast<uint32_t*>(A.take((n_units + 1) * 4 + 8));
    C->seed_off = static_cast<uint64_t*>(A.take((n_units + 1) * 8 + 8));
    C->nchains = static_cast<uint32_t*>(A.take(n_units * 4 + 8));
    uint64_t* n64 = static_cast<uint64_t*>(A.take((n_units + 1) * 8 + 8));
    if (!n64) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (seeds)");
    SeedArgs S{};
    S.I = idx->view;
    S.sk_val = sk_val;
    S.sk_pos = sk_pos;
    S.sk_off = sk_off;
    S.sk_n = sk_n;
    S.n_units = n_units;
    S.nseeds = C->nseeds;
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(C->nseeds, 0, (n_units + 1) * 4, st));
    if (n_units) {
        KernelScope ks(ctx, "seed_count");
        seed_count_kernel<<<blocks_for(n_units * 32, T), T, 0, st>>>(S);
    }
    {
        KernelScope ks(ctx, "seed_widen");
        u32_to_u64_kernel<<<blocks_for(n_units + 1, T), T, 0, st>>>(C->nseeds, n64, n_units + 1);
    }
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, n64, C->seed_off, static_cast<int>(n_units + 1), st);
    void* tmp = A.take(tb + 256);
    if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (seed scan)");
    cub::DeviceScan::ExclusiveSum(tmp, tb, n64, C->seed_off, static_cast<int>(n_units + 1), st);
    uint64_t total = 0;
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&total, C->seed_off + n_units, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    C->total_seeds = total;
    if (total > 0x7FFFFFF0ull) return set_error(ctx, PHR_ERR_CAPACITY, "too many seeds in one batch");
    const uint64_t tt = total + 1;
    // per-seed arrays live in their own arena, sized from the exact count
    DeviceArena& SA = ctx->seeds;
    SA.reset();
    PHR_CUDA_TRY(ctx, SA.reserve(tt * 160 + (16 << 20)));
    auto takeS = [&](size_t b) { return SA.take(b); };
    uint64_t* skey = static_cast<uint64_t*>(takeS(tt * 8));
    uint32_t* sidx = static_cast<uint32_t*>(takeS(tt * 4));
    C->smin = static_cast<uint64_t*>(takeS(tt * 8));
    C->skey_sorted = static_cast<uint64_t*>(takeS(tt * 8));
    C->sidx_sorted = static_cast<uint32_t*>(takeS(tt * 4));
    C->f = static_cast<int32_t*>(takeS(tt * 4));
    C->pred = static_cast<int32_t*>(takeS(tt * 4));
    uint32_t* dom = static_cast<uint32_t*>(takeS(tt * 4));
    uint64_t* okey = static_cast<uint64_t*>(takeS(tt * 8));
    uint32_t* oval = static_cast<uint32_t*>(takeS(tt * 4));
    uint64_t* okey_s = static_cast<uint64_t*>(takeS(tt * 8));
    uint32_t* order = static_cast<uint32_t*>(takeS(tt * 4));
    uint8_t* used = static_cast<uint8_t*>(takeS(tt));
    C->ch_score = static_cast<int64_t*>(takeS(tt * 8));
    C->ch_first = static_cast<uint32_t*>(takeS(tt * 4));
    C->ch_len = static_cast<uint32_t*>(takeS(tt * 4));
    C->ch_tstart = static_cast<uint32_t*>(takeS(tt * 4));
    C->ch_seed_key = static_cast<uint64_t*>(takeS(tt * 8));
    C->ch_seed_min = static_cast<uint64_t*>(takeS(tt * 8));
    int* beg = static_cast<int*>(A.take(n_units * 4 + 8));
    int* end = static_cast<int*>(A.take(n_units * 4 + 8));
    if (!end) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (chain arrays)");
    S.seed_off = C->seed_off;
    S.skey = skey;
    S.sidx = sidx;
    S.smin = C->smin;
    if (n_units) {
        KernelScope ks(ctx, "seed_emit");
        seed_emit_kernel<<<blocks_for(n_units * 32, T), T, 0, st>>>(S);
    }
    if (n_units) {
        KernelScope ks(ctx, "seg_bounds");
        seg_bounds_kernel<<<blocks_for(n_units, T), T, 0, st>>>(n_units, C->seed_off, C->nseeds, beg, end);
    }
    if (total) {
        tb = 0;
        cub::DeviceSegmentedSort::SortPairs(nullptr, tb, skey, C->skey_sorted, sidx, C->sidx_sorted,
                                            static_cast<int>(total), static_cast<int>(n_units), beg, end, st);
        tmp = A.take(tb + 256);
        if (!tmp) {
            PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
            tmp = SA.take(tb + 256);
        }
        if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (seed sort)");
        cub::DeviceSegmentedSort::SortPairs(tmp, tb, skey, C->skey_sorted, sidx, C->sidx_sorted,
                                            static_cast<int>(total), static_cast<int>(n_units), beg, end, st);
        PHR_CUDA_TRY(ctx, cudaMemsetAsync(dom, 0, tt * 4, st));
        ChainArgs CA{n_units, C->nseeds, C->seed_off, C->skey_sorted, C->f, C->pred, dom};
        {
            KernelScope ks(ctx, "chain_dp");
            chain_dp_kernel<<<blocks_for(n_units * 32, T), T, 0, st>>>(CA);
        }
        {
            KernelScope ks(ctx, "order_key");
            order_key_kernel<<<static_cast<unsigned>(n_units), 64, 0, st>>>(n_units, C->nseeds, C->seed_off, C->f,
                                                                             okey, oval);
        }
        tb = 0;
        cub::DeviceSegmentedSort::SortPairs(nullptr, tb, okey, okey_s, oval, order, static_cast<int>(total),
                                            static_cast<int>(n_units), beg, end, st);
        tmp = A.take(tb + 256);
        if (!tmp) tmp = SA.take(tb + 256);
        if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (order sort)");
        cub::DeviceSegmentedSort::SortPairs(tmp, tb, okey, okey_s, oval, order, static_cast<int>(total),
                                            static_cast<int>(n_units), beg, end, st);
        PHR_CUDA_TRY(ctx, cudaMemsetAsync(used, 0, tt, st));
    }
    BacktrackArgs B{n_units, C->nseeds, C->seed_off, C->skey_sorted, C->sidx_sorted, C->smin, C->f, C->pred,
                    order, used, C->nchains, C->ch_score, C->ch_first, C->ch_len, C->ch_tstart, C->ch_seed_key,
                    C->ch_seed_min};
    if (n_units) {
        KernelScope ks(ctx, "chain_backtrack");
        chain_backtrack_kernel<<<blocks_for(n_units, 128), 128, 0, st>>>(B);
    }
    PHR_CUDA_TRY(ctx, cudaGetLastError());
    return PHR_OK;
}

size_t align_arena_need(uint64_t n, uint64_t seq_bytes, uint64_t stored_total) {
    // query arena 2x, sketch scratch ~ 40 B per base and orientation, seeds/chains
    // ~ 160 B per seed (seeds <= minimizers * cap; a generous per-base bound is used),
    // per-read bookkeeping and the per-engine extension outputs.
    return 2 * seq_bytes + 2 * seq_bytes * 48 + 2 * seq_bytes * 64 + stored_total * 12 + n * 4096 + (256ull << 20);
}

phr_status align_reads_device(Ctx* ctx, const phr_index* idx, const uint8_t* d_seq, const uint64_t* d_off,
                              const uint32_t* d_len, uint64_t n, uint64_t seq_bytes, const uint8_t* d_has_stored,
                              const uint64_t* d_s_off, const uint32_t* d_s_n, const uint64_t* d_s_val,
                              const uint32_t* d_s_pos, const phr_align_config& cfg, AlignOutput* out) {
    cudaStream_t st = ctx->stream;
    const unsigned T = 256;
    DeviceArena& A = ctx->pipe;
    const bool dna = idx->alphabet == PHR_ALPHABET_DNA;
    // query arena: [fwd reads as given | rc reads at seq_bytes + off]
    uint8_t* qarena = static_cast<uint8_t*>(A.take(2 * seq_bytes + 64));
    uint64_t* rd_off = static_cast<uint64_t*>(A.take(2 * n * 8 + 8));
    uint32_t* rd_len = static_cast<uint32_t*>(A.take(2 * n * 4 + 8));
    if (!rd_len) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (reads)");
    if (seq_bytes) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(qarena, d_seq, seq_bytes, cudaMemcpyDeviceToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(rd_off, d_off, n * 8, cudaMemcpyDeviceToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(rd_len, d_len, n * 4, cudaMemcpyDeviceToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(rd_len + n, d_len, n * 4, cudaMemcpyDeviceToDevice, st));
    uint64_t* rc_off = rd_off + n;
    out->qarena = qarena;
    out->rd_off = rd_off;
    out->rd_len = rd_len;
    if (n) {
        KernelScope ks(ctx, "rc_offsets");
        offset_add_kernel<<<blocks_for(n, T), T, 0, st>>>(d_off, rc_off, n, seq_bytes);
    }
    if (dna && n) {
        KernelScope ks(ctx, "revcomp");
        revcomp_kernel<<<static_cast<unsigned>(n), 128, 0, st>>>(d_seq, d_off, d_len, n, qarena, rc_off);
    }
    // sketches: forward for every read, reverse complement for DNA (executor.rs:615-660)
    const uint64_t n_units = 2 * n;
    uint64_t *sk_val = nullptr, *sk_off = nullptr;
    uint32_t *sk_pos = nullptr, *sk_n = nullptr;
    uint64_t sk_total = 0;
    phr_status s = sketch_device(ctx, A, qarena, rd_off, rd_len, dna ? 2 * n : n, idx->k, idx->w, idx->alphabet,
                                 &sk_val, &sk_pos, &sk_off, &sk_n, &sk_total, nullptr);
    if (s != PHR_OK) return s;
    if (!dna) {  // protein: reverse units are empty (no reverse strand, ADR-0013)
        uint64_t* so2 = static_cast<uint64_t*>(A.take(n_units * 8 + 8));
        uint32_t* sn2 = static_cast<uint32_t*>(A.take(n_units * 4 + 8));
        if (!sn2) return set_error(ctx, PHR_ERR_OOM, "arena exhausted");
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(so2, sk_off, n * 8, cudaMemcpyDeviceToDevice, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(sn2, sk_n, n * 4, cudaMemcpyDeviceToDevice, st));
        PHR_CUDA_TRY(ctx, cudaMemsetAsync(so2 + n, 0, n * 8, st));
        PHR_CUDA_TRY(ctx, cudaMemsetAsync(sn2 + n, 0, n * 4, st));
        sk_off = so2;
        sk_n = sn2;
    }
    if (d_has_stored) {
        // append the stored entries and re-point those reads' forward units
        uint64_t stored_total = 0;
        {
            // total stored entries = max over reads of s_off + s_n; caller sizes are exact
            std::vector<uint64_t> so(n);
            std::vector<uint32_t> sn(n);
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(so.data(), d_s_off, n * 8, cudaMemcpyDeviceToHost, st));
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(sn.data(), d_s_n, n * 4, cudaMemcpyDeviceToHost, st));
            PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
            for (uint64_t r = 0; r < n; ++r) stored_total = std::max(stored_total, so[r] + sn[r]);
        }
        uint64_t* v2 = static_cast<uint64_t*>(A.take((sk_total + stored_total) * 8 + 8));
        uint32_t* p2 = static_cast<uint32_t*>(A.take((sk_total + stored_total) * 4 + 8));
        if (!p2) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (stored sketches)");
        if (sk_total) {
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(v2, sk_val, sk_total * 8, cudaMemcpyDeviceToDevice, st));
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(p2, sk_pos, sk_total * 4, cudaMemcpyDeviceToDevice, st));
        }
        if (stored_total) {
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(v2 + sk_total, d_s_val, stored_total * 8, cudaMemcpyDeviceToDevice, st));
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(p2 + sk_total, d_s_pos, stored_total * 4, cudaMemcpyDeviceToDevice, st));
        }
        {
            KernelScope ks(ctx, "stored_patch");
            stored_patch_kernel<<<blocks_for(n, T), T, 0, st>>>(n, d_has_stored, d_s_off, d_s_n, sk_total, sk_off,
                                                                sk_n);
        }
        sk_val = v2;
        sk_pos = p2;
    }
    ChainResult C;
    s = seed_chain_device(ctx, A, idx, sk_val, sk_pos, sk_off, sk_n, n_units, &C);
    if (s != PHR_OK) return s;

    // ---- anchor gating and per-engine pair lists ----
    const uint32_t K = cfg.strategy == PHR_FAST ? 1 : cfg.strategy == PHR_BALANCED ? 2 : 50;
    const uint64_t stride = n + 1;
    GateArgs G{};
    G.n_reads = n;
    G.alphabet = idx->alphabet;
    G.strategy = cfg.strategy;
    G.gap_model = cfg.gap_model;
    G.chain_cap = K;
    G.len = d_len;
    G.has_stored = d_has_stored;
    G.sk_n = sk_n;
    G.nseeds = C.nseeds;
    G.nchains = C.nchains;
    G.seed_off = C.seed_off;
    G.ch_tstart = C.ch_tstart;
    G.target_len = idx->target_len;
    G.ou_engine = static_cast<int8_t*>(A.take(2 * n + 8));
    G.ou_count = static_cast<uint32_t*>(A.take(2 * n * 4 + 8));
    G.read_early = static_cast<int32_t*>(A.take(n * 4 + 8));
    G.had_seeds = static_cast<uint8_t*>(A.take(n + 8));
    G.rev_searched = static_cast<uint8_t*>(A.take(n + 8));
    G.eng_count = static_cast<uint32_t*>(A.take(3 * stride * 4 + 16));
    uint64_t* cnt64 = static_cast<uint64_t*>(A.take(3 * stride * 8 + 16));
    uint64_t* eng_first = static_cast<uint64_t*>(A.take(3 * stride * 8 + 16));
    uint64_t* ou_first = static_cast<uint64_t*>(A.take(2 * n * 8 + 8));
    if (!ou_first) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (gating)");
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(G.eng_count, 0, 3 * stride * 4, st));
    if (n) {
        KernelScope ks(ctx, "gate");
        gate_kernel<<<blocks_for(n, T), T, 0, st>>>(G);
    }
    {
        KernelScope ks(ctx, "pair_count_widen");
        u32_to_u64_kernel<<<blocks_for(3 * stride, T), T, 0, st>>>(G.eng_count, cnt64, 3 * stride);
    }
    uint64_t eng_total[3] = {0, 0, 0};
    {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt64, eng_first, static_cast<int>(stride), st);
        void* tmp = A.take(tb + 256);
        if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (pair scan)");
        for (int e = 0; e < 3; ++e) {
            size_t t2 = tb;
            cub::DeviceScan::ExclusiveSum(tmp, t2, cnt64 + e * stride, eng_first + e * stride,
                                          static_cast<int>(stride), st);
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&eng_total[e], eng_first + e * stride + n, 8, cudaMemcpyDeviceToHost, st));
        }
        PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    }
    PairBuildArgs PB{};
    PB.n_reads = n;
    PB.ou_engine = G.ou_engine;
    PB.ou_count = G.ou_count;
    PB.eng_first = eng_first;
    PB.nchains = C.nchains;
    PB.seed_off = C.seed_off;
    PB.ch_tstart = C.ch_tstart;
    PB.read_off = rd_off;
    PB.rc_off = rc_off;
    PB.len = d_len;
    PB.rev_searched = G.rev_searched;
    PB.alphabet = idx->alphabet;
    PB.target_len = idx->target_len;
    PB.ou_first = ou_first;
    for (int e = 0; e < 3; ++e) {
        const uint64_t np = eng_total[e] + 1;
        PB.q_off[e] = static_cast<uint64_t*>(A.take(np * 8));
        PB.q_len[e] = static_cast<uint32_t*>(A.take(np * 4));
        PB.t_off[e] = static_cast<uint64_t*>(A.take(np * 8));
        PB.t_len[e] = static_cast<uint32_t*>(A.take(np * 4));
        PB.t_seed[e] = static_cast<uint32_t*>(A.take(np * 4));
        if (!PB.t_seed[e]) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (pairs)");
    }
    if (n) {
        KernelScope ks(ctx, "pair_build");
        pair_build_kernel<<<blocks_for(n, T), T, 0, st>>>(PB);
    }
    // ---- extension: one batched engine call per engine in use ----
    static const phr_engine slot_engine[3] = {PHR_ENGINE_MYERS_FIT, PHR_ENGINE_WFA_LINEAR, PHR_ENGINE_WFA_AFFINE};
    uint64_t sum_qt_e[3] = {0, 0, 0};
    for (int e = 0; e < 3; ++e) {
        if (!eng_total[e]) continue;
        std::vector<uint32_t> ql(eng_total[e]), tl(eng_total[e]), ts(eng_total[e]);
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(ql.data(), PB.q_len[e], eng_total[e] * 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(tl.data(), PB.t_len[e], eng_total[e] * 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(ts.data(), PB.t_seed[e], eng_total[e] * 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        for (uint64_t i = 0; i < eng_total[e]; ++i) sum_qt_e[e] += static_cast<uint64_t>(ql[i]) + tl[i] - ts[i];
    }
    // extension outputs: alignments + worst-case CIGAR text (2 * (q + t) per pair) in ctx->io
    {
        size_t need = 1024;
        for (int e = 0; e < 3; ++e)
            need += eng_total[e] * (sizeof(phr_alignment) + 16) + 2 * sum_qt_e[e] + 1024;
        ctx->io.reset();
        PHR_CUDA_TRY(ctx, ctx->io.reserve(need));
    }
    for (int e = 0; e < 3; ++e) {
        out->eng_pairs[e] = eng_total[e];
        if (!eng_total[e]) continue;
        const uint64_t cap = 2 * sum_qt_e[e] + 16 * eng_total[e];
        out->eng_aln[e] = static_cast<phr_alignment*>(ctx->io.take(eng_total[e] * sizeof(phr_alignment)));
        out->eng_cigar[e] = static_cast<char*>(ctx->io.take(cap + 16));
        if (!out->eng_cigar[e]) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (extension outputs)");
        DevPairs dp;
        dp.n = eng_total[e];
        dp.seq = qarena;
        dp.seq_bytes = 2 * seq_bytes;
        dp.q_off = PB.q_off[e];
        dp.q_len = PB.q_len[e];
        dp.t_off = PB.t_off[e];
        dp.t_len = PB.t_len[e];
        dp.q_seed = nullptr;
        dp.t_seed = PB.t_seed[e];
        dp.t_seq = idx->d_target;
        DevResults r;
        r.aln = out->eng_aln[e];
        r.cigar = out->eng_cigar[e];
        r.cigar_capacity = cap;
        phr_affine_costs costs{2, 4, 1};  // AffineCosts::default (wfa_simd.rs:537-539)
        {
            HostScope hs(ctx, "host:extend");
            s = run_extend(ctx, slot_engine[e], dp, costs, &r, sum_qt_e[e]);
        }
        if (s != PHR_OK) return s;
    }
    // ---- score_alignments + orientation choice ----
    SelectArgs SA{};
    SA.n_reads = n;
    SA.alphabet = idx->alphabet;
    SA.strategy = cfg.strategy;
    SA.len = d_len;
    SA.had_seeds = G.had_seeds;
    SA.read_early = G.read_early;
    SA.ou_engine = G.ou_engine;
    SA.ou_count = G.ou_count;
    SA.ou_first = ou_first;
    for (int e = 0; e < 3; ++e) {
        SA.aln[e] = out->eng_aln[e];
        SA.cigar[e] = out->eng_cigar[e];
    }
    out->res = static_cast<phr_read_result*>(A.take(n * sizeof(phr_read_result) + 8));
    out->stats = static_cast<uint64_t*>(A.take(64));
    SA.res = out->res;
    SA.sel_cap = 2 * K;
    SA.sel_pair = static_cast<uint64_t*>(A.take(n * SA.sel_cap * 8 + 8));
    SA.stats = out->stats;
    if (!SA.sel_pair || !out->stats) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (select)");
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(out->stats, 0, 64, st));
    if (n) {
        KernelScope ks(ctx, "select");
        select_kernel<<<blocks_for(n, 128), 128, 0, st>>>(SA);
    }
    out->sel_pair = SA.sel_pair;
    out->sel_cap = SA.sel_cap;
    PHR_CUDA_TRY(ctx, cudaGetLastError());
    return PHR_OK;
}

// Packs device results into caller-visible device buffers, then copies them to the host
// arena. Returns PHR_ERR_CAPACITY if the host arena is too small.
static phr_status pack_to_host(Ctx* ctx, DeviceArena& A, uint64_t n, const AlignOutput& o,
                               phr_read_result_arena* host, phr_align_stats* stats, PackedDev* dev = nullptr) {
    cudaStream_t st = ctx->stream;
    const unsigned T = 256;
    uint64_t* n_aln = static_cast<uint64_t*>(A.take((n + 1) * 8 + 8));
    uint64_t* cig_len = static_cast<uint64_t*>(A.take((n + 1) * 8 + 8));
    uint64_t* aln_off = static_cast<uint64_t*>(A.take((n + 1) * 8 + 8));
    uint64_t* cig_off = static_cast<uint64_t*>(A.take((n + 1) * 8 + 8));
    if (!cig_off) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (pack)");
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(n_aln + n, 0, 8, st));
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(cig_len + n, 0, 8, st));
    if (n) {
        KernelScope ks(ctx, "read_cigar_len");
        read_cigar_len_kernel<<<blocks_for(n, T), T, 0, st>>>(n, o.res, o.sel_pair, o.sel_cap, o.eng_aln[0],
                                                              o.eng_aln[1], o.eng_aln[2], n_aln, cig_len);
    }
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, n_aln, aln_off, static_cast<int>(n + 1), st);
    void* tmp = A.take(tb + 256);
    if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (pack scan)");
    size_t t2 = tb;
    cub::DeviceScan::ExclusiveSum(tmp, t2, n_aln, aln_off, static_cast<int>(n + 1), st);
    t2 = tb;
    cub::DeviceScan::ExclusiveSum(tmp, t2, cig_len, cig_off, static_cast<int>(n + 1), st);
    uint64_t tot[2] = {0, 0};
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[0], aln_off + n, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[1], cig_off + n, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (tot[0] > host->aln_capacity) return set_error(ctx, PHR_ERR_CAPACITY, "alignment arena too small");
    if (tot[1] > host->cigar_capacity) return set_error(ctx, PHR_ERR_CAPACITY, "CIGAR arena too small");
    phr_read_result* d_res = static_cast<phr_read_result*>(A.take(n * sizeof(phr_read_result) + 8));
    phr_alignment* d_aln = static_cast<phr_alignment*>(A.take(tot[0] * sizeof(phr_alignment) + 8));
    char* d_cig = static_cast<char*>(A.take(tot[1] + 8));
    if (!d_cig) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (pack out)");
    PackOutArgs P{n, o.res, o.sel_pair, o.sel_cap, aln_off, cig_off, {o.eng_aln[0], o.eng_aln[1], o.eng_aln[2]},
                  {o.eng_cigar[0], o.eng_cigar[1], o.eng_cigar[2]}, d_res, d_aln, d_cig};
    if (n) {
        KernelScope ks(ctx, "pack_out");
        pack_out_kernel<<<blocks_for(n * 32, T), T, 0, st>>>(P);
    }
    uint64_t hst[8] = {0};
    if (n) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(host->reads, d_res, n * sizeof(phr_read_result), cudaMemcpyDeviceToHost, st));
    if (tot[0])
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(host->aln, d_aln, tot[0] * sizeof(phr_alignment), cudaMemcpyDeviceToHost, st));
    if (tot[1]) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(host->cigar, d_cig, tot[1], cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(hst, o.stats, 40, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    host->aln_used = tot[0];
    host->cigar_used = tot[1];
    if (dev) {
        dev->res = d_res;
        dev->aln = d_aln;
        dev->cigar = d_cig;
    }
    if (stats) {
        stats->placed += hst[PHR_OUT_PLACED];
        stats->no_seed += hst[PHR_OUT_NO_SEED];
        stats->below_threshold += hst[PHR_OUT_BELOW_THRESHOLD];
        stats->fast_cutoff += hst[PHR_OUT_FAST_CUTOFF];
        stats->no_alignment += hst[PHR_OUT_NO_ALIGNMENT];
    }
    return PHR_OK;
}

// Variant observations of the packed results (align_read, executor.rs:735-775): a count
// pass, three exclusive scans, a write pass into device buffers, then one copy per array
// into the caller's arena. On PHR_ERR_CAPACITY the arena's *_used fields hold the sizes
// needed.
static phr_status variants_to_host(Ctx* ctx, DeviceArena& A, uint64_t n, const phr_index* idx, const AlignOutput& o,
                                   const PackedDev& pd, const phr_align_config& cfg, const phr_variant_config* vcfg,
                                   phr_variant_arena* vout) {
    cudaStream_t st = ctx->stream;
    const unsigned T = 256;
    VariantArgs V{};
    V.n = n;
    V.res = pd.res;
    V.aln = pd.aln;
    V.cigar = pd.cigar;
    V.qarena = o.qarena;
    V.rd_off = o.rd_off;
    V.rd_len = o.rd_len;
    V.target = idx->d_target;
    V.tlen = idx->target_len;
    V.n_rep = idx->rep_start.size();
    V.rep_start = idx->d_rep;
    V.rep_end = idx->d_rep ? idx->d_rep + V.n_rep : nullptr;
    // AlignConfig::new (executor.rs:124-128): the strategy's coverage radius
    V.radius = vcfg && vcfg->coverage_radius ? vcfg->coverage_radius
               : cfg.strategy == PHR_FAST    ? 150
               : cfg.strategy == PHR_BALANCED ? 50
                                              : 25;
    const uint64_t nhs = vcfg && vcfg->hotspot_start && vcfg->hotspot_end ? vcfg->n_hotspots : 0;
    V.n_hs = nhs;
    if (nhs) {
        uint32_t* hs = static_cast<uint32_t*>(A.take(nhs * 8 + 16));
        if (!hs) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (hotspots)");
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(hs, vcfg->hotspot_start, nhs * 4, cudaMemcpyHostToDevice, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(hs + nhs, vcfg->hotspot_end, nhs * 4, cudaMemcpyHostToDevice, st));
        V.hs_start = hs;
        V.hs_end = hs + nhs;
    }
    const uint64_t n1 = n + 1;
    uint64_t* cnt = static_cast<uint64_t*>(A.take(3 * n1 * 8 + 8));
    uint64_t* off = static_cast<uint64_t*>(A.take(3 * n1 * 8 + 8));
    if (!off) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (variant counts)");
    for (int k = 0; k < 3; ++k) PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt + k * n1 + n, 0, 8, st));
    V.cnt = cnt;
    if (n) {
        KernelScope ks(ctx, "variant_count");
        variant_kernel<false><<<blocks_for(n * 32, T), T, 0, st>>>(V);
    }
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, static_cast<int>(n1), st);
    void* tmp = A.take(tb + 256);
    if (!tmp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (variant scan)");
    for (int k = 0; k < 3; ++k) {
        size_t t2 = tb;
        cub::DeviceScan::ExclusiveSum(tmp, t2, cnt + k * n1, off + k * n1, static_cast<int>(n1), st);
    }
    uint64_t tot[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k)
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[k], off + k * n1 + n, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    vout->variant_used = tot[0];
    vout->coverage_used = tot[1];
    vout->allele_used = tot[2];
    if (tot[0] > vout->variant_capacity) return set_error(ctx, PHR_ERR_CAPACITY, "variant arena too small");
    if (tot[1] > vout->coverage_capacity) return set_error(ctx, PHR_ERR_CAPACITY, "coverage arena too small");
    if (tot[2] > vout->allele_capacity) return set_error(ctx, PHR_ERR_CAPACITY, "allele arena too small");
    V.off = off;
    V.var = static_cast<phr_variant*>(A.take(tot[0] * sizeof(phr_variant) + 8));
    V.cov = static_cast<uint32_t*>(A.take(tot[1] * 4 + 8));
    V.al = static_cast<phr_allele*>(A.take(tot[2] * sizeof(phr_allele) + 8));
    if (!V.al) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (variant outputs)");
    if (n) {
        KernelScope ks(ctx, "variant_write");
        variant_kernel<true><<<blocks_for(n * 32, T), T, 0, st>>>(V);
    }
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(vout->read_variant_off, off, n1 * 8, cudaMemcpyDeviceToHost, st));
    if (tot[0]) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(vout->variants, V.var, tot[0] * sizeof(phr_variant), cudaMemcpyDeviceToHost, st));
    if (tot[1]) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(vout->coverage, V.cov, tot[1] * 4, cudaMemcpyDeviceToHost, st));
    if (tot[2]) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(vout->alleles, V.al, tot[2] * sizeof(phr_allele), cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return PHR_OK;
}

phr_status align_reads_host(Ctx* ctx, const phr_index* idx, const phr_read_batch* rb, const phr_align_config& cfg,
                            phr_read_result_arena* out, phr_align_stats* stats, const phr_variant_config* vcfg,
                            phr_variant_arena* vout) {
    cudaStream_t st = ctx->stream;
    const uint64_t n = rb->n_reads;
    out->aln_used = 0;
    out->cigar_used = 0;
    if (n == 0) return PHR_OK;
    for (uint64_t i = 0; i < n; ++i)
        if (rb->off[i] + rb->len[i] > rb->seq_bytes) return set_error(ctx, PHR_ERR_ARG, "read reaches past seq_bytes");
    uint64_t stored_total = 0;
    const bool has_st = rb->has_stored && rb->s_off && rb->s_n && rb->s_values && rb->s_positions;
    if (has_st)
        for (uint64_t i = 0; i < n; ++i)
            if (rb->has_stored[i]) stored_total = std::max<uint64_t>(stored_total, rb->s_off[i] + rb->s_n[i]);
    HostScope hs_all(ctx, "host:align_reads");
    DeviceArena& A = ctx->pipe;
    A.reset();
    PHR_CUDA_TRY(ctx, A.reserve(align_arena_need(n, rb->seq_bytes, stored_total) + rb->seq_bytes + n * 32));
    uint8_t* d_seq = static_cast<uint8_t*>(A.take(rb->seq_bytes + 64));
    uint64_t* d_off = static_cast<uint64_t*>(A.take(n * 8));
    uint32_t* d_len = static_cast<uint32_t*>(A.take(n * 4));
    uint8_t* d_hs = nullptr;
    uint64_t *d_so = nullptr, *d_sv = nullptr;
    uint32_t *d_sn = nullptr, *d_sp = nullptr;
    if (!d_len) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (read upload)");
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_seq, rb->seq, rb->seq_bytes, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_off, rb->off, n * 8, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_len, rb->len, n * 4, cudaMemcpyHostToDevice, st));
    if (has_st) {
        d_hs = static_cast<uint8_t*>(A.take(n + 8));
        d_so = static_cast<uint64_t*>(A.take(n * 8 + 8));
        d_sn = static_cast<uint32_t*>(A.take(n * 4 + 8));
        d_sv = static_cast<uint64_t*>(A.take(stored_total * 8 + 8));
        d_sp = static_cast<uint32_t*>(A.take(stored_total * 4 + 8));
        if (!d_sp) return set_error(ctx, PHR_ERR_OOM, "arena exhausted (stored sketches)");
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_hs, rb->has_stored, n, cudaMemcpyHostToDevice, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_so, rb->s_off, n * 8, cudaMemcpyHostToDevice, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_sn, rb->s_n, n * 4, cudaMemcpyHostToDevice, st));
        if (stored_total) {
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_sv, rb->s_values, stored_total * 8, cudaMemcpyHostToDevice, st));
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_sp, rb->s_positions, stored_total * 4, cudaMemcpyHostToDevice, st));
        }
    }
    AlignOutput o;
    PackedDev pd;
    phr_status s;
    {
        HostScope hs(ctx, "host:device_pipeline");
        s = align_reads_device(ctx, idx, d_seq, d_off, d_len, n, rb->seq_bytes, d_hs, d_so, d_sn, d_sv, d_sp, cfg, &o);
    }
    if (s != PHR_OK) return s;
    {
        HostScope hs(ctx, "host:pack_to_host");
        s = pack_to_host(ctx, A, n, o, out, stats, vout ? &pd : nullptr);
    }
    if (s == PHR_OK && vout) {
        HostScope hs(ctx, "host:variants");
        s = variants_to_host(ctx, A, n, idx, o, pd, cfg, vcfg, vout);
    }
    if (ctx->timing) ctx->resolve_timings();
    return s;
}

}  // namespace phr

phr_index::~phr_index() {
    if (d_rep) cudaFree(d_rep);
    if (d_block) cudaFree(d_block);
    if (d_target) cudaFree(d_target);
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

phr_status phr_index_create(phr_ctx* c, const uint8_t* target, uint64_t target_len, const phr_sketch* sketch,
                            phr_alphabet alphabet, phr_index** out) {
    if (!c || !out || (!target && target_len)) return PHR_ERR_ARG;
    if (alphabet != PHR_ALPHABET_DNA && alphabet != PHR_ALPHABET_PROTEIN) return PHR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->impl.mu);
    cudaSetDevice(c->impl.device);
    *out = nullptr;
    return phr::index_create(&c->impl, target, target_len, sketch, alphabet, out);
}

void phr_index_destroy(phr_index* idx) {
    if (!idx) return;
    cudaSetDevice(idx->ctx->device);
    delete idx;
}

phr_status phr_index_get_info(const phr_index* idx, phr_index_info* info) {
    if (!idx || !info) return PHR_ERR_ARG;
    info->n_minimizers = idx->n_min;
    info->n_distinct = idx->n_distinct;
    info->occurrence_cap = idx->view.occ_cap;
    info->target_len = idx->target_len;
    info->device_bytes = idx->device_bytes;
    return PHR_OK;
}

phr_status phr_sketch_batch(phr_ctx* c, const phr_seq_batch* seqs, int32_t k, int32_t w, phr_alphabet alphabet,
                            const uint64_t* out_off, uint64_t* values, uint32_t* positions, uint32_t* out_n) {
    if (!c || !seqs || !out_off || !values || !positions || !out_n) return PHR_ERR_ARG;
    phr::Ctx* ctx = &c->impl;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (k <= 0 || w <= 0 || k > 32) return phr::set_error(ctx, PHR_ERR_ARG, "k must be in 1..32, w >= 1");
    const uint64_t n = seqs->n;
    if (n == 0) return PHR_OK;
    uint64_t cap_total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (seqs->off[i] + seqs->len[i] > seqs->seq_bytes) return phr::set_error(ctx, PHR_ERR_ARG, "sequence past seq_bytes");
        const uint64_t kc = seqs->len[i] >= static_cast<uint32_t>(k) ? seqs->len[i] - k + 1 : 0;
        cap_total = std::max(cap_total, out_off[i] + kc);
    }
    cudaStream_t st = ctx->stream;
    phr::DeviceArena& A = ctx->pipe;
    A.reset();
    PHR_CUDA_TRY(ctx, A.reserve(seqs->seq_bytes * 40 + cap_total * 12 + n * 64 + (64 << 20)));
    uint8_t* d_seq = static_cast<uint8_t*>(A.take(seqs->seq_bytes + 64));
    uint64_t* d_off = static_cast<uint64_t*>(A.take(n * 8));
    uint32_t* d_len = static_cast<uint32_t*>(A.take(n * 4));
    uint64_t* d_oo = static_cast<uint64_t*>(A.take(n * 8));
    uint64_t* d_val = static_cast<uint64_t*>(A.take(cap_total * 8 + 8));
    uint32_t* d_pos = static_cast<uint32_t*>(A.take(cap_total * 4 + 8));
    uint32_t* d_n = static_cast<uint32_t*>(A.take(n * 4 + 8));
    if (!d_n) return phr::set_error(ctx, PHR_ERR_OOM, "arena exhausted");
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_seq, seqs->seq, seqs->seq_bytes, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_off, seqs->off, n * 8, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_len, seqs->len, n * 4, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_oo, out_off, n * 8, cudaMemcpyHostToDevice, st));
    uint64_t* skoff = nullptr;
    uint64_t total = 0;
    phr_status s = phr::sketch_device(ctx, A, d_seq, d_off, d_len, n, k, w, alphabet, &d_val, &d_pos, &skoff, &d_n,
                                      &total, d_oo);
    if (s != PHR_OK) return s;
    if (cap_total) {
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(values, d_val, cap_total * 8, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(positions, d_pos, cap_total * 4, cudaMemcpyDeviceToHost, st));
    }
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(out_n, d_n, n * 4, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (ctx->timing) ctx->resolve_timings();
    return PHR_OK;
}

phr_status phr_seed_chain_batch(phr_ctx* c, const phr_index* idx, const phr_sketch* sketches, uint64_t n,
                                phr_chain_arena* out) {
    if (!c || !idx || (!sketches && n) || !out || !out->n_seeds_found || !out->n_chains || !out->chain_off ||
        (!out->chains && out->chain_capacity) || (!out->seeds && out->seed_capacity))
        return PHR_ERR_ARG;
    phr::Ctx* ctx = &c->impl;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (n == 0) return PHR_OK;
    std::vector<uint64_t> h_off(n), vals;
    std::vector<uint32_t> h_n(n), poss;
    for (uint64_t i = 0; i < n; ++i) {
        h_off[i] = vals.size();
        h_n[i] = static_cast<uint32_t>(sketches[i].n);
        if (sketches[i].n && (!sketches[i].values || !sketches[i].positions))
            return phr::set_error(ctx, PHR_ERR_ARG, "sketch arrays are NULL");
        vals.insert(vals.end(), sketches[i].values, sketches[i].values + sketches[i].n);
        poss.insert(poss.end(), sketches[i].positions, sketches[i].positions + sketches[i].n);
    }
    cudaStream_t st = ctx->stream;
    phr::DeviceArena& A = ctx->pipe;
    A.reset();
    PHR_CUDA_TRY(ctx, A.reserve(vals.size() * 64 + n * 256 + (64 << 20)));
    uint64_t* d_val = static_cast<uint64_t*>(A.take(vals.size() * 8 + 8));
    uint32_t* d_pos = static_cast<uint32_t*>(A.take(poss.size() * 4 + 8));
    uint64_t* d_off = static_cast<uint64_t*>(A.take(n * 8));
    uint32_t* d_n = static_cast<uint32_t*>(A.take(n * 4));
    if (!d_n) return phr::set_error(ctx, PHR_ERR_OOM, "arena exhausted");
    if (!vals.empty()) {
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_val, vals.data(), vals.size() * 8, cudaMemcpyHostToDevice, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_pos, poss.data(), poss.size() * 4, cudaMemcpyHostToDevice, st));
    }
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_off, h_off.data(), n * 8, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(d_n, h_n.data(), n * 4, cudaMemcpyHostToDevice, st));
    phr::ChainResult C;
    phr_status s = phr::seed_chain_device(ctx, A, idx, d_val, d_pos, d_off, d_n, n, &C);
    if (s != PHR_OK) return s;
    const uint64_t T = C.total_seeds;
    std::vector<uint32_t> nseeds(n), nch(n);
    std::vector<uint64_t> soff(n + 1);
    std::vector<int64_t> score(T + 1);
    std::vector<uint32_t> first(T + 1), len(T + 1), tstart(T + 1);
    std::vector<uint64_t> skey(T + 1), smin(T + 1);
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(nseeds.data(), C.nseeds, n * 4, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(nch.data(), C.nchains, n * 4, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(soff.data(), C.seed_off, (n + 1) * 8, cudaMemcpyDeviceToHost, st));
    if (T) {
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(score.data(), C.ch_score, T * 8, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(first.data(), C.ch_first, T * 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(len.data(), C.ch_len, T * 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(tstart.data(), C.ch_tstart, T * 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(skey.data(), C.ch_seed_key, T * 8, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(smin.data(), C.ch_seed_min, T * 8, cudaMemcpyDeviceToHost, st));
    }
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (ctx->timing) ctx->resolve_timings();
    uint64_t co = 0, so = 0;
    for (uint64_t u = 0; u < n; ++u) {
        out->n_seeds_found[u] = nseeds[u];
        out->n_chains[u] = nch[u];
        out->chain_off[u] = co;
        const uint64_t base = soff[u];
        for (uint32_t cix = 0; cix < nch[u]; ++cix) {
            if (co >= out->chain_capacity) return phr::set_error(ctx, PHR_ERR_CAPACITY, "chain arena too small");
            phr_chain& ch = out->chains[co++];
            ch.score = score[base + cix];
            ch.seed_off = static_cast<uint32_t>(so);
            ch.n_seeds = len[base + cix];
            ch.target_start = tstart[base + cix];
            ch._pad = 0;
            for (uint32_t k = 0; k < ch.n_seeds; ++k) {
                if (so >= out->seed_capacity) return phr::set_error(ctx, PHR_ERR_CAPACITY, "seed arena too small");
                const uint64_t key = skey[base + first[base + cix] + k];
                out->seeds[so].query_pos = static_cast<uint32_t>(key & 0xffffffffu);
                out->seeds[so].target_pos = static_cast<uint32_t>(key >> 32);
                out->seeds[so].minimizer = smin[base + first[base + cix] + k];
                ++so;
            }
        }
    }
    return PHR_OK;
}

phr_status phr_align_reads(phr_ctx* c, const phr_index* idx, const phr_read_batch* reads, const phr_align_config* cfg,
                           phr_read_result_arena* out, phr_align_stats* stats) {
    if (!c || !idx || !reads || !cfg || !out || (reads->n_reads && (!reads->off || !reads->len || !out->reads)))
        return PHR_ERR_ARG;
    phr::Ctx* ctx = &c->impl;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (cfg->strategy < PHR_FAST || cfg->strategy > PHR_SENSITIVE) return phr::set_error(ctx, PHR_ERR_ARG, "strategy");
    return phr::align_reads_host(ctx, idx, reads, *cfg, out, stats, nullptr, nullptr);
}

phr_status phr_align_reads_variants(phr_ctx* c, const phr_index* idx, const phr_read_batch* reads,
                                    const phr_align_config* cfg, phr_read_result_arena* out,
                                    const phr_variant_config* vcfg, phr_variant_arena* vout,
                                    phr_align_stats* stats) {
    if (!c || !idx || !reads || !cfg || !out || !vout || !vout->read_variant_off ||
        (reads->n_reads && (!reads->off || !reads->len || !out->reads)))
        return PHR_ERR_ARG;
    if (vcfg && vcfg->n_hotspots && (!vcfg->hotspot_start || !vcfg->hotspot_end)) return PHR_ERR_ARG;
    phr::Ctx* ctx = &c->impl;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (cfg->strategy < PHR_FAST || cfg->strategy > PHR_SENSITIVE) return phr::set_error(ctx, PHR_ERR_ARG, "strategy");
    vout->variant_used = vout->coverage_used = vout->allele_used = 0;
    if (reads->n_reads == 0) {
        vout->read_variant_off[0] = 0;
        out->aln_used = out->cigar_used = 0;
        return PHR_OK;
    }
    return phr::align_reads_host(ctx, idx, reads, *cfg, out, stats, vcfg, vout);
}

struct phr_coverage {
    phr::Ctx* ctx = nullptr;
    uint64_t tlen = 0;
    int depth = 0;
    uint32_t* d_track = nullptr;
    phr_alignment* d_aln = nullptr;
    uint64_t aln_cap = 0;
};

phr_status phr_coverage_create(phr_ctx* c, const phr_index* idx, phr_coverage_mode mode, phr_coverage** out) {
    if (!c || !idx || !out || (mode != PHR_COVERAGE_QUANTIZED && mode != PHR_COVERAGE_DEPTH)) return PHR_ERR_ARG;
    phr::Ctx* ctx = &c->impl;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    phr_coverage* cv = new phr_coverage();
    cv->ctx = ctx;
    cv->tlen = idx->target_len;
    cv->depth = mode == PHR_COVERAGE_DEPTH;
    cudaError_t e = cudaMalloc(&cv->d_track, cv->tlen * 4 + 16);
    if (e == cudaSuccess) e = cudaMemsetAsync(cv->d_track, 0, cv->tlen * 4 + 16, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        if (cv->d_track) cudaFree(cv->d_track);
        delete cv;
        return phr::cuda_status(ctx, e, "coverage track");
    }
    *out = cv;
    return PHR_OK;
}

phr_status phr_coverage_add(phr_coverage* cv, const phr_alignment* aln, uint64_t n_aln) {
    if (!cv || (n_aln && !aln)) return PHR_ERR_ARG;
    if (n_aln == 0) return PHR_OK;
    phr::Ctx* ctx = cv->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    if (n_aln > cv->aln_cap) {
        if (cv->d_aln) cudaFree(cv->d_aln);
        cv->d_aln = nullptr;
        cv->aln_cap = 0;
        PHR_CUDA_TRY(ctx, cudaMalloc(&cv->d_aln, n_aln * sizeof(phr_alignment)));
        cv->aln_cap = n_aln;
    }
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(cv->d_aln, aln, n_aln * sizeof(phr_alignment), cudaMemcpyHostToDevice, st));
    {
        phr::KernelScope ks(ctx, "coverage_add");
        phr::coverage_add_kernel<<<phr::blocks_for(n_aln * 32, 256), 256, 0, st>>>(cv->d_aln, n_aln, cv->tlen,
                                                                                  cv->depth, cv->d_track);
    }
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return PHR_OK;
}

phr_status phr_coverage_read(phr_coverage* cv, uint32_t* track, uint64_t len) {
    if (!cv || (len && !track) || len != cv->tlen) return PHR_ERR_ARG;
    phr::Ctx* ctx = cv->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (len) PHR_CUDA_TRY(ctx, cudaMemcpy(track, cv->d_track, len * 4, cudaMemcpyDeviceToHost));
    return PHR_OK;
}

void phr_coverage_destroy(phr_coverage* cv) {
    if (!cv) return;
    cudaSetDevice(cv->ctx->device);
    if (cv->d_aln) cudaFree(cv->d_aln);
    if (cv->d_track) cudaFree(cv->d_track);
    delete cv;
}

phr_status phr_index_repeat_regions(const phr_index* idx, uint32_t* start, uint32_t* end, uint64_t cap, uint64_t* n) {
    if (!idx || !n || (cap && (!start || !end))) return PHR_ERR_ARG;
    const uint64_t nr = idx->rep_start.size();
    const uint64_t k = std::min(nr, cap);
    if (k) {
        std::memcpy(start, idx->rep_start.data(), k * 4);
        std::memcpy(end, idx->rep_end.data(), k * 4);
    }
    *n = nr;
    return PHR_OK;
}

}  // extern "C"
