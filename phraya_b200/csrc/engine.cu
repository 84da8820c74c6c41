// engine.cu -- extension batch driver: pair preparation (suffixes, 2-bit packing),
// length-bucketed task lists, persistent-kernel launches with overflow redo passes,
// and packing of the CIGAR text into the caller's arena.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_set>

#include "engine.cuh"

namespace phr {

// ---------------------------------------------------------------------------
// DeviceArena
// ---------------------------------------------------------------------------
cudaError_t DeviceArena::reserve(size_t need) {
    if (need <= cap) return cudaSuccess;
    auto alloc = [&](size_t bytes) -> cudaError_t {
        void* p = nullptr;
        cudaError_t e = stream ? cudaMallocAsync(&p, bytes, stream) : cudaMalloc(&p, bytes);
        base = static_cast<char*>(p);
        return e;
    };
    if (base) {
        if (stream)
            cudaFreeAsync(base, stream);
        else
            cudaFree(base);
    }
    base = nullptr;
    cap = 0;
    size_t want = std::max(need + need / 4, static_cast<size_t>(64) << 20);
    cudaError_t e = alloc(want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = alloc(need);
        if (e != cudaSuccess) {
            base = nullptr;
            return e;
        }
        want = need;
    }
    cap = want;
    used = 0;
    return cudaSuccess;
}

void Ctx::bind_stream() {
    for (DeviceArena* a : {&arena, &scratch, &io, &pipe, &seeds}) a->stream = stream;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
}

void* DeviceArena::take(size_t bytes, size_t align) {
    size_t off = (used + align - 1) / align * align;
    if (off + bytes > cap) return nullptr;
    used = off + bytes;
    return base + off;
}

DeviceArena::~DeviceArena() {
    if (base) cudaFree(base);
}

void Ctx::begin_kernel(const char* name, cudaEvent_t* a) {
    if (cudaEventCreate(a) != cudaSuccess) {
        *a = nullptr;
        return;
    }
    cudaEventRecord(*a, stream);
}

void Ctx::end_kernel(const char* name, cudaEvent_t a) {
    cudaEvent_t b;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return;
    }
    cudaEventRecord(b, stream);
    pending.push_back({name, a, b});
}

void Ctx::resolve_timings() {
    for (auto& p : pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            auto& t = timings[p.name];
            t.first += 1;
            t.second += ms;
        }
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    pending.clear();
}

Ctx::~Ctx() {
    for (auto& p : pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    if (d_counters) cudaFree(d_counters);
    if (h_pinned) cudaFreeHost(h_pinned);
    if (copy_in) cudaStreamDestroy(copy_in);
    if (copy_out) cudaStreamDestroy(copy_out);
    if (stream) cudaStreamDestroy(stream);
}

phr_status set_error(Ctx* ctx, phr_status st, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return st;
}

phr_status cuda_status(Ctx* ctx, cudaError_t e, const char* what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return set_error(ctx, PHR_ERR_OOM, msg);
    return set_error(ctx, PHR_ERR_CUDA, msg);
}

namespace {

constexpr uint32_t kInvalidKey = 0xFFFFFFFFu;

__device__ __forceinline__ int next_pow2_cap32(int v) {
    int g = 1;
    while (g < v && g < 32) g <<= 1;
    return g;
}

struct PrepParams {
    DevPairs in;
    int32_t engine;
    phr_affine_costs costs;
    PairDesc* desc;
    PairOut* out;
    uint64_t* w2;      // 2-bit words per pair -> scanned in place to offsets
    uint64_t* wb;      // byte words per pair
    uint64_t* tb;      // text bound per pair
};

// Suffix lengths, seed validation, arena sizes. One thread per pair.
__global__ void prep_sizes_kernel(PrepParams P) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= P.in.n) return;
    const uint32_t ql = P.in.q_len[i], tl = P.in.t_len[i];
    uint32_t qs = P.in.q_seed ? P.in.q_seed[i] : 0, ts = P.in.t_seed ? P.in.t_seed[i] : 0;
    if (P.engine == PHR_ENGINE_MYERS_GLOBAL) qs = ts = 0;
    PairDesc d = {};
    const bool invalid = qs > ql || ts > tl;
    d.qs = static_cast<int32_t>(qs);
    d.ts = static_cast<int32_t>(ts);
    d.qn = invalid ? 0 : static_cast<int32_t>(ql - qs);
    d.tn = invalid ? 0 : static_cast<int32_t>(tl - ts);
    d.trivial = (invalid || d.qn == 0 || d.tn == 0) ? 1 : 0;
    d.mode = 0;
    P.desc[i] = d;
    PairOut o = {};
    o.status = invalid ? PHR_INVALID_INPUT : -1;  // -1: not yet produced
    P.out[i] = o;
    const uint64_t qn = d.qn, tn = d.tn;
    P.w2[i] = d.trivial ? 0 : (qn + 15) / 16 + 4 + (tn + 15) / 16 + 4;
    P.wb[i] = d.trivial ? 0 : (qn + 3) / 4 + 4 + (tn + 3) / 4 + 4;
    P.tb[i] = 2 * (qn + tn) + 16;
}

__device__ __forceinline__ uint32_t code2(uint8_t b, bool& pure) {
    switch (b) {
        case 'A': return 0;
        case 'C': return 1;
        case 'G': return 2;
        case 'T': return 3;
        default: pure = false; return 0;
    }
}

// The first `keep` (0..4) of four ASCII bytes -> their 2-bit codes (A, C, G, T = 0..3) in
// the low 8 bits (the other bytes' codes are zero); `pure` turns false unless those bytes
// are all A, C, G or T. The code of A/C/G/T is bits 1-2 of the byte XOR bits 2-3 (0x41,
// 0x43, 0x47, 0x54 -> 0, 1, 2, 3); a byte is one of them exactly when the letter of its
// code ('A', 'C', 'G', 'T' picked by one byte permute) is the byte itself.
__device__ __forceinline__ uint32_t code2x4m(uint32_t x, int keep, bool& pure) {
    const uint32_t bytes = keep >= 4 ? 0xFFFFFFFFu : (1u << (8 * keep)) - 1u;
    const uint32_t c = ((x >> 1) ^ (x >> 2)) & 0x03030303u;
    const uint32_t sel = (c & 0x3u) | ((c >> 4) & 0x30u) | ((c >> 8) & 0x300u) | ((c >> 12) & 0x3000u);
    if (((__byte_perm(0x54474341u, 0u, sel) ^ x) & bytes) != 0) pure = false;
    uint32_t cm = c & bytes;
    cm |= cm >> 6;
    cm |= cm >> 12;
    return cm & 0xFFu;
}

// Writes "<n><op>" at p, returns its length.
__device__ uint32_t write_count_op(char* p, uint32_t n, char op) {
    const uint32_t nd = ndigits(n);
    for (int d = static_cast<int>(nd) - 1; d >= 0; --d) {
        p[d] = static_cast<char>('0' + n % 10);
        n /= 10;
    }
    p[nd] = op;
    return nd + 1;
}

struct PackParams {
    DevPairs in;
    int32_t engine;
    phr_affine_costs costs;
    PairDesc* desc;
    PairOut* out;
    const uint64_t* w2_off;
    const uint64_t* wb_off;
    const uint64_t* text_off;
    uint32_t* arena2;
    uint32_t* arenab;
    char* text;
    uint32_t* keys;
    uint32_t* vals;
    int wfa_g_short, wfa_g_long;
    int wfa_long_min;   // qn + tn from which a WFA pair gets wfa_g_long lanes
    int band_base;      // Myers band half-width base
};

// 2-bit packing (16 bases per word) of both suffixes; a pair holding any byte other
// than A/C/G/T is also copied word-aligned to the byte arena and runs the byte path.
// Trivial pairs (an empty suffix) get their final result here. One warp per pair.
__global__ void pack_kernel(PackParams P) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= P.in.n) return;
    const uint64_t i = warp;
    PairDesc d = P.desc[i];
    if (d.trivial) {
        if (lane == 0) {
            PairOut o = P.out[i];
            P.keys[i] = kInvalidKey;
            P.vals[i] = static_cast<uint32_t>(i);
            if (o.status == PHR_INVALID_INPUT) {
                o.ed = 0;
                o.t_consumed = 0;
                o.text_len = 0;
                P.out[i] = o;
                return;
            }
            char* t = P.text + P.text_off[i];
            uint32_t len = 0;
            o.status = PHR_OK;
            o.affine_score = 0;
            const int qn = d.qn, tn = d.tn;
            if (P.engine == PHR_ENGINE_MYERS_GLOBAL) {
                if (qn == 0) {
                    o.ed = tn;
                    if (tn > 0) len = write_count_op(t, tn, 'I');
                } else {
                    o.ed = qn;
                    len = write_count_op(t, qn, 'D');
                }
                o.t_consumed = tn;
            } else if (qn == 0) {
                o.ed = 0;  // wfa_simd.rs:194-203 / :365-367 / :592-601, :3793-3795
                o.t_consumed = 0;
            } else {      // tn == 0: every query base is query-extra
                o.ed = qn;
                len = write_count_op(t, qn, 'D');
                o.t_consumed = 0;
                if (P.engine == PHR_ENGINE_WFA_AFFINE) o.affine_score = P.costs.gap_open + qn * P.costs.gap_extend;
            }
            o.n_runs = len ? 1 : 0;
            o.text_len = len;
            P.out[i] = o;
        }
        return;
    }
    const uint8_t* qsrc = P.in.seq + P.in.q_off[i] + d.qs;
    const uint8_t* tsrc = (P.in.t_seq ? P.in.t_seq : P.in.seq) + P.in.t_off[i] + d.ts;
    const uint64_t w2 = P.w2_off[i];
    const uint64_t q2w = (d.qn + 15) / 16 + 4;
    bool pure = true;
    // bytes a lane may read with aligned 32-bit loads: those of the batch arena (targets
    // from a separate arena take the byte loop)
    const uintptr_t ok_lo = reinterpret_cast<uintptr_t>(P.in.seq);
    const uintptr_t ok_hi = ok_lo + P.in.seq_bytes;
    // query words then target words, dealt to the warp's lanes as one list
    const int nwq = (d.qn + 15) / 16, nwt = (d.tn + 15) / 16;
    for (int x = lane; x < nwq + nwt; x += 32) {
        const int side = x >= nwq;
        const int w = side ? x - nwq : x;
        const uint8_t* src = side ? tsrc : qsrc;
        const bool wide = !(side && P.in.t_seq);
        const int len = side ? d.tn : d.qn;
        uint32_t* dst = P.arena2 + w2 + (side ? q2w : 0);
        uint32_t word = 0;
        const int p0 = w * 16;
        const int lim = min(16, len - p0);
        const uint8_t* cp = src + p0;
        const uintptr_t a0 = reinterpret_cast<uintptr_t>(cp) & ~static_cast<uintptr_t>(3);
        if (wide && a0 >= ok_lo && a0 + 20 <= ok_hi) {
            // 16 bases from five aligned words, four bases per step; in the last word of a
            // sequence the bytes past its end are read (inside the arena) but neither
            // coded nor checked
            const uint32_t* wp = reinterpret_cast<const uint32_t*>(a0);
            const uint32_t sh = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(cp) & 3) * 8;
            uint32_t v[5];
#pragma unroll
            for (int j = 0; j < 5; ++j) v[j] = __ldg(wp + j);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int keep = min(max(lim - 4 * j, 0), 4);  // bytes of this group inside the sequence
                word |= code2x4m(__funnelshift_r(v[j], v[j + 1], sh), keep, pure) << (8 * j);
            }
        } else {
            for (int b = 0; b < lim; ++b) word |= code2(cp[b], pure) << (2 * b);
        }
        dst[w] = word;
    }
    pure = __all_sync(PHR_FULL_MASK, pure);
    if (pure) {
        d.mode = 0;
        d.q_word = w2;
        d.t_word = w2 + q2w;
    } else {
        const uint64_t wb = P.wb_off[i];
        const uint64_t qbw = (d.qn + 3) / 4 + 4;
        for (int side = 0; side < 2; ++side) {
            const uint8_t* src = side ? tsrc : qsrc;
            const int len = side ? d.tn : d.qn;
            uint32_t* dst = P.arenab + wb + (side ? qbw : 0);
            const int nw = (len + 3) / 4;
            for (int w = lane; w < nw; w += 32) {
                uint32_t word = 0;
                const int p0 = w * 4;
                const int lim = min(4, len - p0);
                for (int b = 0; b < lim; ++b) word |= static_cast<uint32_t>(src[p0 + b]) << (8 * b);
                dst[w] = word;
            }
        }
        d.mode = 1;
        d.q_word = wb;
        d.t_word = wb + qbw;
    }
    if (lane == 0) {
        P.desc[i] = d;
        int G;
        uint32_t len;
        if (P.engine == PHR_ENGINE_MYERS_FIT || P.engine == PHR_ENGINE_MYERS_GLOBAL) {
            G = next_pow2_cap32((d.qn + 63) / 64);
            // global 2-bit pairs whose band fits the lane kernel's window: one lane each
            if (P.engine == PHR_ENGINE_MYERS_GLOBAL && d.mode == 0) {
                const LaneBand b = lane_band(d.qn, d.tn, P.band_base);
                if (lane_slots(b.dmin, b.dmax, (d.qn + 63) / 64) <= kLaneMaxSlots - 2) G = 1;
            }
            len = static_cast<uint32_t>(d.tn) * (static_cast<uint32_t>((d.qn + 63) / 64));
        } else {
            G = (d.qn + d.tn < P.wfa_long_min) ? P.wfa_g_short : P.wfa_g_long;
            len = static_cast<uint32_t>(d.qn + d.tn);
        }
        const uint32_t glog = static_cast<uint32_t>(__ffs(G) - 1);
        const uint32_t lk = 0x0FFFFFFFu - min(len, 0x0FFFFFFFu);  // longest first within a bucket
        P.keys[i] = (static_cast<uint32_t>(d.mode) << 31) | (glog << 28) | lk;
        P.vals[i] = static_cast<uint32_t>(i);
    }
}

struct TaskBuild {
    const uint32_t* keys;      // sorted
    const uint32_t* order;     // sorted pair ids
    uint64_t n;
    uint32_t* head;            // scratch: segment head positions
    uint32_t* flag;
    uint32_t* tidx;
    uint32_t* task_first;
    uint8_t* task_count;
    uint8_t* task_group;
    uint32_t* ranges;          // {0, split, split, n_tasks}
    uint32_t* split_min;
    uint32_t* g1_min;          // first 2-bit task of more than one lane per pair
    const PairDesc* desc;
    int32_t engine;
    int32_t band_base;
    unsigned long long* need_max;
    uint64_t* task_need;          // per task
    unsigned int* need_hist;      // 64 buckets by bit length of the need
    int32_t big_min;              // linear WFA pairs for the CTA-per-pair kernel (not in the
    uint32_t big_smem;            // main pass, so not in its slot statistics)
    int32_t lane_ckpt;            // lane kernel mode (its scratch need)
};

__device__ __forceinline__ int key_group(uint32_t k) { return 1 << ((k >> 28) & 7); }
__device__ __forceinline__ uint32_t key_seg(uint32_t k) { return k >> 28; }

__global__ void task_head_kernel(TaskBuild T) {
    const uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (p >= T.n) return;
    const uint32_t k = T.keys[p];
    T.head[p] = (p == 0 || key_seg(T.keys[p - 1]) != key_seg(k)) ? static_cast<uint32_t>(p) : 0u;
}

__global__ void task_flag_kernel(TaskBuild T) {
    const uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (p >= T.n) return;
    const uint32_t k = T.keys[p];
    const uint32_t per = 32 / key_group(k);
    T.flag[p] = (k != kInvalidKey && ((p - T.head[p]) % per) == 0) ? 1u : 0u;
}

__device__ __forceinline__ uint64_t myers_need_est(int m, int n, int G, int band_base) {
    const int nb = (m + 63) >> 6;
    int E = min(band_base + abs(m - n) + (m >> 4), max(m, n));
    int W = min((2 * (E + 2) + 1 + 63) / 64 + 1, nb);
    uint64_t need = ((static_cast<uint64_t>(n) * W * 16) + 15) & ~15ull;  // 16-byte VP/HP records
    if (nb > G) need += (static_cast<uint64_t>(n) + 15) & ~15ull;
    need += (static_cast<uint64_t>(m + n + 2) * 4 + 15) & ~15ull;
    return need;
}

__global__ void task_fill_kernel(TaskBuild T) {
    const uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    // every lane stays to the warp-level reductions at the end; lanes without a task
    // contribute nothing to them
    const bool has_task = p < T.n && T.flag[p];
    uint64_t need = 0;
    uint32_t t_split = 0xFFFFFFFFu, t_g1 = 0xFFFFFFFFu;
    if (has_task) {
        const uint32_t k = T.keys[p];
        const int G = key_group(k);
        const uint32_t per = 32 / G;
        uint32_t cnt = 0;
        uint64_t region = 0;
        // lane-kernel tasks (global Myers, 2-bit, one lane per pair): window over the union band
        const bool lane_task = T.engine == PHR_ENGINE_MYERS_GLOBAL && G == 1 && !((k >> 31) & 1);
        int dmin = 0x7fffffff, dmax = static_cast<int>(0x80000000), n_max = 0, m_max = 0;
        for (uint32_t c = 0; c < per && p + c < T.n; ++c) {
            const uint32_t kc = T.keys[p + c];
            if (kc == kInvalidKey || key_seg(kc) != key_seg(k)) break;
            const PairDesc d = T.desc[T.order[p + c]];
            if (lane_task) {
                const LaneBand b = lane_band(d.qn, d.tn, T.band_base);
                dmin = min(dmin, b.dmin);
                dmax = max(dmax, b.dmax);
                n_max = max(n_max, d.tn);
                m_max = max(m_max, d.qn);
            } else if (T.engine == PHR_ENGINE_MYERS_FIT || T.engine == PHR_ENGINE_MYERS_GLOBAL)
                need += myers_need_est(d.qn, d.tn, G, T.band_base);
            else if (!big_pair(T.engine, T.big_min, T.big_smem, d.qn, d.tn, d.mode))
                region = max(region, wfa_region_est(d.qn, d.tn, T.engine == PHR_ENGINE_WFA_AFFINE));
            ++cnt;
        }
        if (T.engine != PHR_ENGINE_MYERS_FIT && T.engine != PHR_ENGINE_MYERS_GLOBAL) need = region * per;
        if (lane_task && cnt) need = lane_task_need(n_max, m_max, lane_slots(dmin, dmax, (m_max + 63) >> 6), T.lane_ckpt);
        const uint32_t t = T.tidx[p];
        T.task_first[t] = static_cast<uint32_t>(p);
        T.task_count[t] = static_cast<uint8_t>(cnt);
        T.task_group[t] = static_cast<uint8_t>(G);
        T.task_need[t] = need;
        if ((k >> 31) & 1) t_split = t;
        else if (G > 1) t_g1 = t;
    }
    // one atomic per warp and value instead of one per task (a million tasks would
    // otherwise queue on the same three addresses)
    uint64_t nmax = need;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(PHR_FULL_MASK, nmax, o));
    t_split = __reduce_min_sync(PHR_FULL_MASK, t_split);
    t_g1 = __reduce_min_sync(PHR_FULL_MASK, t_g1);
    const int bucket = need ? 64 - __clzll(need) : 64;   // 64: no histogram entry
    const uint32_t same = __match_any_sync(PHR_FULL_MASK, bucket);
    const int lane = threadIdx.x & 31;
    if (bucket < 64 && lane == __ffs(same) - 1) atomicAdd(&T.need_hist[bucket], static_cast<unsigned>(__popc(same)));
    if (lane == 0) {
        if (nmax) atomicMax(T.need_max, static_cast<unsigned long long>(nmax));
        if (t_split != 0xFFFFFFFFu) atomicMin(T.split_min, t_split);
        if (t_g1 != 0xFFFFFFFFu) atomicMin(T.g1_min, t_g1);
    }
}

__global__ void task_finalize_kernel(TaskBuild T) {
    uint32_t nt = 0;
    if (T.n > 0) nt = T.tidx[T.n - 1] + T.flag[T.n - 1];
    const uint32_t split = min(*T.split_min, nt);
    T.ranges[0] = 0;
    T.ranges[1] = split;
    T.ranges[2] = split;
    T.ranges[3] = nt;
    // lane-kernel range {0, g1} and warp-group 2-bit range {g1, split} (global Myers)
    const uint32_t g1 = min(*T.g1_min, split);
    T.ranges[28] = 0;
    T.ranges[29] = g1;
    T.ranges[30] = g1;
    T.ranges[31] = split;
}

// Redo pass task list: one pair per task, in redo order.
__global__ void redo_tasks_kernel(const uint32_t* redo_list, const uint32_t* redo_count, const PairDesc* desc,
                                  int32_t engine, int wfa_g_short, int wfa_g_long, int wfa_long_min, int32_t big_min,
                                  uint32_t big_smem, uint32_t* task_first, uint8_t* task_count,
                                  uint8_t* task_group, uint32_t* ranges) {
    const uint32_t n = *redo_count;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        ranges[0] = 0;
        ranges[1] = n;
    }
    if (t >= n) return;
    const PairDesc d = desc[redo_list[t]];
    int G;
    if (engine == PHR_ENGINE_MYERS_FIT || engine == PHR_ENGINE_MYERS_GLOBAL)
        G = next_pow2_cap32((d.qn + 63) / 64);
    else
        G = (d.qn + d.tn < wfa_long_min) ? wfa_g_short : wfa_g_long;
    task_first[t] = t;
    task_count[t] = 1;
    task_group[t] = static_cast<uint8_t>(G);
    if (big_pair(engine, big_min, big_smem, d.qn, d.tn, d.mode)) task_group[t] = kBigTask | 32;
}

struct FinishParams {
    uint64_t n;
    int32_t engine;
    const PairDesc* desc;
    const PairOut* out;
    const uint64_t* text_off;
    const char* text;
    uint64_t* cig_off;       // exclusive scan of text_len
    phr_alignment* aln;
    char* cigar;
    uint64_t cigar_capacity;
    uint32_t* error_flag;
    uint64_t cigar_base;
};

__global__ void text_len_kernel(const PairOut* out, uint64_t n, uint64_t* len) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const PairOut o = out[i];
    len[i] = (o.status == PHR_OK) ? o.text_len : 0;
}

// Packs CIGAR text and writes the phr_alignment records. One warp per 32 consecutive
// pairs: lane l writes pair first + l's record (the warp's records are contiguous), then
// the lanes copy the pairs' texts one pair after the other.
__global__ void finish_kernel(FinishParams F) {
    const uint64_t first = ((blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5) * 32;
    const int lane = threadIdx.x & 31;
    if (first >= F.n) return;
    const uint64_t i = first + lane;
    uint64_t off = 0, toff = 0;
    uint32_t len = 0;
    bool copy = false;
    if (i < F.n) {
        const PairOut o = F.out[i];
        if (o.status == -1) {
            atomicOr(F.error_flag, 8u);
        } else {
            const PairDesc d = F.desc[i];
            off = F.cig_off[i];
            toff = F.text_off[i];
            len = (o.status == PHR_OK) ? o.text_len : 0;
            copy = off + len <= F.cigar_capacity;
            if (!copy) atomicOr(F.error_flag, 16u);
            phr_alignment a;
            a.status = o.status;
            a.edit_distance = o.status == PHR_OK ? static_cast<uint32_t>(o.ed) : 0;
            a.cigar_off = F.cigar_base + off;
            a.cigar_len = len;
            a.affine_score = o.status == PHR_OK ? static_cast<uint32_t>(o.affine_score) : 0;
            if (F.engine == PHR_ENGINE_MYERS_GLOBAL) {
                a.query_start = 0;
                a.query_end = static_cast<uint32_t>(d.qn);
                a.target_start = 0;
                a.target_end = static_cast<uint32_t>(d.tn);
            } else if (o.status != PHR_OK) {
                a.query_start = a.query_end = a.target_start = a.target_end = 0;
            } else {
                a.query_start = static_cast<uint32_t>(d.qs);
                a.query_end = static_cast<uint32_t>(d.qs + d.qn);
                a.target_start = static_cast<uint32_t>(d.ts);
                a.target_end = static_cast<uint32_t>(d.ts + o.t_consumed);
            }
            F.aln[i] = a;
        }
    }
    const unsigned todo = __ballot_sync(PHR_FULL_MASK, copy && len > 0);
    for (unsigned m = todo; m; m &= m - 1) {
        const int j = __ffs(m) - 1;
        const uint32_t lj = __shfl_sync(PHR_FULL_MASK, len, j);
        const uint64_t oj = __shfl_sync(PHR_FULL_MASK, off, j);
        const uint64_t tj = __shfl_sync(PHR_FULL_MASK, toff, j);
        for (uint32_t c = lane; c < lj; c += 32) F.cigar[oj + c] = F.text[tj + c];
    }
}

__global__ void total_kernel(const uint64_t* off, const uint64_t* len, uint64_t n, uint64_t* total) {
    *total = n ? off[n - 1] + len[n - 1] : 0;
}

inline unsigned blocks_for(uint64_t n, unsigned t) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

namespace {
__global__ void sum_lengths_kernel(const uint32_t* a, const uint32_t* b, uint64_t n, unsigned long long* out) {
    unsigned long long acc = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        acc += static_cast<unsigned long long>(a[i]) + b[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(PHR_FULL_MASK, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}
}  // namespace

uint64_t device_length_sum(Ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n, cudaError_t* err) {
    *err = cudaSuccess;
    if (!ctx->d_counters) {
        *err = cudaMalloc(&ctx->d_counters, 256);
        if (*err != cudaSuccess) return 0;
    }
    if (!ctx->h_pinned) {
        *err = cudaMallocHost(&ctx->h_pinned, 256);
        if (*err != cudaSuccess) return 0;
    }
    unsigned long long* d = reinterpret_cast<unsigned long long*>(ctx->d_counters);
    unsigned long long* h = static_cast<unsigned long long*>(ctx->h_pinned);
    cudaStream_t st = ctx->stream;
    if ((*err = cudaMemsetAsync(d, 0, 8, st)) != cudaSuccess) return 0;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4ull * ctx->sm_count));
    {
        KernelScope ks(ctx, "sum_lengths");
        sum_lengths_kernel<<<std::max(1u, grid), 256, 0, st>>>(a, b, n, d);
    }
    if ((*err = cudaMemcpyAsync(h, d, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return 0;
    if ((*err = cudaStreamSynchronize(st)) != cudaSuccess) return 0;
    return *h;
}

size_t extend_arena_need(uint64_t n, uint64_t seq_bytes, uint64_t sum_qt) {
    size_t s = 0;
    auto add = [&](size_t b) { s += (b + 511) / 256 * 256; };
    add(n * sizeof(PairDesc));
    add(n * sizeof(PairOut));
    add(n * 8 * 3);                       // w2, wb, tb (scanned in place)
    add(n * 8 * 3);                       // scan outputs
    add((sum_qt / 16 + 12 * n + 64) * 4);  // 2-bit arena
    add((sum_qt / 4 + 12 * n + 64) * 4);   // byte arena
    add(2 * sum_qt + 16 * n + 64);        // text staging
    add(n * 4 * 4);                       // keys/vals (2x for sort)
    add(n * 4 * 6);                       // task build scratch
    add(n * 6);                           // task count/group
    add(n * 8 * 2);                       // text len + cigar offsets
    add(n * 4);                           // redo list
    add(n * 8 * 4 + 256);                 // task needs, redo needs, redo task offsets/lengths
    add(64ull << 20);                     // CUB temp
    add(4096);
    return s;
}

phr_status run_extend(Ctx* ctx, phr_engine engine, const DevPairs& in, phr_affine_costs costs, DevResults* res,
                      uint64_t sum_qt) {
    const uint64_t n = in.n;
    cudaStream_t st = ctx->stream;
    res->cigar_used = 0;
    if (n == 0) return PHR_OK;
    if (n > 0xFFFFFFF0ull) return set_error(ctx, PHR_ERR_ARG, "too many pairs in one batch");
    HostScope hs_setup(ctx, "host:extend_setup");
    DeviceArena& A = ctx->arena;
    A.reset();
    PHR_CUDA_TRY(ctx, A.reserve(extend_arena_need(n, in.seq_bytes, sum_qt)));
    auto take = [&](size_t b) { return A.take(b); };
    PairDesc* desc = static_cast<PairDesc*>(take(n * sizeof(PairDesc)));
    PairOut* pout = static_cast<PairOut*>(take(n * sizeof(PairOut)));
    uint64_t* w2 = static_cast<uint64_t*>(take(n * 8));
    uint64_t* wb = static_cast<uint64_t*>(take(n * 8));
    uint64_t* tb = static_cast<uint64_t*>(take(n * 8));
    uint64_t* w2o = static_cast<uint64_t*>(take(n * 8));
    uint64_t* wbo = static_cast<uint64_t*>(take(n * 8));
    uint64_t* tbo = static_cast<uint64_t*>(take(n * 8));
    // per sequence ceil(len/16)+4 (2-bit) / ceil(len/4)+4 (byte) words: <= len/16 + 5 per sequence
    uint32_t* arena2 = static_cast<uint32_t*>(take((sum_qt / 16 + 12 * n + 64) * 4));
    uint32_t* arenab = static_cast<uint32_t*>(take((sum_qt / 4 + 12 * n + 64) * 4));
    char* text = static_cast<char*>(take(2 * sum_qt + 16 * n + 64));
    uint32_t* keys = static_cast<uint32_t*>(take(n * 4));
    uint32_t* vals = static_cast<uint32_t*>(take(n * 4));
    uint32_t* keys_s = static_cast<uint32_t*>(take(n * 4));
    uint32_t* order = static_cast<uint32_t*>(take(n * 4));
    uint32_t* head = static_cast<uint32_t*>(take(n * 4));
    uint32_t* head_s = static_cast<uint32_t*>(take(n * 4));
    uint32_t* flag = static_cast<uint32_t*>(take(n * 4));
    uint32_t* tidx = static_cast<uint32_t*>(take(n * 4));
    uint32_t* task_first = static_cast<uint32_t*>(take(n * 4));
    uint32_t* redo_list = static_cast<uint32_t*>(take(n * 4));
    uint8_t* task_count = static_cast<uint8_t*>(take(n));
    uint8_t* task_group = static_cast<uint8_t*>(take(n));
    uint64_t* tlen = static_cast<uint64_t*>(take(n * 8));
    uint64_t* cigoff = static_cast<uint64_t*>(take(n * 8));
    uint64_t* task_need = static_cast<uint64_t*>(take(n * 8));
    unsigned long long* redo_need = static_cast<unsigned long long*>(take(n * 8));
    uint64_t* rtask_off = static_cast<uint64_t*>(take(n * 8));
    uint64_t* rtask_len = static_cast<uint64_t*>(take(n * 8));
    unsigned int* need_hist = static_cast<unsigned int*>(take(64 * 4));
    // counters: [0..3] ranges, [4] split_min, [5] queue head 0, [6] queue head 1,
    // [7] redo count, [8..9] need max (u64), [10] error flag, [12..13] total (u64), [14..17] redo ranges,
    // [20] first multi-lane 2-bit task, [24..25] CTA-kernel queue heads, [26] lane-kernel queue head,
    // [28..31] lane-kernel and warp-group 2-bit ranges (global Myers), [32..39] work counters (u64)
    uint32_t* cnt = static_cast<uint32_t*>(take(256));
    if (!cnt) return set_error(ctx, PHR_ERR_OOM, "device arena exhausted");
    unsigned long long* need_max = reinterpret_cast<unsigned long long*>(cnt + 8);
    uint64_t* total = reinterpret_cast<uint64_t*>(cnt + 12);
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt, 0, 256, st));
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt + 4, 0xFF, 4, st));
    PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt + 20, 0xFF, 4, st));

    // CUB temp sizes
    size_t t_sort = 0, t_scan = 0, t_max = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t_sort, keys, keys_s, vals, order, static_cast<int>(n), 0, 32, st);
    cub::DeviceScan::ExclusiveSum(nullptr, t_scan, w2, w2o, static_cast<int>(n), st);
    cub::DeviceScan::InclusiveScan(nullptr, t_max, head, head_s, cub::Max(), static_cast<int>(n), st);
    size_t t_scan32 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t_scan32, flag, tidx, static_cast<int>(n), st);
    const size_t t_need = std::max({t_sort, t_scan, t_max, t_scan32});
    void* tmp = take(t_need);
    if (!tmp) return set_error(ctx, PHR_ERR_OOM, "device arena exhausted (cub)");

    const unsigned T = 256;
    // lanes per short WFA pair: affine and linear tune separately
    const int g_short = engine == PHR_ENGINE_WFA_AFFINE ? ctx->tune.wfa_affine_group_short : ctx->tune.wfa_group_short;
    PrepParams pp{in, engine, costs, desc, pout, w2, wb, tb};
    {
        KernelScope ks(ctx, "prep_sizes");
        prep_sizes_kernel<<<blocks_for(n, T), T, 0, st>>>(pp);
    }
    size_t tn_ = t_need;
    cub::DeviceScan::ExclusiveSum(tmp, tn_, w2, w2o, static_cast<int>(n), st);
    tn_ = t_need;
    cub::DeviceScan::ExclusiveSum(tmp, tn_, wb, wbo, static_cast<int>(n), st);
    tn_ = t_need;
    cub::DeviceScan::ExclusiveSum(tmp, tn_, tb, tbo, static_cast<int>(n), st);

    PackParams pk{in, engine, costs, desc, pout, w2o, wbo, tbo, arena2, arenab, text, keys, vals,
                  g_short, ctx->tune.wfa_group_long, ctx->tune.wfa_long_min,
                  ctx->tune.myers_band_base};
    {
        KernelScope ks(ctx, "pack");
        pack_kernel<<<blocks_for(n * 32, T), T, 0, st>>>(pk);
    }
    tn_ = t_need;
    cub::DeviceRadixSort::SortPairs(tmp, tn_, keys, keys_s, vals, order, static_cast<int>(n), 0, 32, st);

    PHR_CUDA_TRY(ctx, cudaMemsetAsync(need_hist, 0, 64 * 4, st));
    TaskBuild tbp{keys_s, order, n, head, flag, tidx, task_first, task_count, task_group, cnt, cnt + 4, cnt + 20, desc,
                  engine, ctx->tune.myers_band_base, need_max, task_need, need_hist,
                  ctx->tune.wfa_big_min, static_cast<uint32_t>(ctx->tune.wfa_big_smem), ctx->tune.myers_lane_ckpt};
    {
        KernelScope ks(ctx, "task_head");
        task_head_kernel<<<blocks_for(n, T), T, 0, st>>>(tbp);
    }
    tn_ = t_need;
    cub::DeviceScan::InclusiveScan(tmp, tn_, head, head_s, cub::Max(), static_cast<int>(n), st);
    tbp.head = head_s;
    {
        KernelScope ks(ctx, "task_flag");
        task_flag_kernel<<<blocks_for(n, T), T, 0, st>>>(tbp);
    }
    tn_ = t_need;
    cub::DeviceScan::ExclusiveSum(tmp, tn_, flag, tidx, static_cast<int>(n), st);
    {
        KernelScope ks(ctx, "task_fill");
        task_fill_kernel<<<blocks_for(n, T), T, 0, st>>>(tbp);
    }
    {
        KernelScope ks(ctx, "task_finalize");
        task_finalize_kernel<<<1, 1, 0, st>>>(tbp);
    }

    // Main-pass slot: the smallest power of two that covers 99.5 % of the tasks (and no
    // less than the largest task when that still fits a full grid); tasks needing more
    // are deferred to the redo passes, which size scratch per task.
    uint64_t h_need = 0;
    unsigned int h_hist[64];
    uint32_t h_ranges[4];
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&h_need, need_max, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(h_hist, need_hist, sizeof(h_hist), cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(h_ranges, cnt, sizeof(h_ranges), cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    PHR_CUDA_TRY(ctx, cudaGetLastError());
    hs_setup.stop();
    {
        uint64_t n_tasks = 0;  // tasks of the main pass with a scratch need
        for (int b = 0; b < 64; ++b) n_tasks += h_hist[b];
        const uint64_t full_grid_warps =
            static_cast<uint64_t>(ctx->sm_count) * ctx->tune.max_blocks_per_sm * (ctx->tune.block_threads / 32);
        if (h_need * full_grid_warps > ctx->scratch_budget && n_tasks > 0) {
            uint64_t acc = 0, slot = 4096;
            for (int b = 0; b < 64; ++b) {
                acc += h_hist[b];
                slot = b >= 63 ? ~0ull : (1ull << b);
                if (acc * 1000 >= n_tasks * 995) break;
            }
            h_need = std::min(h_need, std::max<uint64_t>(slot, 64 << 10));
        }
    }

    const bool is_myers = engine == PHR_ENGINE_MYERS_FIT || engine == PHR_ENGINE_MYERS_GLOBAL;
    ExtendParams P{};
    P.desc = desc;
    P.out = pout;
    P.packed2 = arena2;
    P.bytes = arenab;
    P.text = text;
    P.text_off = tbo;
    P.scratch = nullptr;
    P.redo_list = redo_list;
    P.redo_count = cnt + 7;
    P.redo_need_max = need_max;
    P.redo_need = redo_need;
    P.task_need = task_need;
    P.engine = engine;
    P.full_band = 0;
    P.band_base = ctx->tune.myers_band_base;
    P.lane_ckpt = ctx->tune.myers_lane_ckpt;
    P.costs = costs;
    P.error_flag = cnt + 10;
    P.big_min = ctx->tune.wfa_big_min;
    P.big_smem = static_cast<uint32_t>(ctx->tune.wfa_big_smem);
    P.work = reinterpret_cast<unsigned long long*>(cnt + 32);

    const int block = ctx->tune.block_threads;
    // main pass (per_task false): per-warp slots of `slot` bytes; redo passes: per-task
    // scratch (P.task_off / P.task_len set by the caller, `per_task_total` bytes in all,
    // `n_tasks_hint` tasks)
    auto launch_pass = [&](const uint32_t* ord, const uint32_t* tfirst, const uint8_t* tcount, const uint8_t* tgroup,
                           const uint32_t* range0, const uint32_t* range1, uint64_t slot, int full_band,
                           bool per_task = false, uint64_t per_task_total = 0,
                           uint64_t n_tasks_hint = 0) -> phr_status {
        const uint64_t warps_per_block = block / 32;
        uint64_t grid = static_cast<uint64_t>(ctx->sm_count) * ctx->tune.max_blocks_per_sm;
        if (!per_task) {
            slot = std::max<uint64_t>((slot + 255) & ~255ull, 4096);
            // grid: resident blocks per SM, no more warps than tasks, shrunk to the scratch budget
            grid = std::max<uint64_t>(1, std::min<uint64_t>(grid, (h_ranges[3] + warps_per_block - 1) / warps_per_block));
            while (grid > 1 && grid * warps_per_block * slot > ctx->scratch_budget) grid = (grid + 1) / 2;
            PHR_CUDA_TRY(ctx, ctx->scratch.reserve(grid * warps_per_block * slot));
        } else {
            grid = std::max<uint64_t>(1, std::min<uint64_t>(grid, (n_tasks_hint + warps_per_block - 1) / warps_per_block));
            PHR_CUDA_TRY(ctx, ctx->scratch.reserve(per_task_total));
        }
        P.scratch = reinterpret_cast<uint8_t*>(ctx->scratch.base);
        P.slot_bytes = slot;
        P.full_band = full_band;
        P.tasks.order = ord;
        P.tasks.task_first = tfirst;
        P.tasks.task_count = tcount;
        P.tasks.task_group = tgroup;
        PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt + 5, 0, 8, st));
        static const char* const names[2][3][2] = {
            {{"myers", "myers_bytes"}, {"wfa_linear", "wfa_linear_bytes"}, {"wfa_affine", "wfa_affine_bytes"}},
            {{"myers_redo", "myers_bytes_redo"}, {"wfa_linear_redo", "wfa_linear_bytes_redo"},
             {"wfa_affine_redo", "wfa_affine_bytes_redo"}}};
        const int ek = is_myers ? 0 : engine == PHR_ENGINE_WFA_LINEAR ? 1 : 2;
        const char* kname = names[per_task][ek][0];
        const char* kname_b = names[per_task][ek][1];
        if (!per_task && engine == PHR_ENGINE_MYERS_GLOBAL) {
            // global 2-bit pairs of one lane each (tasks [0, g1)); the warp-group kernel
            // below takes the remaining 2-bit tasks [g1, split)
            const uint64_t lane_grid =
                std::min<uint64_t>(grid * warps_per_block / (kLaneThreads / 32),
                                   static_cast<uint64_t>(ctx->sm_count) * myers_lane_blocks_per_sm(P.lane_ckpt));
            PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt + 26, 0, 4, st));
            P.tasks.range = cnt + 28;
            P.queue_head = cnt + 26;
            {
                KernelScope ks(ctx, "myers_lane");
                launch_myers_lane(P, static_cast<int>(std::max<uint64_t>(lane_grid, 1)), st);
            }
            range0 = cnt + 30;
        }
        P.tasks.range = range0;
        P.queue_head = cnt + 5;
        {
            KernelScope ks(ctx, kname);
            if (is_myers)
                launch_myers(P, static_cast<int>(grid), block, st);
            else if (engine == PHR_ENGINE_WFA_LINEAR)
                launch_wfa_linear(P, static_cast<int>(grid), block, st);
            else
                launch_wfa_affine(P, static_cast<int>(grid), block, st);
        }
        P.tasks.range = range1;
        P.queue_head = cnt + 6;
        {
            KernelScope ks(ctx, kname_b);
            if (is_myers)
                launch_myers_bytes(P, static_cast<int>(grid), block, st);
            else if (engine == PHR_ENGINE_WFA_LINEAR)
                launch_wfa_linear_bytes(P, static_cast<int>(grid), block, st);
            else
                launch_wfa_affine_bytes(P, static_cast<int>(grid), block, st);
        }
        if (per_task && (engine == PHR_ENGINE_WFA_LINEAR || engine == PHR_ENGINE_WFA_AFFINE) && P.big_min > 0 &&
            n_tasks_hint > 0) {
            // long pairs of this redo list, one CTA each
            // linear: two CTAs of kBigThreads per SM (one when the tune keeps fewer blocks
            // resident); gap-affine: kBigAffineThreads / wfa_affine_big_threads CTAs per SM
            const int aff_threads = ctx->tune.wfa_affine_big_threads;
            const uint64_t big_per_sm = engine == PHR_ENGINE_WFA_AFFINE
                                            ? static_cast<uint64_t>(kBigAffineThreads / aff_threads)
                                            : (ctx->tune.max_blocks_per_sm >= 4 ? 2 : 1);
            const int big_grid = static_cast<int>(std::min<uint64_t>(n_tasks_hint, ctx->sm_count * big_per_sm));
            PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt + 24, 0, 8, st));
            for (int mode = 0; mode < 2; ++mode) {
                P.tasks.range = mode ? range1 : range0;
                P.queue_head = cnt + 24 + mode;
                if (engine == PHR_ENGINE_WFA_LINEAR) {
                    KernelScope ks(ctx, mode ? "wfa_linear_big_bytes" : "wfa_linear_big");
                    launch_wfa_linear_big(P, big_grid, mode, st);
                } else {
                    KernelScope ks(ctx, mode ? "wfa_affine_big_bytes" : "wfa_affine_big");
                    launch_wfa_affine_big(P, big_grid, aff_threads, mode, st);
                }
            }
        }
        PHR_CUDA_TRY(ctx, cudaGetLastError());
        return PHR_OK;
    };

    phr_status s = launch_pass(order, task_first, task_count, task_group, cnt + 0, cnt + 2, h_need, 0);
    if (s != PHR_OK) return s;

    // Redo passes: each pair that did not fit its slot (or, for Myers, whose edit distance
    // left the stored band) runs again alone, with scratch sized for it: pairs are packed
    // into passes of at most the workspace budget, one variable-size region per task.
    uint32_t* rlist = redo_list;
    uint32_t* rlist2 = head;  // reuse: free after task build
    P.task_need = nullptr;
    std::vector<uint32_t> h_list;
    std::vector<unsigned long long> h_rneed;
    std::unordered_set<uint32_t> clamped;
    // a pair that still overflows the whole budget ends with status PHR_ERR_OOM (the
    // other pairs of the call go on)
    static const PairOut kOomOut = {PHR_ERR_OOM, 0, 0, 0, 0, 0};
    uint64_t n_oom = 0;
    HostScope hs_redo(ctx, "host:redo");
    for (int round = 0; round < 12; ++round) {
        uint32_t h_redo = 0;
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&h_redo, cnt + 7, 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        if (h_redo == 0) break;
        if (round == 11) return set_error(ctx, PHR_ERR_CAPACITY, "extension did not fit after repeated redo passes");
        h_list.resize(h_redo);
        h_rneed.resize(h_redo);
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(h_list.data(), rlist, h_redo * 4, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(h_rneed.data(), redo_need, h_redo * 8, cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        PHR_CUDA_TRY(ctx, cudaMemsetAsync(cnt + 7, 0, 4, st));
        // largest first, packed into passes within the budget
        std::vector<uint32_t> idx(h_redo);
        for (uint32_t i = 0; i < h_redo; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return h_rneed[a] > h_rneed[b]; });
        if (const char* tp = std::getenv("PHRAYA_EXTEND_TRACE")) {
            // one line per redo round: engine round pairs budget, then the eight largest
            // needs as qn:tn:need_bytes
            if (FILE* f = std::fopen(tp, "a")) {
                std::fprintf(f, "engine %d round %d pairs %u budget %llu", static_cast<int>(engine), round, h_redo,
                             static_cast<unsigned long long>(ctx->scratch_budget));
                for (uint32_t i = 0; i < std::min<uint32_t>(h_redo, 8); ++i) {
                    PairDesc hd{};
                    PHR_CUDA_TRY(ctx, cudaMemcpy(&hd, desc + h_list[idx[i]], sizeof(PairDesc), cudaMemcpyDeviceToHost));
                    std::fprintf(f, " %d:%d:%llu", hd.qn, hd.tn, h_rneed[idx[i]]);
                }
                std::fprintf(f, "\n");
                std::fclose(f);
            }
        }
        size_t pos = 0;
        while (pos < idx.size()) {
            std::vector<uint32_t> pl;
            std::vector<uint64_t> po, pn;
            uint64_t tot = 0;
            while (pos < idx.size()) {
                uint64_t need = (std::max<uint64_t>(h_rneed[idx[pos]], 4096) + 255) & ~255ull;
                bool clamp = false;
                if (need > ctx->scratch_budget) {
                    // first-pass needs are estimates: try once with the whole budget
                    if (clamped.count(h_list[idx[pos]])) {
                        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(pout + h_list[idx[pos]], &kOomOut, sizeof(PairOut),
                                                          cudaMemcpyHostToDevice, st));
                        ++n_oom;
                        ++pos;
                        continue;
                    }
                    clamp = true;
                    need = ctx->scratch_budget & ~255ull;
                }
                if (!pl.empty() && tot + need > ctx->scratch_budget) break;  // this pair opens the next pass
                // the whole-budget try is spent only once the pair is placed in a pass
                if (clamp) clamped.insert(h_list[idx[pos]]);
                pl.push_back(h_list[idx[pos]]);
                po.push_back(tot);
                pn.push_back(need);
                tot += need;
                ++pos;
            }
            const uint32_t m = static_cast<uint32_t>(pl.size());
            if (m == 0) continue;
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(rlist2, pl.data(), m * 4, cudaMemcpyHostToDevice, st));
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(rtask_off, po.data(), m * 8, cudaMemcpyHostToDevice, st));
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(rtask_len, pn.data(), m * 8, cudaMemcpyHostToDevice, st));
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(cnt + 18, &m, 4, cudaMemcpyHostToDevice, st));
            {
                KernelScope ks(ctx, "redo_tasks");
                redo_tasks_kernel<<<blocks_for(m, T), T, 0, st>>>(rlist2, cnt + 18, desc, engine,
                                                                 g_short, ctx->tune.wfa_group_long,
                                                                 ctx->tune.wfa_long_min,
                                                                 P.big_min, P.big_smem, task_first, task_count,
                                                                 task_group, cnt + 14);
            }
            // byte-mode and 2-bit pairs share this list: both launches walk all of it
            PHR_CUDA_TRY(ctx, cudaMemcpyAsync(cnt + 16, cnt + 14, 8, cudaMemcpyDeviceToDevice, st));
            P.redo_list = rlist;   // fresh overflows of this pass are appended here
            P.task_off = rtask_off;
            P.task_len = rtask_len;
            // synchronise before the scratch buffer may be reallocated for this pass
            PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
            s = launch_pass(rlist2, task_first, task_count, task_group, cnt + 14, cnt + 16, 0, 1, true, tot, m);
            P.task_off = nullptr;
            P.task_len = nullptr;
            if (s != PHR_OK) return s;
            PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        }
    }

    hs_redo.stop();
    if (n_oom) ctx->counters["scratch_oom_pairs"] += n_oom;
    if (const char* tp = std::getenv("PHRAYA_EXTEND_TRACE")) {
        // one line per pair of qlen + tlen >= 65536: its final status and distance
        std::vector<PairDesc> hd(n);
        std::vector<PairOut> ho(n);
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(hd.data(), desc, n * sizeof(PairDesc), cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(ho.data(), pout, n * sizeof(PairOut), cudaMemcpyDeviceToHost, st));
        PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        if (FILE* f = std::fopen(tp, "a")) {
            for (uint64_t i = 0; i < n; ++i)
                if (static_cast<int64_t>(hd[i].qn) + hd[i].tn >= 65536)
                    std::fprintf(f, "engine %d pair %llu %d:%d seed %d:%d status %d ed %d\n", static_cast<int>(engine),
                                 static_cast<unsigned long long>(i), hd[i].qn, hd[i].tn, hd[i].qs, hd[i].ts,
                                 ho[i].status, ho[i].ed);
            std::fclose(f);
        }
    }
    HostScope hs_tail(ctx, "host:extend_tail");
    // pack CIGAR text
    {
        KernelScope ks(ctx, "text_len");
        text_len_kernel<<<blocks_for(n, T), T, 0, st>>>(pout, n, tlen);
    }
    tn_ = t_need;
    cub::DeviceScan::ExclusiveSum(tmp, tn_, tlen, cigoff, static_cast<int>(n), st);
    {
        KernelScope ks(ctx, "total");
        total_kernel<<<1, 1, 0, st>>>(cigoff, tlen, n, total);
    }
    uint64_t h_total = 0;
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&h_total, total, 8, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (h_total > res->cigar_capacity)
        return set_error(ctx, PHR_ERR_CAPACITY, "CIGAR arena too small: need " + std::to_string(h_total) + " bytes");
    FinishParams F{n,           engine,     desc,       pout,    tbo, text, cigoff, res->aln, res->cigar,
                   res->cigar_capacity, cnt + 10, res->cigar_base};
    {
        KernelScope ks(ctx, "finish");
        finish_kernel<<<blocks_for((n + 31) / 32 * 32, T), T, 0, st>>>(F);
    }
    uint32_t h_err = 0;
    unsigned long long h_work[4] = {0, 0, 0, 0};
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(&h_err, cnt + 10, 4, cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(h_work, cnt + 32, sizeof(h_work), cudaMemcpyDeviceToHost, st));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (h_work[0]) ctx->counters["myers_lane_block_columns"] += h_work[0];
    if (h_work[1]) ctx->counters["myers_lane_redo_pairs"] += h_work[1];
    if (h_work[2] || h_work[3]) {
        const std::string e = engine == PHR_ENGINE_WFA_AFFINE ? "wfa_affine" : "wfa_linear";
        ctx->counters[e + "_cells"] += h_work[2];
        ctx->counters[e + "_lcp_words"] += h_work[3];
    }
    PHR_CUDA_TRY(ctx, cudaGetLastError());
    if (ctx->timing) ctx->resolve_timings();
    if (h_err) return set_error(ctx, PHR_ERR_CUDA, "internal consistency check failed (flags " + std::to_string(h_err) + ")");
    res->cigar_used = h_total;
    return PHR_OK;
}

}  // namespace phr
