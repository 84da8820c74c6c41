// api.cu -- C ABI entry points (include/phraya_gpu.h): context and pairs API.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "engine.cuh"

using phr::Ctx;

namespace {

phr_status check_ctx(phr_ctx* c) { return c ? PHR_OK : PHR_ERR_ARG; }

// Copies a host pair batch (bounds already checked) into the context's io arena and
// returns device views.
phr_status upload_pairs(Ctx* ctx, const phr_pair_batch* b, phr::DevPairs* dp, size_t extra) {
    const uint64_t n = b->n_pairs;
    const size_t need = b->seq_bytes + 64 + n * (8 + 4 + 8 + 4 + 4 + 4) + 8 * 256 + extra;
    ctx->io.reset();
    PHR_CUDA_TRY(ctx, ctx->io.reserve(need));
    auto take = [&](size_t bytes) { return ctx->io.take(bytes); };
    uint8_t* seq = static_cast<uint8_t*>(take(b->seq_bytes + 64));
    uint64_t* qo = static_cast<uint64_t*>(take(n * 8));
    uint32_t* ql = static_cast<uint32_t*>(take(n * 4));
    uint64_t* to = static_cast<uint64_t*>(take(n * 8));
    uint32_t* tl = static_cast<uint32_t*>(take(n * 4));
    uint32_t* qs = b->q_seed ? static_cast<uint32_t*>(take(n * 4)) : nullptr;
    uint32_t* ts = b->t_seed ? static_cast<uint32_t*>(take(n * 4)) : nullptr;
    cudaStream_t st = ctx->stream;
    if (b->seq_bytes) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(seq, b->seq, b->seq_bytes, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(qo, b->q_off, n * 8, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(ql, b->q_len, n * 4, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(to, b->t_off, n * 8, cudaMemcpyHostToDevice, st));
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(tl, b->t_len, n * 4, cudaMemcpyHostToDevice, st));
    if (qs) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(qs, b->q_seed, n * 4, cudaMemcpyHostToDevice, st));
    if (ts) PHR_CUDA_TRY(ctx, cudaMemcpyAsync(ts, b->t_seed, n * 4, cudaMemcpyHostToDevice, st));
    dp->n = n;
    dp->seq = seq;
    dp->seq_bytes = b->seq_bytes;
    dp->q_off = qo;
    dp->q_len = ql;
    dp->t_off = to;
    dp->t_len = tl;
    dp->q_seed = qs;
    dp->t_seed = ts;
    return PHR_OK;
}

bool valid_engine(phr_engine e) {
    return e == PHR_ENGINE_WFA_LINEAR || e == PHR_ENGINE_WFA_AFFINE || e == PHR_ENGINE_MYERS_FIT ||
           e == PHR_ENGINE_MYERS_GLOBAL;
}

// One chunk of a pipelined host batch: pairs [a, b), sequence bytes [lo, hi).
struct HostChunk {
    uint64_t a, b, lo, hi, sum_qt;
};

// One pass over a host batch on up to 16 threads: bounds of every pair, and per segment
// of consecutive pairs its byte span and length sum. Returns the first pair that reaches
// past seq_bytes (n when none).
struct HostSeg {
    uint64_t a, b, lo, hi, sum_qt, bad;
};

uint64_t scan_host_batch(const phr_pair_batch* b, std::vector<HostSeg>* segs, uint64_t nseg) {
    const uint64_t n = b->n_pairs;
    nseg = std::max<uint64_t>(1, std::min(nseg, n));
    segs->assign(nseg, HostSeg{0, 0, UINT64_MAX, 0, 0, n});
    auto work = [&](uint64_t s0, uint64_t s1) {
        for (uint64_t s = s0; s < s1; ++s) {
            HostSeg& g = (*segs)[s];
            g.a = n * s / nseg;
            g.b = n * (s + 1) / nseg;
            for (uint64_t i = g.a; i < g.b; ++i) {
                const uint64_t qe = b->q_off[i] + b->q_len[i], te = b->t_off[i] + b->t_len[i];
                if ((qe > b->seq_bytes || te > b->seq_bytes) && g.bad == n) g.bad = i;
                g.lo = std::min(g.lo, std::min(b->q_off[i], b->t_off[i]));
                g.hi = std::max(g.hi, std::max(qe, te));
                g.sum_qt += static_cast<uint64_t>(b->q_len[i]) + b->t_len[i];
            }
        }
    };
    const uint64_t nthr = std::min<uint64_t>(std::min<uint64_t>(16, std::max(1u, std::thread::hardware_concurrency())),
                                             n >= (1u << 16) ? nseg : 1);
    if (nthr <= 1) {
        work(0, nseg);
    } else {
        std::vector<std::thread> th;
        for (uint64_t t = 0; t < nthr; ++t) th.emplace_back(work, nseg * t / nthr, nseg * (t + 1) / nthr);
        for (std::thread& x : th) x.join();
    }
    uint64_t bad = n;
    for (const HostSeg& g : *segs) bad = std::min(bad, g.bad);
    return bad;
}

// Groups consecutive segments into chunks of about `target` sequence bytes each.
std::vector<HostChunk> plan_chunks(const std::vector<HostSeg>& segs, uint64_t target) {
    std::vector<HostChunk> out;
    HostChunk c{0, 0, UINT64_MAX, 0, 0};
    for (const HostSeg& g : segs) {
        if (g.b == g.a) continue;
        const uint64_t nlo = std::min(c.lo, g.lo), nhi = std::max(c.hi, g.hi);
        if (c.b > c.a && nhi - nlo > target) {
            out.push_back(c);
            c = HostChunk{g.a, g.a, g.lo, g.hi, 0};
        } else {
            c.lo = nlo;
            c.hi = nhi;
        }
        c.b = g.b;
        c.sum_qt += g.sum_qt;
    }
    if (c.b > c.a) out.push_back(c);
    return out;
}

// Host batch in one piece: copy in, align, copy out.
phr_status extend_host_whole(phr_ctx* c, phr_engine engine, const phr_pair_batch* batch, phr_affine_costs costs,
                             phr_result_arena* out, uint64_t sum_qt) {
    Ctx* ctx = &c->impl;
    const uint64_t n = batch->n_pairs;
    // device output: alignments + worst-case packed text, in the io arena after the inputs
    const uint64_t text_cap = std::min<uint64_t>(out->cigar_capacity, 2 * sum_qt + 16 * n);
    const size_t extra = n * sizeof(phr_alignment) + text_cap + 1024;
    phr::DevPairs dp;
    phr_status s = upload_pairs(ctx, batch, &dp, extra);
    if (s != PHR_OK) return s;
    phr::DevResults r;
    r.aln = static_cast<phr_alignment*>(ctx->io.take(n * sizeof(phr_alignment)));
    r.cigar = static_cast<char*>(ctx->io.take(text_cap + 16));
    r.cigar_capacity = text_cap;
    s = phr::run_extend(ctx, engine, dp, costs, &r, sum_qt);
    if (s != PHR_OK) return s;
    if (r.cigar_used > out->cigar_capacity)
        return phr::set_error(ctx, PHR_ERR_CAPACITY, "CIGAR arena too small");
    PHR_CUDA_TRY(ctx, cudaMemcpyAsync(out->aln, r.aln, n * sizeof(phr_alignment), cudaMemcpyDeviceToHost, ctx->stream));
    if (r.cigar_used)
        PHR_CUDA_TRY(ctx, cudaMemcpyAsync(out->cigar, r.cigar, r.cigar_used, cudaMemcpyDeviceToHost, ctx->stream));
    PHR_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    out->cigar_used = r.cigar_used;
    return PHR_OK;
}

// Host batch in chunks through two device slots: while chunk c aligns on the context
// stream, chunk c+1's inputs travel host -> device on copy_in and chunk c-1's results
// device -> host on copy_out. Results are identical to the one-piece path: pairs are
// independent, and each chunk's CIGAR text lands right after the previous chunk's.
phr_status extend_host_chunked(phr_ctx* c, phr_engine engine, const phr_pair_batch* batch, phr_affine_costs costs,
                               phr_result_arena* out, const std::vector<HostChunk>& ch) {
    Ctx* ctx = &c->impl;
    for (cudaStream_t* sp : {&ctx->copy_in, &ctx->copy_out})
        if (!*sp) PHR_CUDA_TRY(ctx, cudaStreamCreateWithFlags(sp, cudaStreamNonBlocking));
    const bool seeds_q = batch->q_seed != nullptr, seeds_t = batch->t_seed != nullptr;
    uint64_t max_span = 0, max_n = 0, max_text = 0;
    for (const HostChunk& k : ch) {
        max_span = std::max(max_span, k.hi - k.lo);
        max_n = std::max(max_n, k.b - k.a);
        max_text = std::max(max_text, std::min<uint64_t>(out->cigar_capacity, 2 * k.sum_qt + 16 * (k.b - k.a)));
    }
    auto a256 = [](uint64_t x) { return (x + 511) / 256 * 256; };
    const uint64_t slot_in = a256(max_span + 64) + 2 * a256(max_n * 8) + 4 * a256(max_n * 4);
    const uint64_t slot_out = a256(max_n * sizeof(phr_alignment)) + a256(max_text + 16);
    ctx->io.reset();
    PHR_CUDA_TRY(ctx, ctx->io.reserve(2 * (slot_in + slot_out) + 4096));
    struct Slot {
        uint8_t* seq;
        uint64_t *qo, *to;
        uint32_t *ql, *tl, *qs, *ts;
        phr_alignment* aln;
        char* cig;
    } slot[2];
    for (Slot& sl : slot) {
        sl.seq = static_cast<uint8_t*>(ctx->io.take(max_span + 64));
        sl.qo = static_cast<uint64_t*>(ctx->io.take(max_n * 8));
        sl.to = static_cast<uint64_t*>(ctx->io.take(max_n * 8));
        sl.ql = static_cast<uint32_t*>(ctx->io.take(max_n * 4));
        sl.tl = static_cast<uint32_t*>(ctx->io.take(max_n * 4));
        sl.qs = static_cast<uint32_t*>(ctx->io.take(max_n * 4));
        sl.ts = static_cast<uint32_t*>(ctx->io.take(max_n * 4));
        sl.aln = static_cast<phr_alignment*>(ctx->io.take(max_n * sizeof(phr_alignment)));
        sl.cig = static_cast<char*>(ctx->io.take(max_text + 16));
        if (!sl.seq || !sl.qo || !sl.to || !sl.ql || !sl.tl || !sl.qs || !sl.ts || !sl.aln || !sl.cig)
            return phr::set_error(ctx, PHR_ERR_OOM, "io arena exhausted");
    }
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr}, ev_done = nullptr;
    auto cleanup = [&]() {
        cudaStreamSynchronize(ctx->copy_in);
        cudaStreamSynchronize(ctx->copy_out);
        for (cudaEvent_t e : {ev_in[0], ev_in[1], ev_out[0], ev_out[1], ev_done})
            if (e) cudaEventDestroy(e);
    };
    phr_status st = PHR_OK;
    auto fail = [&](phr_status s) {
        cleanup();
        return s;
    };
    for (cudaEvent_t* e : {&ev_in[0], &ev_in[1], &ev_out[0], &ev_out[1], &ev_done})
        if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess)
            return fail(phr::cuda_status(ctx, cudaGetLastError(), "cudaEventCreate"));
    auto upload = [&](size_t ci) -> cudaError_t {
        const HostChunk& k = ch[ci];
        const Slot& sl = slot[ci & 1];
        const uint64_t m = k.b - k.a;
        cudaStream_t s = ctx->copy_in;
        cudaError_t e = cudaMemcpyAsync(sl.seq, batch->seq + k.lo, k.hi - k.lo, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.qo, batch->q_off + k.a, m * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.ql, batch->q_len + k.a, m * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.to, batch->t_off + k.a, m * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.tl, batch->t_len + k.a, m * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && seeds_q) e = cudaMemcpyAsync(sl.qs, batch->q_seed + k.a, m * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && seeds_t) e = cudaMemcpyAsync(sl.ts, batch->t_seed + k.a, m * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaEventRecord(ev_in[ci & 1], s);
        return e;
    };
    {
        phr::HostScope hs(ctx, "host:e2e_first_uploads");
        for (size_t ci = 0; ci < std::min<size_t>(2, ch.size()); ++ci)
            if (cudaError_t e = upload(ci); e != cudaSuccess) return fail(phr::cuda_status(ctx, e, "chunk upload"));
    }
    uint64_t base = 0;
    for (size_t ci = 0; ci < ch.size(); ++ci) {
        const HostChunk& k = ch[ci];
        const Slot& sl = slot[ci & 1];
        const uint64_t m = k.b - k.a;
        cudaError_t e = cudaStreamWaitEvent(ctx->stream, ev_in[ci & 1], 0);
        if (e == cudaSuccess && ci >= 2) e = cudaStreamWaitEvent(ctx->stream, ev_out[ci & 1], 0);
        if (e != cudaSuccess) return fail(phr::cuda_status(ctx, e, "chunk wait"));
        phr::DevPairs dp;
        dp.n = m;
        // offsets stay absolute: the slot holds bytes [lo, hi) at sl.seq
        dp.seq = reinterpret_cast<const uint8_t*>(reinterpret_cast<uintptr_t>(sl.seq) - k.lo);
        dp.seq_bytes = k.hi;
        dp.q_off = sl.qo;
        dp.q_len = sl.ql;
        dp.t_off = sl.to;
        dp.t_len = sl.tl;
        dp.q_seed = seeds_q ? sl.qs : nullptr;
        dp.t_seed = seeds_t ? sl.ts : nullptr;
        phr::DevResults r;
        r.aln = sl.aln;
        r.cigar = sl.cig;
        r.cigar_capacity = std::min<uint64_t>(out->cigar_capacity - base, max_text);
        r.cigar_base = base;
        {
            phr::HostScope hs(ctx, "host:e2e_run_extend");
            st = phr::run_extend(ctx, engine, dp, costs, &r, k.sum_qt);
        }
        if (st != PHR_OK) return fail(st);
        e = cudaEventRecord(ev_done, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_out, ev_done, 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out->aln + k.a, sl.aln, m * sizeof(phr_alignment), cudaMemcpyDeviceToHost,
                                ctx->copy_out);
        if (e == cudaSuccess && r.cigar_used)
            e = cudaMemcpyAsync(out->cigar + base, sl.cig, r.cigar_used, cudaMemcpyDeviceToHost, ctx->copy_out);
        if (e == cudaSuccess) e = cudaEventRecord(ev_out[ci & 1], ctx->copy_out);
        if (e != cudaSuccess) return fail(phr::cuda_status(ctx, e, "chunk download"));
        base += r.cigar_used;
        // this slot's inputs were consumed by the (synchronous) alignment above
        if (ci + 2 < ch.size())
            if (cudaError_t e2 = upload(ci + 2); e2 != cudaSuccess) return fail(phr::cuda_status(ctx, e2, "chunk upload"));
    }
    {
        phr::HostScope hs(ctx, "host:e2e_drain");
        cleanup();
    }
    if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) return phr::cuda_status(ctx, e, "chunked batch");
    out->cigar_used = base;
    return PHR_OK;
}

phr_status extend_host(phr_ctx* c, phr_engine engine, const phr_pair_batch* batch, phr_affine_costs costs,
                       phr_result_arena* out) {
    Ctx* ctx = &c->impl;
    if (!batch || !out || (batch->n_pairs && (!batch->q_off || !batch->q_len || !batch->t_off || !batch->t_len ||
                                               !out->aln || (!batch->seq && batch->seq_bytes))))
        return phr::set_error(ctx, PHR_ERR_ARG, "NULL batch/arena pointer");
    if (!valid_engine(engine)) return phr::set_error(ctx, PHR_ERR_ARG, "unknown engine");
    out->cigar_used = 0;
    const uint64_t n = batch->n_pairs;
    if (n == 0) return PHR_OK;
    std::vector<HostSeg> segs;
    {
        phr::HostScope hs(ctx, "host:e2e_scan");
        const uint64_t bad = scan_host_batch(batch, &segs, 64);
        if (bad < n) return phr::set_error(ctx, PHR_ERR_ARG, "pair " + std::to_string(bad) + " reaches past seq_bytes");
    }
    // batches of more than 2 kChunkMin sequence bytes run in about host_chunks overlapped
    // chunks of at least 4 kChunkMin / host_chunks bytes
    constexpr uint64_t kChunkMin = 64ull << 20;
    if (batch->seq_bytes > 2 * kChunkMin) {
        const uint64_t nch = static_cast<uint64_t>(ctx->tune.host_chunks);
        const std::vector<HostChunk> ch =
            plan_chunks(segs, std::max<uint64_t>(4 * kChunkMin / nch, batch->seq_bytes / nch));
        uint64_t span = 0;
        for (const HostChunk& k : ch) span += k.hi - k.lo;
        // chunks whose pairs reference scattered bytes would copy more than the batch: one piece
        if (ch.size() > 1 && span <= batch->seq_bytes + batch->seq_bytes / 4)
            return extend_host_chunked(c, engine, batch, costs, out, ch);
    }
    uint64_t sum_qt = 0;
    for (const HostSeg& g : segs) sum_qt += g.sum_qt;
    return extend_host_whole(c, engine, batch, costs, out, sum_qt);
}

}  // namespace

extern "C" {

int32_t phr_abi_version(void) { return PHR_ABI_VERSION; }

const char* phr_status_string(phr_status s) {
    switch (s) {
        case PHR_OK: return "ok";
        case PHR_INVALID_INPUT: return "invalid input (seed beyond sequence end)";
        case PHR_ALIGNMENT_FAILED: return "alignment failed (search exhausted)";
        case PHR_ERR_OOM: return "out of device memory";
        case PHR_ERR_CUDA: return "CUDA error";
        case PHR_ERR_ARG: return "bad argument";
        case PHR_ERR_CAPACITY: return "output arena too small";
        case PHR_ERR_STATE: return "call out of order";
    }
    return "unknown status";
}

phr_status phr_ctx_create(int32_t device, const phr_config* cfg, phr_ctx** out) {
    if (!out) return PHR_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PHR_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return PHR_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return PHR_ERR_CUDA;
    phr_ctx* c = new (std::nothrow) phr_ctx();
    if (!c) return PHR_ERR_OOM;
    Ctx* ctx = &c->impl;
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return PHR_ERR_CUDA;
    }
    ctx->bind_stream();
    {
        // default scratch cap: a fifth of the device memory, within [8 GiB, 48 GiB]
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess)
            ctx->scratch_budget = std::min<size_t>(std::max<size_t>(tot / 5, 8ull << 30), 48ull << 30);
        cudaGetLastError();
    }
    if (cfg && cfg->workspace_bytes) ctx->scratch_budget = cfg->workspace_bytes;
    if (cfg && cfg->tune_file_enable) {
        ctx->tune_file_enable = true;
        ctx->tune_file = cfg->tune_file ? cfg->tune_file : "phraya_b200_tune.txt";
        if (FILE* f = std::fopen(ctx->tune_file.c_str(), "r")) {
            char key[64];
            long long v = 0;
            while (std::fscanf(f, "%63s %lld", key, &v) == 2) phr_ctx_set_tune(c, key, v);
            std::fclose(f);
        }
    }
    *out = c;
    return PHR_OK;
}

namespace {
int* tune_field(phr::EngineTune& t, const char* key) {
    if (!std::strcmp(key, "wfa_group_short")) return &t.wfa_group_short;
    if (!std::strcmp(key, "wfa_affine_group_short")) return &t.wfa_affine_group_short;
    if (!std::strcmp(key, "wfa_group_long")) return &t.wfa_group_long;
    if (!std::strcmp(key, "myers_band_base")) return &t.myers_band_base;
    if (!std::strcmp(key, "block_threads")) return &t.block_threads;
    if (!std::strcmp(key, "wfa_big_min")) return &t.wfa_big_min;
    if (!std::strcmp(key, "wfa_big_smem")) return &t.wfa_big_smem;
    if (!std::strcmp(key, "max_blocks_per_sm")) return &t.max_blocks_per_sm;
    if (!std::strcmp(key, "wfa_long_min")) return &t.wfa_long_min;
    if (!std::strcmp(key, "host_chunks")) return &t.host_chunks;
    if (!std::strcmp(key, "myers_lane_ckpt")) return &t.myers_lane_ckpt;
    if (!std::strcmp(key, "wfa_affine_big_threads")) return &t.wfa_affine_big_threads;
    return nullptr;
}
bool tune_valid(const char* key, int64_t v) {
    if (!std::strcmp(key, "wfa_group_short") || !std::strcmp(key, "wfa_group_long") ||
        !std::strcmp(key, "wfa_affine_group_short"))
        return v >= 1 && v <= 32 && (v & (v - 1)) == 0;
    if (!std::strcmp(key, "myers_band_base")) return v >= 0 && v <= (1 << 20);
    if (!std::strcmp(key, "block_threads")) return v >= 32 && v <= 256 && v % 32 == 0;
    if (!std::strcmp(key, "wfa_big_min")) return v >= 0 && v <= INT32_MAX;
    if (!std::strcmp(key, "wfa_big_smem")) return v >= (16 << 10) && v <= (200 << 10) && v % 16 == 0;
    if (!std::strcmp(key, "max_blocks_per_sm")) return v >= 1 && v <= 4;
    if (!std::strcmp(key, "wfa_long_min")) return v >= 0 && v <= INT32_MAX;
    if (!std::strcmp(key, "host_chunks")) return v >= 2 && v <= 32;
    if (!std::strcmp(key, "myers_lane_ckpt")) return v == 0 || v == 1;
    if (!std::strcmp(key, "wfa_affine_big_threads")) return v == 256 || v == 512 || v == 1024;
    return false;
}
}  // namespace

phr_status phr_ctx_set_tune(phr_ctx* c, const char* key, int64_t value) {
    if (!c || !key) return PHR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->impl.mu);
    int* f = tune_field(c->impl.tune, key);
    if (!f) return phr::set_error(&c->impl, PHR_ERR_ARG, std::string("unknown tune key ") + key);
    if (!tune_valid(key, value)) return phr::set_error(&c->impl, PHR_ERR_ARG, std::string("tune value out of range for ") + key);
    *f = static_cast<int>(value);
    return PHR_OK;
}

phr_status phr_ctx_get_tune(const phr_ctx* c, const char* key, int64_t* value) {
    if (!c || !key || !value) return PHR_ERR_ARG;
    int* f = tune_field(const_cast<phr::EngineTune&>(c->impl.tune), key);
    if (!f) return PHR_ERR_ARG;
    *value = *f;
    return PHR_OK;
}

void phr_ctx_destroy(phr_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->impl.device);
    cudaStreamSynchronize(c->impl.stream);
    delete c;
}

phr_status phr_ctx_set_timing(phr_ctx* c, int32_t enable) {
    if (!c) return PHR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->impl.mu);
    c->impl.timing = enable != 0;
    return PHR_OK;
}

uint32_t phr_ctx_get_timing(const phr_ctx* c, phr_kernel_timing* out, uint32_t max) {
    if (!c) return 0;
    uint32_t i = 0;
    for (const auto& kv : c->impl.timings) {
        if (out && i < max) {
            std::memset(&out[i], 0, sizeof(out[i]));
            std::strncpy(out[i].name, kv.first.c_str(), sizeof(out[i].name) - 1);
            out[i].launches = kv.second.first;
            out[i].total_ms = kv.second.second;
        }
        ++i;
    }
    return i;
}

void phr_ctx_reset_timing(phr_ctx* c) {
    if (!c) return;
    std::lock_guard<std::mutex> lk(c->impl.mu);
    c->impl.timings.clear();
    c->impl.counters.clear();
}

uint64_t phr_ctx_counter(const phr_ctx* c, const char* name) {
    if (!c || !name) return 0;
    phr_ctx* m = const_cast<phr_ctx*>(c);
    std::lock_guard<std::mutex> lk(m->impl.mu);
    auto it = m->impl.counters.find(name);
    return it == m->impl.counters.end() ? 0 : it->second;
}

void* phr_ctx_stream(const phr_ctx* c) { return c ? static_cast<void*>(c->impl.stream) : nullptr; }

const char* phr_ctx_last_error(const phr_ctx* c) { return c ? c->impl.last_error.c_str() : "null context"; }

uint64_t phr_ctx_kernel_launches(const phr_ctx* c) { return c ? c->impl.launches.load() : 0; }

phr_status phr_extend_batch(phr_ctx* c, phr_engine engine, const phr_pair_batch* batch, phr_affine_costs costs,
                            phr_result_arena* out) {
    if (check_ctx(c) != PHR_OK) return PHR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->impl.mu);
    cudaSetDevice(c->impl.device);
    return extend_host(c, engine, batch, costs, out);
}

phr_status phr_extend_batch_device(phr_ctx* c, phr_engine engine, const phr_pair_batch* batch,
                                   phr_affine_costs costs, phr_result_arena* out) {
    if (check_ctx(c) != PHR_OK) return PHR_ERR_ARG;
    Ctx* ctx = &c->impl;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!batch || !out) return phr::set_error(ctx, PHR_ERR_ARG, "NULL batch/arena");
    if (!valid_engine(engine)) return phr::set_error(ctx, PHR_ERR_ARG, "unknown engine");
    // sum of lengths (device arrays): one reduction kernel
    const uint64_t n = batch->n_pairs;
    out->cigar_used = 0;
    if (n == 0) return PHR_OK;
    cudaError_t e = cudaSuccess;
    const uint64_t sum_qt = phr::device_length_sum(ctx, batch->q_len, batch->t_len, n, &e);
    if (e != cudaSuccess) return phr::cuda_status(ctx, e, "length sum");
    phr::DevPairs dp;
    dp.n = n;
    dp.seq = batch->seq;
    dp.seq_bytes = batch->seq_bytes;
    dp.q_off = batch->q_off;
    dp.q_len = batch->q_len;
    dp.t_off = batch->t_off;
    dp.t_len = batch->t_len;
    dp.q_seed = batch->q_seed;
    dp.t_seed = batch->t_seed;
    phr::DevResults r;
    r.aln = out->aln;
    r.cigar = out->cigar;
    r.cigar_capacity = out->cigar_capacity;
    phr_status s = phr::run_extend(ctx, engine, dp, costs, &r, sum_qt);
    out->cigar_used = r.cigar_used;
    return s;
}

phr_status phr_extend_percall(phr_ctx* c, phr_engine engine, const phr_pair_batch* batch, phr_affine_costs costs,
                              phr_result_arena* out) {
    if (check_ctx(c) != PHR_OK) return PHR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->impl.mu);
    cudaSetDevice(c->impl.device);
    Ctx* ctx = &c->impl;
    if (!batch || !out) return phr::set_error(ctx, PHR_ERR_ARG, "NULL batch/arena");
    uint64_t used = 0;
    for (uint64_t i = 0; i < batch->n_pairs; ++i) {
        phr_pair_batch one = *batch;
        one.n_pairs = 1;
        one.q_off = batch->q_off + i;
        one.q_len = batch->q_len + i;
        one.t_off = batch->t_off + i;
        one.t_len = batch->t_len + i;
        one.q_seed = batch->q_seed ? batch->q_seed + i : nullptr;
        one.t_seed = batch->t_seed ? batch->t_seed + i : nullptr;
        phr_result_arena o;
        o.aln = out->aln + i;
        o.cigar = out->cigar + used;
        o.cigar_capacity = out->cigar_capacity - used;
        o.cigar_used = 0;
        phr_status s = extend_host(c, engine, &one, costs, &o);
        if (s != PHR_OK) return s;
        out->aln[i].cigar_off += used;
        used += o.cigar_used;
    }
    out->cigar_used = used;
    return PHR_OK;
}

}  // extern "C"
