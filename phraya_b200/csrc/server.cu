// server.cu -- serving loop over a device-resident index (phr_server_*).
//
// No counterpart in the reference (phraya's CLI aligns files in batches of 4096 reads,
// phraya-cli/src/main.rs:583-590). Requests are single reads. A scheduler thread forms
// batches continuously from two length buckets (short reads <= 500 bases ride the Myers
// path, long ones the WFA path): it fills a batch from one bucket up to
// max_batch_reads / max_batch_bases and hands it to an idle worker, which starts it once
// the device has the free memory the batch needs (cudaMemGetInfo minus the configured
// reserve). The scheduler itself makes no CUDA call, so nothing a worker waits on
// delays the dispatch of other batches.
//
// Each worker owns a context (its own CUDA stream, device arenas and pinned host
// buffers) and runs the whole align_read pipeline for its batch; workers overlap on the
// device and the index is shared read-only. With a short lane, worker 0 takes only
// short-read batches on a high-priority stream, and the other workers' persistent
// extension kernels keep to long_blocks_per_sm resident blocks per SM, so a long batch
// never holds every SM while short reads wait. Results are queued with their latency
// (submit -> result ready) and handed out by phr_server_poll.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "pipeline.cuh"


namespace {

// Servers raise the release threshold of their device's default memory pool to its
// maximum (freed memory stays in the pool, so workers growing and shrinking arenas never
// wait on unmapping while others run). Servers on one device share that setting: the
// first one saves the caller's threshold and the last one to go restores it.
struct PoolHold {
    int servers = 0;
    cudaMemPool_t pool = nullptr;
    uint64_t saved = 0;
};
std::mutex g_pool_mu;
PoolHold g_pool_hold[256];

bool pool_hold_acquire(int dev) {
    if (dev < 0 || dev >= 256) return false;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    PoolHold& h = g_pool_hold[dev];
    if (h.servers == 0) {
        cudaMemPool_t pool = nullptr;
        uint64_t saved = 0;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &saved) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        uint64_t keep = UINT64_MAX;
        if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        h.pool = pool;
        h.saved = saved;
    }
    ++h.servers;
    return true;
}

void pool_hold_release(int dev) {
    if (dev < 0 || dev >= 256) return;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    PoolHold& h = g_pool_hold[dev];
    if (h.servers <= 0) return;
    if (--h.servers == 0 && h.pool) {
        cudaMemPoolSetAttribute(h.pool, cudaMemPoolAttrReleaseThreshold, &h.saved);
        cudaGetLastError();
        h.pool = nullptr;
    }
}

// Restores the caller's current device when a server call returns.
struct DeviceRestore {
    int dev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    }
    ~DeviceRestore() {
        if (dev >= 0) cudaSetDevice(dev);
    }
};

}  // namespace

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id;
    std::vector<uint8_t> seq;
    Clock::time_point t0;
};

struct Done {
    phr_server_result res;
    std::vector<phr_alignment> aln;
    std::string cigar;
};

constexpr uint32_t kShortMax = 500;  // MYERS_MAX_QUERY_LEN (executor.rs:248)

// Grow-only pinned host buffer (page-locked, so the worker's copies are truly async).
struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    bool ensure(size_t need) {
        if (need <= cap) return true;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max(need + need / 2, static_cast<size_t>(1) << 20);
        if (cudaHostAlloc(&p, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cap = want;
        return true;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
};

}  // namespace

struct phr_server {
    phr::Ctx* owner = nullptr;
    const phr_index* idx = nullptr;
    phr_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work;   // scheduler: new requests / idle worker
    std::condition_variable cv_done;   // pollers: new results
    std::deque<Request> pending[2];    // per bucket: short, long
    std::deque<Done> done;
    uint64_t next_id = 1;
    uint64_t in_flight = 0;            // submitted, not yet completed
    uint64_t completions = 0;          // batches finished (admission waits on it)
    bool stopping = false;
    // this server holds a reference on its device's memory-pool setting (pool_hold_*)
    bool pool_held = false;
    bool short_lane = false;
    phr_status fatal = PHR_OK;
    std::string fatal_msg;
    struct Worker {
        phr::Ctx ctx;
        std::thread th;
        std::vector<Request> batch;
        bool busy = false;
        bool has_work = false;
        bool short_only = false;
        int index = 0;
        std::condition_variable cv;
        PinnedBuf seq, off, len, rr, aln, cig;
    };
    std::vector<Worker*> workers;
    std::thread scheduler;
    // PHRAYA_SERVER_TRACE=<file>: one line per batch:
    // worker bucket reads bases start_ms(since create) run_ms queued_ms(oldest read)
    FILE* trace = nullptr;
    std::mutex trace_mu;
    Clock::time_point t_create;
};

namespace {

void finish_batch(phr_server* S, phr_server::Worker* W, std::vector<Request>& batch, phr_status st,
                  const phr_read_result* rr, const phr_alignment* aln, const char* cig) {
    const auto t1 = Clock::now();
    const uint64_t n = batch.size();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (st != PHR_OK && S->fatal == PHR_OK) {
            S->fatal = st;
            S->fatal_msg = W->ctx.last_error;
        }
        for (uint64_t i = 0; i < n; ++i) {
            Done d{};
            d.res.request_id = batch[i].id;
            d.res.latency_us = std::chrono::duration<double, std::micro>(t1 - batch[i].t0).count();
            if (st == PHR_OK) {
                d.res.outcome = rr[i].outcome;
                d.res.has_result = rr[i].has_result;
                d.res.reverse = rr[i].reverse;
                d.res.n_aln = rr[i].n_aln;
                for (uint32_t k = 0; k < rr[i].n_aln; ++k) {
                    phr_alignment a = aln[rr[i].aln_off + k];
                    const uint64_t co = d.cigar.size();
                    d.cigar.append(cig + a.cigar_off, a.cigar_len);
                    a.cigar_off = co;
                    d.aln.push_back(a);
                }
            } else {
                d.res.outcome = PHR_OUT_NO_ALIGNMENT;
                d.res.has_result = 0;
                d.res.n_aln = 0;
            }
            S->done.push_back(std::move(d));
        }
        S->in_flight -= n;
        S->completions += 1;
        W->busy = false;
    }
    S->cv_done.notify_all();
    S->cv_work.notify_all();
}

// Device bytes one batch may add to a worker's arenas (upper estimate).
uint64_t batch_need(uint64_t n, uint64_t bases) {
    return phr::align_arena_need(n, bases, 0) + bases * 64 + (64ull << 20);
}

void run_worker(phr_server* S, phr_server::Worker* W) {
    cudaSetDevice(W->ctx.device);
    for (;;) {
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            W->cv.wait(lk, [&] { return W->has_work || S->stopping; });
            if (!W->has_work && S->stopping) return;
            batch.swap(W->batch);
            W->has_work = false;
        }
        // pack the batch into the worker's pinned buffers and run align_read on it
        const uint64_t n = batch.size();
        uint64_t bases = 0, maxlen = 1, cig_cap = 0;
        const uint32_t K = S->cfg.align.strategy == PHR_FAST ? 1 : S->cfg.align.strategy == PHR_BALANCED ? 2 : 50;
        for (auto& r : batch) {
            bases += r.seq.size();
            maxlen = std::max<uint64_t>(maxlen, r.seq.size());
        }
        const uint64_t acap = n * K + 16;
        // CIGAR text: each alignment of a read of length L spans at most L query bases
        // and, per the extension window, a bounded target stretch: 6 * L + 16 per alignment
        for (auto& r : batch) cig_cap += K * (6 * r.seq.size() + 16);
        cig_cap += 64;
        if (!W->seq.ensure(bases + 64) || !W->off.ensure(n * 8) || !W->len.ensure(n * 4) ||
            !W->rr.ensure(n * sizeof(phr_read_result)) || !W->aln.ensure(acap * sizeof(phr_alignment)) ||
            !W->cig.ensure(cig_cap)) {
            W->ctx.last_error = "pinned host buffer allocation failed";
            finish_batch(S, W, batch, PHR_ERR_OOM, nullptr, nullptr, nullptr);
            continue;
        }
        uint8_t* seq = W->seq.as<uint8_t>();
        uint64_t* off = W->off.as<uint64_t>();
        uint32_t* len = W->len.as<uint32_t>();
        uint64_t o = 0;
        for (uint64_t i = 0; i < n; ++i) {
            off[i] = o;
            len[i] = static_cast<uint32_t>(batch[i].seq.size());
            if (len[i]) std::memcpy(seq + o, batch[i].seq.data(), len[i]);
            o += len[i];
        }
        phr_read_batch rb{};
        rb.n_reads = n;
        rb.seq = seq;
        rb.seq_bytes = bases;
        rb.off = off;
        rb.len = len;
        phr_read_result_arena ar{W->rr.as<phr_read_result>(), W->aln.as<phr_alignment>(), acap, 0,
                                 W->cig.as<char>(), cig_cap, 0};
        if (!W->short_only) {
            // admission by free HBM: wait while a batch this size does not fit and another
            // worker may still free memory. The short lane skips it: its arenas were sized
            // for a full short batch at creation.
            const uint64_t need = batch_need(n, bases);
            for (;;) {
                size_t free_b = SIZE_MAX, total_b = 0;
                cudaMemGetInfo(&free_b, &total_b);
                if (free_b >= need + S->cfg.hbm_reserve_bytes) break;
                std::unique_lock<std::mutex> lk(S->mu);
                const bool others_busy = std::any_of(S->workers.begin(), S->workers.end(),
                                                     [&](auto* w) { return w != W && w->busy; });
                if (!others_busy || S->stopping) break;
                const uint64_t seen = S->completions;
                S->cv_work.wait(lk, [&] { return S->stopping || S->completions != seen; });
            }
        }
        const auto tb0 = Clock::now();
        const phr_status st = phr::align_reads_host(&W->ctx, S->idx, &rb, S->cfg.align, &ar, nullptr);
        if (S->trace) {
            const auto tb1 = Clock::now();
            Clock::time_point oldest = batch.empty() ? tb0 : batch[0].t0;
            for (auto& r : batch) oldest = std::min(oldest, r.t0);
            std::lock_guard<std::mutex> lk(S->trace_mu);
            std::string ph;
            for (auto& kv : W->ctx.timings)
                if (kv.second.second >= 0.5) ph += " " + kv.first + "=" + std::to_string(kv.second.second);
            W->ctx.timings.clear();
            std::fprintf(S->trace, "%d %d %llu %llu %.3f %.3f %.3f #%s\n", W->index,
                         batch.empty() ? -1 : (batch[0].seq.size() <= kShortMax ? 0 : 1),
                         static_cast<unsigned long long>(n), static_cast<unsigned long long>(bases),
                         std::chrono::duration<double, std::milli>(tb0 - S->t_create).count(),
                         std::chrono::duration<double, std::milli>(tb1 - tb0).count(),
                         std::chrono::duration<double, std::milli>(tb0 - oldest).count(), ph.c_str());
        }
        finish_batch(S, W, batch, st, W->rr.as<phr_read_result>(), W->aln.as<phr_alignment>(), W->cig.as<char>());
    }
}


void run_scheduler(phr_server* S) {
    std::unique_lock<std::mutex> lk(S->mu);
    // bucket an idle worker can take now: -1 none
    auto pick = [&](const phr_server::Worker* w) -> int {
        const bool s0 = !S->pending[0].empty(), s1 = !S->pending[1].empty();
        if (w->short_only) return s0 ? 0 : -1;
        // with a short lane, short reads are its alone: on a general worker a short batch
        // shares the SMs with long-read kernels on a low-priority stream and can wait for
        // them for tens of milliseconds
        if (S->short_lane) return s1 ? 1 : -1;
        if (s0 && s1) return S->pending[1].front().t0 < S->pending[0].front().t0 ? 1 : 0;
        if (s1) return 1;
        return s0 ? 0 : -1;
    };
    auto ready = [&]() -> bool {
        for (auto* w : S->workers)
            if (!w->busy && pick(w) >= 0) return true;
        return false;
    };
    for (;;) {
        S->cv_work.wait(lk, [&] {
            return ready() || (S->stopping && S->pending[0].empty() && S->pending[1].empty());
        });
        if (S->stopping && S->pending[0].empty() && S->pending[1].empty()) {
            for (auto* w : S->workers) w->cv.notify_all();
            return;
        }
        phr_server::Worker* W = nullptr;
        int b = -1;
        for (auto* w : S->workers)
            if (!w->busy && (b = pick(w)) >= 0) {
                W = w;
                break;
            }
        if (!W) continue;
        // batch-forming window: give late arrivals max_wait_us to join a partial batch
        const auto deadline = S->pending[b].front().t0 + std::chrono::microseconds(S->cfg.max_wait_us);
        while (!S->stopping && S->pending[b].size() < S->cfg.max_batch_reads && Clock::now() < deadline)
            S->cv_work.wait_until(lk, deadline);
        if (S->pending[b].empty() || W->busy) continue;
        std::vector<Request> batch;
        uint64_t bases = 0;
        while (!S->pending[b].empty() && batch.size() < S->cfg.max_batch_reads) {
            const uint64_t l = S->pending[b].front().seq.size();
            if (!batch.empty() && bases + l > S->cfg.max_batch_bases) break;
            bases += l;
            batch.push_back(std::move(S->pending[b].front()));
            S->pending[b].pop_front();
        }
        // (admission by free HBM happens in the worker: a query of free memory can take
        // tens of milliseconds while other threads allocate, and this thread must keep
        // handing short reads to the short lane meanwhile)
        W->batch = std::move(batch);
        W->busy = true;
        W->has_work = true;
        W->cv.notify_all();
    }
}

void enqueue_locked(phr_server* S, const uint8_t* read, uint32_t len, Clock::time_point t0, uint64_t* id) {
    Request r;
    r.seq.assign(read, read + len);
    r.t0 = t0;
    r.id = S->next_id++;
    *id = r.id;
    S->pending[len <= kShortMax ? 0 : 1].push_back(std::move(r));
    S->in_flight += 1;
}

}  // namespace

extern "C" {

phr_status phr_server_create(phr_ctx* c, const phr_index* idx, const phr_server_config* cfg, phr_server** out) {
    if (!c || !idx || !out) return PHR_ERR_ARG;
    *out = nullptr;
    phr_server* S = new phr_server();
    S->owner = &c->impl;
    S->idx = idx;
    if (cfg) S->cfg = *cfg;
    if (S->cfg.max_batch_reads == 0) S->cfg.max_batch_reads = 4096;
    if (S->cfg.max_batch_bases == 0) S->cfg.max_batch_bases = 16ull << 20;
    if (S->cfg.hbm_reserve_bytes == 0) S->cfg.hbm_reserve_bytes = 2ull << 30;
    if (S->cfg.n_streams == 0) S->cfg.n_streams = 2;
    if (S->cfg.align.strategy < PHR_FAST || S->cfg.align.strategy > PHR_SENSITIVE) {
        delete S;
        return PHR_ERR_ARG;
    }
    S->short_lane = S->cfg.short_lane > 0 || (S->cfg.short_lane == 0 && S->cfg.n_streams >= 2);
    if (S->cfg.long_blocks_per_sm == 0) S->cfg.long_blocks_per_sm = 2;
    if (S->cfg.long_blocks_per_sm > 4) {
        delete S;
        return PHR_ERR_ARG;
    }
    DeviceRestore restore_device;
    int prio_low = 0, prio_high = 0;
    cudaSetDevice(c->impl.device);
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    // workers' arenas grow and shrink through the device's default memory pool; keeping
    // freed memory in the pool (no release threshold) spares them unmapping and mapping it
    // again while other workers run
    S->pool_held = pool_hold_acquire(c->impl.device);
    cudaGetLastError();
    for (uint32_t w = 0; w < S->cfg.n_streams; ++w) {
        auto* W = new phr_server::Worker();
        W->ctx.device = c->impl.device;
        W->ctx.sm_count = c->impl.sm_count;
        W->ctx.tune = c->impl.tune;
        W->ctx.scratch_budget = c->impl.scratch_budget;
        W->short_only = S->short_lane && w == 0;
        W->index = static_cast<int>(w);
        if (S->short_lane && w > 0)
            W->ctx.tune.max_blocks_per_sm = std::min<int>(W->ctx.tune.max_blocks_per_sm,
                                                          static_cast<int>(S->cfg.long_blocks_per_sm));
        const int prio = W->short_only ? prio_high : prio_low;
        if (cudaStreamCreateWithPriority(&W->ctx.stream, cudaStreamNonBlocking, prio) != cudaSuccess) {
            delete W;
            for (auto* x : S->workers) delete x;
            if (S->pool_held) pool_hold_release(c->impl.device);
            delete S;
            return PHR_ERR_CUDA;
        }
        W->ctx.bind_stream();
        W->ctx.timing = std::getenv("PHRAYA_SERVER_TRACE") != nullptr;
        // Device arenas and host buffers for a full batch up front: growing them while
        // serving (allocation, page-locking) stalls every worker on the device.
        {
            const uint64_t nr = S->cfg.max_batch_reads;
            const uint64_t nb = W->short_only ? std::min<uint64_t>(S->cfg.max_batch_bases, nr * kShortMax)
                                              : S->cfg.max_batch_bases;
            W->ctx.pipe.reserve(phr::align_arena_need(nr, nb, 0) + nb + nr * 32);
            W->ctx.seeds.reserve(nb * 40 + (16ull << 20));
            W->ctx.io.reserve(nb * 16 + nr * 1024 + (16ull << 20));
            W->ctx.arena.reserve(nb * 24 + nr * 2048 + (96ull << 20));
            W->ctx.scratch.reserve(std::min<uint64_t>(W->ctx.scratch_budget, W->short_only ? (512ull << 20) : (4ull << 30)));
            cudaGetLastError();
            const uint32_t K = S->cfg.align.strategy == PHR_FAST ? 1 : S->cfg.align.strategy == PHR_BALANCED ? 2 : 50;
            W->seq.ensure(nb + 64);
            W->off.ensure(nr * 8);
            W->len.ensure(nr * 4);
            W->rr.ensure(nr * sizeof(phr_read_result));
            W->aln.ensure((nr * K + 16) * sizeof(phr_alignment));
            W->cig.ensure(std::min<uint64_t>(K * (6 * nb + 16 * nr) + 64, 256ull << 20));
        }
        S->workers.push_back(W);
    }
    S->t_create = Clock::now();
    if (const char* tp = std::getenv("PHRAYA_SERVER_TRACE")) S->trace = std::fopen(tp, "w");
    for (auto* W : S->workers) W->th = std::thread(run_worker, S, W);
    S->scheduler = std::thread(run_scheduler, S);
    *out = S;
    return PHR_OK;
}

phr_status phr_server_submit(phr_server* S, const uint8_t* read, uint32_t len, uint64_t* request_id) {
    if (!S || (!read && len) || !request_id) return PHR_ERR_ARG;
    const auto t0 = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) return PHR_ERR_STATE;
        if (S->fatal != PHR_OK) return S->fatal;
        enqueue_locked(S, read, len, t0, request_id);
    }
    S->cv_work.notify_all();
    return PHR_OK;
}

phr_status phr_server_submit_many(phr_server* S, const uint8_t* seq, const uint64_t* off, const uint32_t* len,
                                  uint64_t n, uint64_t* ids) {
    if (!S || (n && (!seq || !off || !len || !ids))) return PHR_ERR_ARG;
    const auto t0 = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) return PHR_ERR_STATE;
        if (S->fatal != PHR_OK) return S->fatal;
        for (uint64_t i = 0; i < n; ++i) enqueue_locked(S, seq + off[i], len[i], t0, ids + i);
    }
    S->cv_work.notify_all();
    return PHR_OK;
}

phr_status phr_server_poll(phr_server* S, phr_server_result* res, uint32_t max_results, phr_alignment* aln,
                           uint64_t aln_capacity, char* cigar, uint64_t cigar_capacity, uint32_t wait_us,
                           uint32_t* n_out) {
    if (!S || !n_out || (max_results && !res)) return PHR_ERR_ARG;
    *n_out = 0;
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->done.empty() && wait_us > 0)
        S->cv_done.wait_for(lk, std::chrono::microseconds(wait_us), [&] { return !S->done.empty(); });
    uint64_t ao = 0, co = 0;
    uint32_t k = 0;
    while (k < max_results && !S->done.empty()) {
        Done& d = S->done.front();
        if (ao + d.aln.size() > aln_capacity || co + d.cigar.size() > cigar_capacity) {
            if (k == 0) return PHR_ERR_CAPACITY;
            break;
        }
        res[k] = d.res;
        for (auto a : d.aln) {
            a.cigar_off += co;
            aln[ao++] = a;
        }
        if (!d.cigar.empty()) std::memcpy(cigar + co, d.cigar.data(), d.cigar.size());
        co += d.cigar.size();
        S->done.pop_front();
        ++k;
    }
    *n_out = k;
    return S->fatal;
}

phr_status phr_server_destroy(phr_server* S) {
    if (!S) return PHR_ERR_ARG;
    DeviceRestore restore_device;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        // drain: every submitted request completes before the workers stop
        S->cv_done.wait(lk, [&] { return S->in_flight == 0 || S->fatal != PHR_OK; });
        S->stopping = true;
    }
    S->cv_work.notify_all();
    for (auto* W : S->workers) W->cv.notify_all();
    if (S->scheduler.joinable()) S->scheduler.join();
    for (auto* W : S->workers) {
        W->cv.notify_all();
        if (W->th.joinable()) W->th.join();
    }
    const phr_status st = S->fatal;
    if (S->trace) std::fclose(S->trace);
    for (auto* W : S->workers) {
        cudaSetDevice(W->ctx.device);
        cudaStreamSynchronize(W->ctx.stream);
        delete W;
    }
    if (S->pool_held) pool_hold_release(S->owner->device);
    delete S;
    return st;
}

}  // extern "C"
