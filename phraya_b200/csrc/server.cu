// server.cu -- serving loop over a device-resident index (phr_server_*).
//
// No counterpart in the reference (phraya's CLI aligns files in batches of 4096 reads,
// phraya-cli/src/main.rs:583-590). Requests are single reads. A scheduler thread forms
// batches continuously: it takes the oldest pending request's length bucket (short
// reads <= 500 bases ride the Myers path, long ones the WFA path), fills a batch from
// that bucket up to max_batch_reads / max_batch_bases, and hands it to the first idle
// worker once the device has the free memory the batch needs (cudaMemGetInfo minus the
// configured reserve). Each worker owns a context (its own CUDA stream and device
// arenas) and runs the whole align_read pipeline for its batch; workers overlap on the
// device. The index is shared read-only. Results are queued with their latency
// (submit -> result ready) and handed out by phr_server_poll.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "pipeline.cuh"

namespace phr {
phr_status align_reads_host(Ctx* ctx, const phr_index* idx, const phr_read_batch* rb, const phr_align_config& cfg,
                            phr_read_result_arena* out, phr_align_stats* stats);
}

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
    phr_status fatal = PHR_OK;
    std::string fatal_msg;
    struct Worker {
        phr::Ctx ctx;
        std::thread th;
        std::vector<Request> batch;
        bool busy = false;
        bool has_work = false;
        std::condition_variable cv;
    };
    std::vector<Worker*> workers;
    std::thread scheduler;
};

namespace {

uint64_t batch_bytes(const std::vector<Request>& b) {
    uint64_t s = 0;
    for (auto& r : b) s += r.seq.size();
    return s;
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
        // pack the batch and run align_read for all of it
        const uint64_t n = batch.size();
        std::vector<uint8_t> seq;
        std::vector<uint64_t> off(n);
        std::vector<uint32_t> len(n);
        for (uint64_t i = 0; i < n; ++i) {
            off[i] = seq.size();
            len[i] = static_cast<uint32_t>(batch[i].seq.size());
            seq.insert(seq.end(), batch[i].seq.begin(), batch[i].seq.end());
        }
        phr_read_batch rb{};
        rb.n_reads = n;
        rb.seq = seq.data();
        rb.seq_bytes = seq.size();
        rb.off = off.data();
        rb.len = len.data();
        const uint32_t K = S->cfg.align.strategy == PHR_FAST ? 1 : S->cfg.align.strategy == PHR_BALANCED ? 2 : 50;
        std::vector<phr_read_result> rr(n);
        std::vector<phr_alignment> aln(n * K + 16);
        uint64_t maxlen = 1;
        for (auto l : len) maxlen = std::max<uint64_t>(maxlen, l);
        std::vector<char> cig(aln.size() * (6 * maxlen + 16));
        phr_read_result_arena ar{rr.data(), aln.data(), aln.size(), 0, cig.data(), cig.size(), 0};
        phr_status st = phr::align_reads_host(&W->ctx, S->idx, &rb, S->cfg.align, &ar, nullptr);
        const auto t1 = Clock::now();
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
                        d.cigar.append(cig.data() + a.cigar_off, a.cigar_len);
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
}

// Device bytes one batch may add to a worker's arenas (upper estimate).
uint64_t batch_need(uint64_t n, uint64_t bases) {
    return phr::align_arena_need(n, bases, 0) + bases * 64 + (64ull << 20);
}

void run_scheduler(phr_server* S) {
    cudaSetDevice(S->owner->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_work.wait(lk, [&] {
            return S->stopping || ((!S->pending[0].empty() || !S->pending[1].empty()) &&
                                   std::any_of(S->workers.begin(), S->workers.end(), [](auto* w) { return !w->busy; }));
        });
        const bool have = !S->pending[0].empty() || !S->pending[1].empty();
        if (!have && S->stopping) {
            for (auto* w : S->workers) w->cv.notify_all();
            return;
        }
        if (!have) continue;
        // oldest request decides the bucket
        int b = 0;
        if (S->pending[0].empty()) b = 1;
        else if (!S->pending[1].empty() && S->pending[1].front().t0 < S->pending[0].front().t0) b = 1;
        // batch-forming window: give late arrivals max_wait_us to join a partial batch
        const auto deadline = S->pending[b].front().t0 + std::chrono::microseconds(S->cfg.max_wait_us);
        while (!S->stopping && S->pending[b].size() < S->cfg.max_batch_reads && Clock::now() < deadline) {
            S->cv_work.wait_until(lk, deadline);
        }
        if (S->pending[b].empty()) continue;
        phr_server::Worker* W = nullptr;
        for (auto* w : S->workers)
            if (!w->busy) {
                W = w;
                break;
            }
        if (!W) continue;
        std::vector<Request> batch;
        uint64_t bases = 0;
        while (!S->pending[b].empty() && batch.size() < S->cfg.max_batch_reads) {
            const uint64_t l = S->pending[b].front().seq.size();
            if (!batch.empty() && bases + l > S->cfg.max_batch_bases) break;
            bases += l;
            batch.push_back(std::move(S->pending[b].front()));
            S->pending[b].pop_front();
        }
        // admission by free HBM: wait while a batch this size does not fit
        size_t free_b = 0, total_b = 0;
        lk.unlock();
        cudaMemGetInfo(&free_b, &total_b);
        lk.lock();
        const uint64_t need = batch_need(batch.size(), bases);
        const bool others_busy =
            std::any_of(S->workers.begin(), S->workers.end(), [](auto* w) { return w->busy; });
        if (free_b < need + S->cfg.hbm_reserve_bytes && others_busy) {
            // put the batch back (front, same order) and wait for a worker to finish
            for (auto it = batch.rbegin(); it != batch.rend(); ++it) S->pending[b].push_front(std::move(*it));
            const uint64_t seen = S->completions;
            S->cv_work.wait(lk, [&] { return S->stopping || S->completions != seen; });
            continue;
        }
        W->batch = std::move(batch);
        W->busy = true;
        W->has_work = true;
        W->cv.notify_all();
    }
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
    for (uint32_t w = 0; w < S->cfg.n_streams; ++w) {
        auto* W = new phr_server::Worker();
        W->ctx.device = c->impl.device;
        W->ctx.sm_count = c->impl.sm_count;
        W->ctx.tune = c->impl.tune;
        W->ctx.scratch_budget = c->impl.scratch_budget;
        cudaSetDevice(W->ctx.device);
        if (cudaStreamCreateWithFlags(&W->ctx.stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete W;
            for (auto* x : S->workers) delete x;
            delete S;
            return PHR_ERR_CUDA;
        }
        S->workers.push_back(W);
    }
    for (auto* W : S->workers) W->th = std::thread(run_worker, S, W);
    S->scheduler = std::thread(run_scheduler, S);
    *out = S;
    return PHR_OK;
}

phr_status phr_server_submit(phr_server* S, const uint8_t* read, uint32_t len, uint64_t* request_id) {
    if (!S || (!read && len) || !request_id) return PHR_ERR_ARG;
    Request r;
    r.seq.assign(read, read + len);
    r.t0 = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) return PHR_ERR_STATE;
        if (S->fatal != PHR_OK) return S->fatal;
        r.id = S->next_id++;
        *request_id = r.id;
        S->pending[len <= kShortMax ? 0 : 1].push_back(std::move(r));
        S->in_flight += 1;
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
    for (auto* W : S->workers) {
        cudaSetDevice(W->ctx.device);
        cudaStreamSynchronize(W->ctx.stream);
        delete W;
    }
    delete S;
    return st;
}

}  // extern "C"
