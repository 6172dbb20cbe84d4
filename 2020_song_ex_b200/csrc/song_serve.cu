// song_serve.cu -- serving loop with continuous batching (host side).
//
// A persistent kernel (serve_kernel in song_serve_kernel.inc) keeps one
// request per warp.  The host publishes requests into a device-resident
// ring with stream-ordered copies (payload first, then the new tail), so a
// request that arrives while others are running is claimed by the first
// warp that finishes -- admission is bounded by the warps that fit in
// shared memory (one slot each, sized for max_ef) and by the ring, sized by
// the HBM budget.  Results are written by the kernel into mapped pinned
// host memory and published by a per-slot done ticket.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "song_b200.h"
#include "song_kernels.cuh"

struct song_server {
    song_index* idx = nullptr;
    song_server_config cfg{};
    song::ServeArgs s{};
    int dim = 0, num_sms = 0, device = 0, cap_limit = 0, warps = 0;
    int slots = 0, slot_bytes = 0;
    unsigned char* d_ring = nullptr;
    long long* d_ctrl = nullptr;       // [0] head, [1] tail, [2] stop, [3] last claim time,
                                       // [4..6] warps that left idle / at the poll cap / at stop
    unsigned char* h_stage = nullptr;  // pinned staging of ring slots
    long long* h_tailbuf = nullptr;    // pinned tail values, one per slot
    long long* h_stop = nullptr;       // pinned source of the stop word
    int32_t* h_ids = nullptr;          // mapped [slots x max_k]
    float* h_dist = nullptr;           // mapped [slots x max_k]
    song_query_trace* h_trace = nullptr;  // mapped [slots]
    long long* h_done = nullptr;       // mapped [slots]
    int32_t* d_scand = nullptr;        // entry-stage candidates per slot (learned model with hubs)
    float* d_sdist = nullptr;
    void* d_split = nullptr;           // the entry stage's split scratch (batches <= 128)
    size_t split_bytes = 0;
    cudaStream_t kst = nullptr, cst = nullptr;
    cudaEvent_t kdone = nullptr;
    cudaEvent_t pubdone = nullptr;  // the last publish's copies (and entry stage) are done
    bool launched = false;
    long long launches = 0;
    long long next = 0;  // next ticket
    std::mutex mu;
};

namespace {

constexpr int kEntrySms = 8;  // SMs the serving kernel leaves to the entry stage

song_status cuda_err(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return song::set_error(e == cudaErrorMemoryAllocation ? SONG_ERR_OOM : SONG_ERR_CUDA, m.c_str());
}

#define SRV_CUDA(call, what)                              \
    do {                                                  \
        cudaError_t _e = (call);                          \
        if (_e != cudaSuccess) return cuda_err(_e, what); \
    } while (0)

long long load_done(const song_server* v, int slot) {
    return reinterpret_cast<const std::atomic<long long>*>(v->h_done + slot)->load(std::memory_order_acquire);
}

bool slot_free(const song_server* v, long long t) {
    return t < v->slots || load_done(v, (int)(t % v->slots)) == t - v->slots;
}

// (Re)launch the persistent kernel if it is not running.
song_status ensure_running(song_server* v) {
    if (v->launched && cudaEventQuery(v->kdone) == cudaErrorNotReady) return SONG_OK;
    // with an entry stage, some SMs stay free for its kernel (launched on the copy
    // stream while this persistent kernel runs)
    const int reserve = v->d_scand != nullptr ? kEntrySms : 0;
    cudaError_t e = song::launch_serve(v->s, v->num_sms, v->cfg.max_ctas, reserve, v->kst, &v->warps);
    if (e != cudaSuccess) return cuda_err(e, "serve launch");
    SRV_CUDA(cudaEventRecord(v->kdone, v->kst), "event");
    v->launched = true;
    v->launches += 1;
    return SONG_OK;
}

void free_server(song_server* v) {
    if (!v) return;
    if (v->h_stop && v->d_ctrl && v->cst) {  // every warp exits at its next poll
        *v->h_stop = 1;
        cudaMemcpyAsync(v->d_ctrl + 2, v->h_stop, 8, cudaMemcpyHostToDevice, v->cst);
        cudaStreamSynchronize(v->cst);
    }
    if (v->kst) cudaStreamSynchronize(v->kst);
    if (v->cst) cudaStreamSynchronize(v->cst);
    cudaFree(v->d_ring);
    cudaFree(v->d_ctrl);
    cudaFree(v->d_scand);
    cudaFree(v->d_sdist);
    cudaFree(v->d_split);
    cudaFreeHost(v->h_stage);
    cudaFreeHost(v->h_tailbuf);
    cudaFreeHost(v->h_stop);
    cudaFreeHost(v->h_ids);
    cudaFreeHost(v->h_dist);
    cudaFreeHost(v->h_trace);
    cudaFreeHost(v->h_done);
    if (v->kdone) cudaEventDestroy(v->kdone);
    if (v->pubdone) cudaEventDestroy(v->pubdone);
    if (v->kst) cudaStreamDestroy(v->kst);
    if (v->cst) cudaStreamDestroy(v->cst);
    delete v;
}

// Stage requests [t0, t0+n) and publish them (payload copies, then the tail).
song_status publish(song_server* v, long long t0, const float* q, int n, const int* ks,
                    const int* efs, const int* flags) {
    const int pq = song::index_pq_size(v->idx);
    const int limit = std::min(v->cfg.max_ef, pq);
    for (int i = 0; i < n; ++i) {
        const long long t = t0 + i;
        const int slot = (int)(t % v->slots);
        unsigned char* p = v->h_stage + (size_t)slot * v->slot_bytes;
        int ef = efs ? efs[i] : limit;
        const int k = ks ? ks[i] : 10;
        if (ef < k) ef = k;  // gpu_search's clamp (kernalGraph.h:315-316)
        if (ef > limit) ef = limit;
        const int cap = ef < 1 ? 1 : ef;
        long long* hl = reinterpret_cast<long long*>(p);
        int* hi = reinterpret_cast<int*>(p);
        hl[0] = t;
        hi[2] = k;
        hi[3] = cap;
        hi[4] = flags ? flags[i] : 0;
        std::memcpy(p + song::kServeHeader, q + (size_t)i * v->dim, (size_t)v->dim * 4);
    }
    long long t = t0;
    while (t < t0 + n) {  // contiguous runs of slots
        const int slot = (int)(t % v->slots);
        const long long run = std::min<long long>(t0 + n - t, v->slots - slot);
        SRV_CUDA(cudaMemcpyAsync(v->d_ring + (size_t)slot * v->slot_bytes,
                                 v->h_stage + (size_t)slot * v->slot_bytes,
                                 (size_t)run * v->slot_bytes, cudaMemcpyHostToDevice, v->cst),
                 "request copy");
        if (v->d_scand != nullptr)  // the entry stage for these slots, before the tail is published
            SRV_CUDA(song::index_entry(v->idx,
                                       reinterpret_cast<const float*>(v->d_ring + (size_t)slot * v->slot_bytes +
                                                                      song::kServeHeader),
                                       v->slot_bytes / 4, (int)run,
                                       v->d_scand + (size_t)slot * song::kEntryK,
                                       v->d_sdist + (size_t)slot * song::kEntryK, v->cst,
                                       v->d_split, v->split_bytes),
                     "entry stage");
        t += run;
    }
    const int last = (int)((t0 + n - 1) % v->slots);
    v->h_tailbuf[last] = t0 + n;
    SRV_CUDA(cudaMemcpyAsync(v->d_ctrl + 1, v->h_tailbuf + last, 8, cudaMemcpyHostToDevice, v->cst),
             "tail copy");
    SRV_CUDA(cudaEventRecord(v->pubdone, v->cst), "event");
    return ensure_running(v);
}

}  // namespace

extern "C" {

void song_server_config_default(song_server_config* c) {
    if (!c) return;
    c->max_k = 100;
    c->max_ef = 256;
    c->precision = SONG_PREC_FP32;
    c->stop_threshold = 0.85f;
    c->ring_slots = 4096;
    c->hbm_budget = 0;
    c->max_ctas = 0;
    c->idle_exit_us = 200000;
}

song_status song_server_create(song_index* index, const song_server_config* cfg,
                               song_server** out) {
    if (!index || !cfg || !out) return song::set_error(SONG_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (cfg->max_k < 1 || cfg->max_ef < 1 || cfg->ring_slots < 1 || cfg->idle_exit_us < 1)
        return song::set_error(SONG_ERR_INVALID_ARG, "bad server config");
    if (cfg->max_ef > 1024) return song::set_error(SONG_ERR_UNSUPPORTED, "max_ef above 1024");
    song_server* v = new (std::nothrow) song_server();
    if (!v) return song::set_error(SONG_ERR_OOM, "host allocation failed");
    v->idx = index;
    v->cfg = *cfg;
    song_search_opts opts{};
    opts.precision = cfg->precision;
    song::SearchArgs a;
    song_status st = song::server_args(index, &opts, cfg->max_k, cfg->max_ef, &a, &v->num_sms, &v->device);
    if (st != SONG_OK) {
        delete v;
        return st;
    }
    const float thr = cfg->stop_threshold;
    a.stop_thr = thr <= 0.0f ? -INFINITY : (thr >= 1.0f ? INFINITY : std::log(thr / (1.0f - thr)));
    v->dim = song::index_dim(index);
    v->slot_bytes = (song::kServeHeader + v->dim * 4 + 15) / 16 * 16;
    long long slots = cfg->ring_slots;
    if (cfg->hbm_budget > 0) slots = std::min<long long>(slots, cfg->hbm_budget / v->slot_bytes);
    if (slots < 1) {
        delete v;
        return song::set_error(SONG_ERR_BUDGET, "hbm_budget holds no request slot");
    }
    v->slots = (int)slots;
    cudaError_t e = cudaSetDevice(v->device);
    const size_t nk = (size_t)v->slots * cfg->max_k;
    if (e == cudaSuccess) e = cudaMalloc(&v->d_ring, (size_t)v->slots * v->slot_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&v->d_ctrl, 64);
    if (e == cudaSuccess) e = cudaMemset(v->d_ctrl, 0, 64);
    if (e == cudaSuccess) e = cudaHostAlloc(&v->h_stage, (size_t)v->slots * v->slot_bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&v->h_tailbuf, (size_t)v->slots * 8, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&v->h_stop, 64, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&v->h_ids, nk * 4, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&v->h_dist, nk * 4, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&v->h_trace, (size_t)v->slots * sizeof(song_query_trace), cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&v->h_done, (size_t)v->slots * 8, cudaHostAllocMapped);
    if (e == cudaSuccess && song::index_model_staged(index)) {
        e = cudaMalloc(&v->d_scand, (size_t)v->slots * song::kEntryK * 4);
        if (e == cudaSuccess) e = cudaMalloc(&v->d_sdist, (size_t)v->slots * song::kEntryK * 4);
        v->split_bytes = song::entry_split_scratch_bytes(128, v->num_sms);
        if (e == cudaSuccess) e = cudaMalloc(&v->d_split, v->split_bytes);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&v->kst, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&v->cst, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&v->kdone, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&v->pubdone, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        song_status s2 = cuda_err(e, "server allocation");
        free_server(v);
        return s2;
    }
    *v->h_stop = 0;
    for (int i = 0; i < v->slots; ++i) v->h_done[i] = -1;
    song::ServeArgs& s = v->s;
    s.base = a;
    s.ring = v->d_ring;
    s.slot_bytes = v->slot_bytes;
    s.slots = v->slots;
    s.max_k = cfg->max_k;
    s.head = v->d_ctrl;
    s.tail = v->d_ctrl + 1;
    s.stop = v->d_ctrl + 2;
    s.res_ids = v->h_ids;
    s.res_dist = v->h_dist;
    s.res_trace = v->h_trace;
    s.res_done = v->h_done;
    s.last_claim = v->d_ctrl + 3;
    s.exits = v->d_ctrl + 4;
    s.scand = v->d_scand;
    s.sdist = v->d_sdist;
    s.idle_ns = (long long)cfg->idle_exit_us * 1000;
    s.sleep_ns = 2000;
    // hard bound: 64x the polls the idle time allows at the longest backoff
    s.max_idle_polls = (int)std::min<long long>(INT32_MAX, (long long)cfg->idle_exit_us * 32);
    *out = v;
    return SONG_OK;
}

song_status song_server_submit(song_server* v, const float* queries, int n, const int* ks,
                               const int* efs, const int* flags, long long* first_ticket) {
    if (!v || !queries || n < 1) return song::set_error(SONG_ERR_INVALID_ARG, "bad submit");
    if (ks)
        for (int i = 0; i < n; ++i)
            if (ks[i] < 0 || ks[i] > v->cfg.max_k)
                return song::set_error(SONG_ERR_INVALID_ARG, "k outside [0, max_k]");
    if (flags)
        for (int i = 0; i < n; ++i)
            if ((flags[i] & SONG_REQ_LEARNED) && !song::index_has_model(v->idx))
                return song::set_error(SONG_ERR_INVALID_ARG, "learned request but no model attached");
    std::lock_guard<std::mutex> lock(v->mu);
    if (n > v->slots) return song::set_error(SONG_ERR_BUDGET, "more requests than ring slots");
    for (int i = 0; i < n; ++i)
        if (!slot_free(v, v->next + i))
            return song::set_error(SONG_ERR_BUDGET, "request ring full (earlier requests still running)");
    const long long t0 = v->next;
    song_status st = publish(v, t0, queries, n, ks, efs, flags);
    if (st != SONG_OK) return st;
    v->next += n;
    if (first_ticket) *first_ticket = t0;
    return SONG_OK;
}

song_status song_server_poll(song_server* v, long long ticket, int32_t* ids, float* dists,
                             song_query_trace* trace, int* done) {
    if (!v || !done || ticket < 0) return song::set_error(SONG_ERR_INVALID_ARG, "bad poll");
    *done = 0;
    const int slot = (int)(ticket % v->slots);
    const long long d = load_done(v, slot);
    if (d == ticket) {
        if (ids) std::memcpy(ids, v->h_ids + (size_t)slot * v->cfg.max_k, (size_t)v->cfg.max_k * 4);
        if (dists) std::memcpy(dists, v->h_dist + (size_t)slot * v->cfg.max_k, (size_t)v->cfg.max_k * 4);
        if (trace) *trace = v->h_trace[slot];
        *done = 1;
        return SONG_OK;
    }
    if (d > ticket) return song::set_error(SONG_ERR_INVALID_ARG, "ticket's slot was reused");
    std::lock_guard<std::mutex> lock(v->mu);
    if (ticket >= v->next) return song::set_error(SONG_ERR_INVALID_ARG, "ticket not submitted");
    return ensure_running(v);
}

song_status song_server_wait(song_server* v, long long ticket, long long timeout_us, int32_t* ids,
                             float* dists, song_query_trace* trace) {
    using clk = std::chrono::steady_clock;
    if (!v || ticket < 0 || timeout_us < 0) return song::set_error(SONG_ERR_INVALID_ARG, "bad wait");
    const auto deadline = clk::now() + std::chrono::microseconds(timeout_us);
    for (long long spins = 0;; ++spins) {
        int done = 0;
        if (song_status st = song_server_poll(v, ticket, ids, dists, trace, &done)) return st;
        if (done) return SONG_OK;
        if (clk::now() >= deadline) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "ticket %lld not finished within %lld us", ticket, timeout_us);
            return song::set_error(SONG_ERR_TIMEOUT, buf);
        }
        if (spins > 64) std::this_thread::yield();
    }
}

song_status song_server_get_stats(song_server* v, song_server_stats* out) {
    if (!v || !out) return song::set_error(SONG_ERR_INVALID_ARG, "bad stats call");
    std::lock_guard<std::mutex> lock(v->mu);
    long long ex[3] = {0, 0, 0};
    SRV_CUDA(cudaMemcpyAsync(ex, v->d_ctrl + 4, sizeof ex, cudaMemcpyDeviceToHost, v->cst), "stats copy");
    SRV_CUDA(cudaStreamSynchronize(v->cst), "stats copy");
    out->launches = v->launches;
    out->idle_exits = ex[0];
    out->poll_cap_exits = ex[1];
    out->stop_exits = ex[2];
    out->running = (v->launched && cudaEventQuery(v->kdone) == cudaErrorNotReady) ? 1 : 0;
    return SONG_OK;
}

song_status song_server_run_poisson(song_server* v, const float* queries, int nq, const int* ks,
                                    const int* efs, const int* flags, double rate_qps,
                                    unsigned seed, double* latency_ms, int32_t* ids_out,
                                    double* wall_s) {
    using clk = std::chrono::steady_clock;
    if (!v || !queries || nq < 1 || !(rate_qps > 0) || !latency_ms)
        return song::set_error(SONG_ERR_INVALID_ARG, "bad run_poisson arguments");
    std::vector<double> arrive(nq);
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rate_qps);
    double t = 0.0;
    for (int i = 0; i < nq; ++i) {
        t += gap(rng);
        arrive[i] = t;
    }
    std::vector<char> seen(nq, 0);
    std::lock_guard<std::mutex> lock(v->mu);
    const long long first = v->next;
    int sub = 0, lo = 0, ndone = 0;
    const auto t0 = clk::now();
    double last = 0.0;
    long long spins = 0;
    // Continuous batching of arrivals: a batch is published once the oldest
    // pending request has waited 20 us and the previous publish (its copies
    // and, with a learned entry stage, that stage's kernels) has finished, or
    // at once when 128 are pending (one tile of the entry stage).  Under load
    // the batches grow instead of the publishes queueing up.
    constexpr int kBatch = 128;
    constexpr double kWindow = 20e-6;
    while (ndone < nq) {
        const double now = std::chrono::duration<double>(clk::now() - t0).count();
        int m = 0;
        while (sub + m < nq && arrive[sub + m] <= now) {
            const long long tk = first + sub + m;
            // the slot's previous request must have been consumed
            if (tk - first >= v->slots && !seen[tk - first - v->slots]) break;
            ++m;
        }
        if (m > kBatch) m = kBatch;
        const bool last_batch = sub + m == nq;
        const bool idle = cudaEventQuery(v->pubdone) != cudaErrorNotReady;
        if (m > 0 && (m >= kBatch || (idle && (last_batch || now - arrive[sub] >= kWindow)))) {
            song_status st = publish(v, first + sub, queries + (size_t)sub * v->dim, m,
                                     ks ? ks + sub : nullptr, efs ? efs + sub : nullptr,
                                     flags ? flags + sub : nullptr);
            if (st != SONG_OK) return st;
            v->next += m;
            sub += m;
        }
        bool any = false;
        for (int i = lo; i < sub; ++i) {
            if (seen[i]) continue;
            const long long tk = first + i;
            const int slot = (int)(tk % v->slots);
            if (load_done(v, slot) == tk) {
                const double tdone = std::chrono::duration<double>(clk::now() - t0).count();
                latency_ms[i] = (tdone - arrive[i]) * 1e3;
                last = std::max(last, tdone);
                if (ids_out)
                    std::memcpy(ids_out + (size_t)i * v->cfg.max_k, v->h_ids + (size_t)slot * v->cfg.max_k,
                                (size_t)v->cfg.max_k * 4);
                seen[i] = 1;
                ++ndone;
                any = true;
            }
        }
        while (lo < sub && seen[lo]) ++lo;
        if (!any && ++spins % 4096 == 0 && lo < sub) {  // nothing finished for a while: kernel alive?
            song_status st = ensure_running(v);
            if (st != SONG_OK) return st;
        }
    }
    if (wall_s) *wall_s = last - arrive[0];
    return SONG_OK;
}

song_status song_server_destroy(song_server* v) {
    free_server(v);
    return SONG_OK;
}

}  // extern "C"
