// song_capi.cu -- the C ABI of include/song_b200.h.
//
// Replaces the reference's host layer: KernelGraph / HashKernelGraph with
// upload_to_gpu (kernalGraph.h:20-71, hashKernelGraph.h:22-126) and
// gpu_search (kernalGraph.h:307-382, hashKernelGraph.h:360-435).
// Differences that do not change results:
//  * the index owns its device buffers for its lifetime (the reference
//    cudaMallocs and frees query/result buffers on every call, :326-330);
//  * every CUDA call is checked and reported as a song_status;
//  * a host-pointer search stages queries in chunks of
//    max(n_multiquery, 16384) and runs each chunk as ONE persistent launch
//    (results do not depend on batching: queries are independent).
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "song_b200.h"
#include "song_kernels.cuh"

namespace song {
extern std::atomic<int64_t> g_launches;
}

struct song_index {
    int kind = SONG_KIND_L2;
    int64_t n = 0;
    int dim = 0;  // floats (L2) or u32 words (Hamming) per vector
    int ld = 0;   // padded row stride in elements (multiple of 4)
    song::BaseRange range;  // integer range of the base (L2), for the exact-integer path
    song_params p{};
    int device = 0;
    int num_sms = 0;
    void* d_base = nullptr;
    int32_t* d_adj = nullptr;
    unsigned* d_counter = nullptr;  // ring of work counters, one per launch (kCounterRing)
    unsigned counter_next = 0;
    int* d_err = nullptr;
    // staging buffers of the host-pointer entry points, grown on demand
    void* d_q = nullptr;
    size_t q_cap = 0;
    int32_t* d_ids = nullptr;
    size_t ids_cap = 0;
    song_query_trace* d_tr = nullptr;
    size_t tr_cap = 0;
    float* d_dist = nullptr;
    size_t dist_cap = 0;
    // precision form: compressed copies of the FP32 rows
    // integer rows in [0, 255]: an exact byte copy the plain search gathers
    // instead of the FP32 rows (same distances, a quarter of the bytes)
    uint8_t* d_u8 = nullptr;
    int u8_ld = 0;  // bytes per row (multiple of 16)
    void* d_bf16 = nullptr;
    int bf16_ld = 0;  // bytes per row
    void* d_fp8 = nullptr;
    float* d_fp8_scale = nullptr;
    int fp8_ld = 0;
    // hub set of the learned entry stage: BF16 tensor-core tiles of the hub
    // rows, their squared norms and node ids (padded to whole tiles)
    std::vector<int32_t> entry_hubs;
    int entry_hpad = 0;
    int32_t* d_entry_ids = nullptr;
    __nv_bfloat16* d_entry_tiles = nullptr;
    float* d_entry_norm = nullptr;
    // Per-call device scratch (the entry stage's candidates and split lists,
    // the Graph::search visited bitmaps) comes from this stream-ordered pool:
    // allocated on the call's stream and freed on it after the launches that
    // use it, so searches of one index on different streams share no buffer.
    cudaMemPool_t pool = nullptr;
    // The learned search's entry-stage buffers come from a ring of kEntryRing
    // persistent slots instead of that pool, so that nothing but kernels sits
    // between consecutive learned calls on a stream: the entry stage of one
    // call may then start while the previous call's search finishes its tail.
    // A slot is reused kEntryRing learned calls later.
    struct EntrySlot {
        int32_t* ecand = nullptr;
        float* edist = nullptr;
        void* split = nullptr;
        size_t split_bytes = 0;
        int cap_nq = 0;
    };
    static constexpr int kEntryRing = 16;
    EntrySlot eslot[kEntryRing];
    unsigned eslot_next = 0;
    // learned entry / stop models
    bool has_model = false;
    bool model_staged = false;  // the entry model scores the entry stage's candidates
    std::vector<int32_t> hubs;
    std::vector<float> entry_p, stop_p;  // FP32 master parameters
    int32_t* d_hubs = nullptr;
    __half* d_entry_w = nullptr;
    __half* d_stop_w = nullptr;
    int ckpt_every = 8, min_expansions = 8, model_k = 10;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_h = nullptr, ev_d = nullptr;  // host-call timing
    int* h_err = nullptr;  // pinned host copy of the error word for host calls
    std::mutex mu;
};

namespace {

thread_local std::string g_err;

song_status fail(song_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

song_status cuda_fail(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(e == cudaErrorMemoryAllocation ? SONG_ERR_OOM : SONG_ERR_CUDA, m);
}

#define SONG_CUDA(call, what)                              \
    do {                                                   \
        cudaError_t _e = (call);                           \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)

// Each launch takes the next work counter of a ring, so launches that
// overlap on different streams do not share one; a counter is reused after
// kCounterRing launches on the same index.  A ring slot is a pair (work
// counter, CTAs done): search launches leave it at zero when they finish,
// so none needs a memset before it (the ring is zeroed once, at creation).
constexpr unsigned kCounterRing = 1024;

song_status check_params(const song_params* p) {
    if (p == nullptr) return fail(SONG_ERR_INVALID_ARG, "params is NULL");
    if (p->block_size < 1) return fail(SONG_ERR_INVALID_ARG, "block_size must be >= 1");
    if (p->pq_size < 1) return fail(SONG_ERR_INVALID_ARG, "pq_size must be >= 1");
    if (p->n_multiprobe < 1) return fail(SONG_ERR_INVALID_ARG, "n_multiprobe must be >= 1");
    if (p->bf_words < 1) return fail(SONG_ERR_INVALID_ARG, "bf_words must be >= 1");
    if (p->bf_nhash < 1 || p->bf_nhash > 4)
        return fail(SONG_ERR_UNSUPPORTED, "bf_nhash must be 1..4 (the reference table holds 4 hashes)");
    if ((int64_t)p->bf_words * 64 > (int64_t)INT32_MAX)
        return fail(SONG_ERR_UNSUPPORTED, "bf_words too large");
    return SONG_OK;
}

song_status check_adj(const int32_t* adj, int64_t n, int bs) {
    const int64_t total = n * (int64_t)bs;
    for (int64_t i = 0; i < total; ++i) {
        const int32_t v = adj[i];
        if (v >= n || v < -1) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "adj[%lld] = %d is neither -1 nor a node id in [0, %lld)",
                          (long long)i, v, (long long)n);
            return fail(SONG_ERR_INVALID_ARG, buf);
        }
    }
    return SONG_OK;
}

void free_index(song_index* x) {
    if (x == nullptr) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(x->device);
    cudaFree(x->d_base);
    cudaFree(x->d_adj);
    cudaFree(x->d_counter);
    cudaFree(x->d_err);
    cudaFree(x->d_q);
    cudaFree(x->d_ids);
    cudaFree(x->d_tr);
    cudaFree(x->d_dist);
    cudaFree(x->d_u8);
    cudaFree(x->d_entry_ids);
    cudaFree(x->d_entry_tiles);
    cudaFree(x->d_entry_norm);
    if (x->pool) cudaMemPoolDestroy(x->pool);  // released once its async frees complete
    for (auto& sl : x->eslot) {
        cudaFree(sl.ecand);
        cudaFree(sl.edist);
        cudaFree(sl.split);
    }
    cudaFree(x->d_bf16);
    cudaFree(x->d_fp8);
    cudaFree(x->d_fp8_scale);
    cudaFree(x->d_hubs);
    cudaFree(x->d_entry_w);
    cudaFree(x->d_stop_w);
    if (x->ev0) cudaEventDestroy(x->ev0);
    if (x->ev1) cudaEventDestroy(x->ev1);
    if (x->ev_h) cudaEventDestroy(x->ev_h);
    if (x->ev_d) cudaEventDestroy(x->ev_d);
    if (x->h_err) cudaFreeHost(x->h_err);
    if (x->stream) cudaStreamDestroy(x->stream);
    cudaSetDevice(cur);
    delete x;
}

// Upload rows of `dim` elements (4 bytes each) into a padded [n x ld] buffer.
song_status create_common(int kind, const void* rows, int64_t n, int dim, const int32_t* adj,
                          const song_params* params, song_index** out) {
    if (out == nullptr) return fail(SONG_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (song_status s = check_params(params)) return s;
    if (rows == nullptr || adj == nullptr) return fail(SONG_ERR_INVALID_ARG, "data or adj is NULL");
    if (n < 1 || n > (int64_t)INT32_MAX) return fail(SONG_ERR_INVALID_ARG, "n must be in [1, 2^31)");
    if (dim < 1) return fail(SONG_ERR_INVALID_ARG, "dim must be >= 1");
    if (kind == SONG_KIND_HAMMING && dim > 32)
        return fail(SONG_ERR_UNSUPPORTED, "hash_words must be <= 32 (1024-bit codes)");
    if (song_status s = check_adj(adj, n, params->block_size)) return s;

    song_index* x = new (std::nothrow) song_index();
    if (x == nullptr) return fail(SONG_ERR_OOM, "host allocation failed");
    x->kind = kind;
    x->n = n;
    x->dim = dim;
    x->ld = song::search_row_stride(kind, dim);
    x->p = *params;
    if (kind == SONG_KIND_L2) x->range = song::scan_base_range((const float*)rows, n, dim);
    cudaError_t e = cudaGetDevice(&x->device);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&x->num_sms, cudaDevAttrMultiProcessorCount, x->device);
    const size_t row_bytes = (size_t)x->ld * 4;
    if (e == cudaSuccess) e = cudaMalloc(&x->d_base, (size_t)n * row_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&x->d_adj, (size_t)n * params->block_size * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&x->d_counter, 2 * kCounterRing * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(x->d_counter, 0, 2 * kCounterRing * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&x->d_err, 256);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        cudaMemPoolProps pp = {};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = x->device;
        e = cudaMemPoolCreate(&x->pool, &pp);
    }
    if (e == cudaSuccess) {
        uint64_t keep = UINT64_MAX;  // keep freed blocks for the next call
        e = cudaMemPoolSetAttribute(x->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) e = cudaEventCreate(&x->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&x->ev1);
    if (e == cudaSuccess) e = cudaEventCreate(&x->ev_h);
    if (e == cudaSuccess) e = cudaEventCreate(&x->ev_d);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&x->h_err, sizeof(int), cudaHostAllocDefault);
    if (e == cudaSuccess && x->ld != dim) e = cudaMemset(x->d_base, 0, (size_t)n * row_bytes);
    if (e == cudaSuccess)
        e = cudaMemcpy2D(x->d_base, row_bytes, rows, (size_t)dim * 4, (size_t)dim * 4, (size_t)n,
                         cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(x->d_adj, adj, (size_t)n * params->block_size * sizeof(int32_t),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(x->d_err, 0, 256);
    // a pageable cudaMemcpy may return before its DMA lands: finish the legacy
    // stream before x->stream (non-blocking) reads the uploaded rows and adjacency
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e == cudaSuccess && kind == SONG_KIND_L2 && x->range.int_base && x->range.lo >= 0.0f &&
        x->range.hi <= 255.0f && dim <= song::kU8MaxDim) {
        x->u8_ld = song::u8_row_bytes(dim);
        e = cudaMalloc(&x->d_u8, (size_t)n * x->u8_ld);
        if (e == cudaSuccess)
            e = song::convert_rows_u8((const float*)x->d_base, n, dim, x->ld, x->d_u8, x->u8_ld,
                                      x->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
    }
    if (e != cudaSuccess) {
        song_status s = cuda_fail(e, "index upload");
        free_index(x);
        return s;
    }
    *out = x;
    return SONG_OK;
}

template <typename T>
cudaError_t grow(T** ptr, size_t* cap, size_t bytes) {
    if (*cap >= bytes) return cudaSuccess;
    cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc((void**)ptr, bytes);
    if (e == cudaSuccess) *cap = bytes;
    return e;
}

// Device scratch of one call, from the index's pool on the call's stream;
// every block is freed on that stream when the object goes out of scope,
// i.e. after the launches the call made.
struct CallScratch {
    song_index* x;
    cudaStream_t st;
    void* p[4] = {nullptr, nullptr, nullptr, nullptr};
    int n = 0;
    CallScratch(song_index* idx, cudaStream_t s) : x(idx), st(s) {}
    CallScratch(const CallScratch&) = delete;
    CallScratch& operator=(const CallScratch&) = delete;
    template <typename T>
    cudaError_t get(T** out, size_t bytes) {
        if (n == 4) return cudaErrorInvalidValue;
        void* q = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&q, bytes, x->pool, st);
        if (e != cudaSuccess) return e;
        p[n++] = q;
        *out = static_cast<T*>(q);
        return cudaSuccess;
    }
    ~CallScratch() {
        for (int i = 0; i < n; ++i) cudaFreeAsync(p[i], st);
    }
};

// Build the entry stage's tables for hub node ids `hubs` (device, stream-ordered).
song_status attach_entry_hubs(song_index* x, const std::vector<int32_t>& hubs) {
    if (x->kind != SONG_KIND_L2) return fail(SONG_ERR_UNSUPPORTED, "entry hubs apply to L2 indexes");
    if (x->dim > song::kEntryMaxDim) return fail(SONG_ERR_UNSUPPORTED, "entry hubs need dim <= 288");
    if (hubs.empty()) return fail(SONG_ERR_INVALID_ARG, "empty hub set");
    for (int32_t h : hubs)
        if (h < 0 || h >= x->n) return fail(SONG_ERR_INVALID_ARG, "hub id out of range");
    const int tile = song::entry_tile_hubs();
    const int hpad = ((int)hubs.size() + tile - 1) / tile * tile;
    const int kp = song::entry_padded_dim(x->dim);
    std::vector<int32_t> ids(hubs);
    ids.resize(hpad, -1);
    cudaFree(x->d_entry_ids);
    cudaFree(x->d_entry_tiles);
    cudaFree(x->d_entry_norm);
    x->d_entry_ids = nullptr;
    x->d_entry_tiles = nullptr;
    x->d_entry_norm = nullptr;
    x->entry_hpad = 0;
    x->entry_hubs.clear();
    cudaError_t e = cudaMalloc(&x->d_entry_ids, (size_t)hpad * 4);
    if (e == cudaSuccess) e = cudaMalloc(&x->d_entry_tiles, (size_t)hpad * kp * 2);
    if (e == cudaSuccess) e = cudaMalloc(&x->d_entry_norm, (size_t)hpad * 4);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(x->d_entry_ids, ids.data(), (size_t)hpad * 4, cudaMemcpyHostToDevice,
                            x->stream);
    if (e == cudaSuccess)
        e = song::build_entry_tables((const float*)x->d_base, x->ld, x->dim, x->d_entry_ids, hpad,
                                     x->d_entry_tiles, x->d_entry_norm, x->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
    if (e != cudaSuccess) return cuda_fail(e, "entry hub tables");
    x->entry_hubs = hubs;
    x->entry_hpad = hpad;
    return SONG_OK;
}

// The entry stage for nq queries at d_q: ids/dists [nq x kEntryK].
song_status run_entry(song_index* x, const void* d_q, int nq, int32_t* d_ids, float* d_d,
                      cudaStream_t st) {
    CallScratch cs(x, st);
    const size_t split_bytes = song::entry_split_scratch_bytes(nq, x->num_sms);
    void* split = nullptr;
    SONG_CUDA(cs.get(&split, split_bytes), "entry split scratch");
    cudaError_t e = song::launch_entry((const float*)d_q, x->dim, nq, x->dim, x->d_entry_tiles,
                                       x->d_entry_norm, x->d_entry_ids, x->entry_hpad, d_ids, d_d,
                                       x->d_err, st, split, split_bytes, x->num_sms);
    if (e != cudaSuccess) return cuda_fail(e, "entry launch");
    return SONG_OK;
}

int clamp_ef(int ef, int k, int pq_size) {  // kernalGraph.h:315-316
    if (ef < k) ef = k;
    if (ef > pq_size) ef = pq_size;
    return ef;
}

// Fill SearchArgs for one launch over `nq` queries at d_q / d_ids / d_tr.
song_status make_args(song_index* x, const void* d_q, int nq, int k, int ef, int32_t* d_ids,
                      song_query_trace* d_tr, song::SearchArgs* a,
                      const song_search_opts* opts = nullptr, float* d_dist = nullptr) {
    const int cap = ef < 1 ? 1 : (ef > x->p.pq_size ? x->p.pq_size : ef);  // Candidates::init
    std::memset(a, 0, sizeof *a);
    a->base = x->d_base;
    a->adj = x->d_adj;
    a->queries = d_q;
    a->out = d_ids;
    a->trace = d_tr;
    a->counter = x->d_counter;
    a->err = x->d_err;
    a->n = x->n;
    a->dim = x->dim;
    a->ld = x->ld;
    a->qld = x->dim;
    a->block_size = x->p.block_size;
    a->k = k;
    a->nq = nq;
    a->cap = cap;
    a->bf_words = x->p.bf_words;
    a->bf_nhash = x->p.bf_nhash;
    a->n_multiprobe = x->p.n_multiprobe;
    a->int_base = x->range.int_base;
    a->base_min = x->range.lo;
    a->base_max = x->range.hi;
    a->out_dist = d_dist;
    a->qdim = x->dim;
    a->u8 = x->d_u8;
    a->u8_ld = x->u8_ld;
    const int prec = opts ? opts->precision : SONG_PREC_FP32;
    if (prec != SONG_PREC_FP32) {
        if (x->kind != SONG_KIND_L2)
            return fail(SONG_ERR_UNSUPPORTED, "the precision form applies to L2 indexes");
        if (prec == SONG_PREC_BF16 && x->d_bf16 == nullptr)
            return fail(SONG_ERR_INVALID_ARG, "BF16 rows not attached (song_index_set_precision)");
        if (prec == SONG_PREC_FP8 && x->d_fp8 == nullptr)
            return fail(SONG_ERR_INVALID_ARG, "FP8 rows not attached (song_index_set_precision)");
        if (prec != SONG_PREC_BF16 && prec != SONG_PREC_FP8)
            return fail(SONG_ERR_INVALID_ARG, "unknown precision");
        a->prec = prec;
        a->lowp = prec == SONG_PREC_BF16 ? x->d_bf16 : x->d_fp8;
        a->scales = x->d_fp8_scale;
        a->lowp_ld = prec == SONG_PREC_BF16 ? x->bf16_ld : x->fp8_ld;
        a->qdim = song::lowp_padded_dim(prec, x->dim);
        a->rerank = opts->rerank ? 1 : 0;
    }
    if (opts && !opts->learned && opts->bloom_hashes != 0)
        return fail(SONG_ERR_INVALID_ARG, "bloom_hashes applies to learned searches only");
    if (opts && opts->learned) {
        if (!x->has_model) return fail(SONG_ERR_INVALID_ARG, "no learned model attached (song_index_learn)");
        if (x->kind != SONG_KIND_L2 || cap > 1024)
            return fail(SONG_ERR_UNSUPPORTED, "learned search: L2 indexes, queues up to 1024 slots");
        a->lm = 2;
        a->hubs = x->d_hubs;
        a->n_hubs = x->model_staged ? 0 : (int)x->hubs.size();
        a->entry_w = x->d_entry_w;
        a->stop_w = x->d_stop_w;
        if (opts->entry < SONG_ENTRY_MODEL || opts->entry > SONG_ENTRY_SEEDS)
            return fail(SONG_ERR_INVALID_ARG, "entry must be SONG_ENTRY_MODEL, _NEAREST or _SEEDS");
        if (opts->entry == SONG_ENTRY_NEAREST) {
            if (!x->model_staged)
                return fail(SONG_ERR_INVALID_ARG, "SONG_ENTRY_NEAREST needs the entry stage's hub set");
            a->entry_w = nullptr;  // the kernel then seeds from the nearest hubs
        } else if (opts->entry == SONG_ENTRY_SEEDS) {
            a->entry_w = nullptr;
            a->n_hubs = 0;
            a->no_entry_stage = 1;
        }
        a->ckpt_every = x->ckpt_every;
        a->min_expansions = x->min_expansions;
        a->beam = opts->beam < 1 ? 1 : (opts->beam > 4 ? 4 : opts->beam);
        if (opts->bloom_hashes != 0) {
            if (opts->bloom_hashes < 1 || opts->bloom_hashes > 4)
                return fail(SONG_ERR_INVALID_ARG, "bloom_hashes must be 0 or in [1, 4]");
            a->bf_nhash = opts->bloom_hashes;
        }
        const float t = opts->stop_threshold;
        a->stop_thr = t <= 0.0f ? -INFINITY : (t >= 1.0f ? INFINITY : std::log(t / (1.0f - t)));
    }
    song::search_warp_smem(x->kind, a->qdim, cap, x->p.bf_words, a);
    if (cap > 4096)
        return fail(SONG_ERR_UNSUPPORTED, "queue capacity above 4096 slots (pq_size and ef) is not supported");
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, x->device);
    if (a->warp_smem > optin) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "per-query shared memory %d B (queue %d, bf_words %d, dim %d) exceeds the "
                      "%d B a CTA may use",
                      a->warp_smem, cap, x->p.bf_words, x->dim, optin);
        return fail(SONG_ERR_UNSUPPORTED, buf);
    }
    return SONG_OK;
}

// The next entry-stage ring slot, holding at least nq queries.  A slot too
// small grows the whole ring at once (the first learned call, or a larger
// batch): after a device synchronisation, since calls in flight may still use
// the old buffers.
song_status entry_slot(song_index* x, int nq, song_index::EntrySlot** out) {
    song_index::EntrySlot& sl = x->eslot[x->eslot_next++ % song_index::kEntryRing];
    if (sl.cap_nq < nq) {
        SONG_CUDA(cudaDeviceSynchronize(), "entry ring growth");
        int cap = std::max(nq, 1024);
        for (auto& r : x->eslot) cap = std::max(cap, r.cap_nq);
        const size_t cells = (size_t)cap * song::kEntryK;
        const size_t sb = song::entry_split_scratch_bytes(cap, x->num_sms);
        for (auto& r : x->eslot) {
            cudaFree(r.ecand);
            cudaFree(r.edist);
            cudaFree(r.split);
            r = song_index::EntrySlot();
            cudaError_t e = cudaMalloc(&r.ecand, cells * 4);
            if (e == cudaSuccess) e = cudaMalloc(&r.edist, cells * 4);
            if (e == cudaSuccess) e = cudaMalloc(&r.split, sb);
            if (e == cudaSuccess) e = cudaMemset(r.split, 0, sb);  // arrival counters start at zero
            if (e != cudaSuccess) {
                cudaFree(r.ecand);
                cudaFree(r.edist);
                cudaFree(r.split);
                r = song_index::EntrySlot();
                return cuda_fail(e, "entry ring slot");
            }
            r.split_bytes = sb;
            r.cap_nq = cap;
        }
    }
    *out = &sl;
    return SONG_OK;
}

song_status launch(song_index* x, song::SearchArgs a, cudaStream_t st) {
    if (a.lm == 2 && x->model_staged && !a.no_entry_stage && a.qseeds == nullptr &&
        a.ecand == nullptr && a.nq > 0) {
        // learned search: the entry stage first, on the same stream, into a ring
        // slot; it may overlap the tail of the previous search launch there
        song_index::EntrySlot* sl = nullptr;
        if (song_status s = entry_slot(x, a.nq, &sl)) return s;
        // without the entry model the search takes the nearest n_multiprobe
        // hubs and reads nothing else of the list
        const int keep = a.entry_w == nullptr ? std::min(std::max(a.n_multiprobe, 1), song::kEntryK)
                                              : song::kEntryK;
        cudaError_t e = song::launch_entry((const float*)a.queries, x->dim, a.nq, x->dim,
                                           x->d_entry_tiles, x->d_entry_norm, x->d_entry_ids,
                                           x->entry_hpad, sl->ecand, sl->edist, x->d_err, st,
                                           sl->split, sl->split_bytes, x->num_sms, true, keep);
        if (e != cudaSuccess) return cuda_fail(e, "entry launch");
        a.ecand = sl->ecand;
        a.edist = sl->edist;
    }
    unsigned* ctr = x->d_counter + 2 * (x->counter_next++ % kCounterRing);
    a.counter = ctr;
    a.done = ctr + 1;
    cudaError_t e = song::launch_search(x->kind, a, x->num_sms, st);
    if (e != cudaSuccess) return cuda_fail(e, "search launch");
    return SONG_OK;
}

song_status host_search(song_index* x, int kind, const void* queries, int nq, int k,
                        int n_multiquery, int ef_search, int32_t* ids, song_query_trace* traces,
                        song_timing* timing, const song_search_opts* opts = nullptr,
                        float* dists = nullptr) {
    using clk = std::chrono::high_resolution_clock;
    auto ms = [](clk::time_point a, clk::time_point b) {
        return std::chrono::duration<double, std::milli>(b - a).count();
    };
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (x->kind != kind) return fail(SONG_ERR_INVALID_ARG, "query type does not match the index kind");
    if (nq < 0 || k < 0) return fail(SONG_ERR_INVALID_ARG, "nq and k must be >= 0");
    if (nq > 0 && (queries == nullptr || (k > 0 && ids == nullptr)))
        return fail(SONG_ERR_INVALID_ARG, "queries or ids is NULL");
    const int ef = clamp_ef(ef_search, k, x->p.pq_size);
    song_timing t{};
    t.ef_search = ef;
    t.batch_limit = n_multiquery;
    std::lock_guard<std::mutex> lock(x->mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != x->device) SONG_CUDA(cudaSetDevice(x->device), "cudaSetDevice");
    const int chunk = std::max(std::max(n_multiquery, 1), std::min(nq, 16384));
    const size_t qrow = (size_t)x->dim * 4;
    auto t0 = clk::now();
    SONG_CUDA(grow(&x->d_q, &x->q_cap, std::max<size_t>(1, (size_t)std::min(nq, chunk) * qrow)),
              "query staging alloc");
    SONG_CUDA(grow(&x->d_ids, &x->ids_cap, std::max<size_t>(4, (size_t)std::min(nq, chunk) * k * 4)),
              "result staging alloc");
    if (traces)
        SONG_CUDA(grow(&x->d_tr, &x->tr_cap,
                       std::max<size_t>(48, (size_t)std::min(nq, chunk) * sizeof(song_query_trace))),
                  "trace staging alloc");
    if (dists)
        SONG_CUDA(grow(&x->d_dist, &x->dist_cap, std::max<size_t>(4, (size_t)std::min(nq, chunk) * k * 4)),
                  "distance staging alloc");
    auto t1 = clk::now();
    t.alloc_ms = ms(t0, t1);
    cudaStream_t st = x->stream;
    SONG_CUDA(cudaMemsetAsync(x->d_err, 0, sizeof(int), st), "error reset");
    *x->h_err = 0;
    // Per batch: copy in, search, copy out, on the index's stream with one
    // synchronisation at the end of the batch; the copy and kernel times come
    // from events between them.
    for (int off = 0; off < nq; off += chunk) {
        const int bs = std::min(chunk, nq - off);
        SONG_CUDA(cudaEventRecord(x->ev_h, st), "event");
        SONG_CUDA(cudaMemcpyAsync(x->d_q, (const char*)queries + (size_t)off * qrow, (size_t)bs * qrow,
                                  cudaMemcpyHostToDevice, st),
                  "query H2D");
        song::SearchArgs a;
        if (song_status s = make_args(x, x->d_q, bs, k, ef, x->d_ids, traces ? x->d_tr : nullptr, &a,
                                      opts, dists ? x->d_dist : nullptr))
            return s;
        SONG_CUDA(cudaEventRecord(x->ev0, st), "event");
        if (song_status s = launch(x, a, st)) return s;
        SONG_CUDA(cudaEventRecord(x->ev1, st), "event");
        if (k > 0)
            SONG_CUDA(cudaMemcpyAsync(ids + (size_t)off * k, x->d_ids, (size_t)bs * k * 4,
                                      cudaMemcpyDeviceToHost, st),
                      "ids D2H");
        if (traces)
            SONG_CUDA(cudaMemcpyAsync(traces + off, x->d_tr, (size_t)bs * sizeof(song_query_trace),
                                      cudaMemcpyDeviceToHost, st),
                      "trace D2H");
        if (dists && k > 0)
            SONG_CUDA(cudaMemcpyAsync(dists + (size_t)off * k, x->d_dist, (size_t)bs * k * 4,
                                      cudaMemcpyDeviceToHost, st),
                      "distance D2H");
        if (off + bs >= nq)
            SONG_CUDA(cudaMemcpyAsync(x->h_err, x->d_err, sizeof(int), cudaMemcpyDeviceToHost, st),
                      "error flag");
        SONG_CUDA(cudaEventRecord(x->ev_d, st), "event");
        SONG_CUDA(cudaStreamSynchronize(st), "search");
        float hms = 0.f, kms = 0.f, dms = 0.f;
        cudaEventElapsedTime(&hms, x->ev_h, x->ev0);
        cudaEventElapsedTime(&kms, x->ev0, x->ev1);
        cudaEventElapsedTime(&dms, x->ev1, x->ev_d);
        t.h2d_ms += hms;
        t.kernel_ms += kms;
        t.d2h_ms += dms;
        t.n_batches += 1;
    }
    if (nq <= 0) {
        SONG_CUDA(cudaMemcpyAsync(x->h_err, x->d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "error flag");
        SONG_CUDA(cudaStreamSynchronize(st), "error flag");
    }
    const int err = *x->h_err;
    if (err == 2) return fail(SONG_ERR_TIMEOUT, "the entry stage's bounded wait gave up");
    if (err) return fail(SONG_ERR_INVALID_ARG, "graph holds an out-of-range neighbour id");
    t.total_ms = ms(t1, clk::now());
    if (timing) *timing = t;
    return SONG_OK;
}

}  // namespace

namespace song {
song_status set_error(song_status status, const char* message) { return fail(status, message); }

// Index-wide search arguments for a server whose slots take requests up to
// (max_k, max_cap); per-request fields are filled by the serving kernel.
song_status server_args(song_index* x, const song_search_opts* opts, int max_k, int max_cap,
                        SearchArgs* a, int* num_sms, int* device) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (x->kind != SONG_KIND_L2) return fail(SONG_ERR_UNSUPPORTED, "the server serves L2 indexes");
    song_status st = make_args(x, nullptr, 1, max_k, max_cap, nullptr, nullptr, a, opts, nullptr);
    if (st != SONG_OK) return st;
    a->lm = 2;
    a->hubs = x->d_hubs;
    a->n_hubs = x->has_model ? (int)x->hubs.size() : 0;
    a->entry_w = x->has_model ? x->d_entry_w : nullptr;
    a->stop_w = x->has_model ? x->d_stop_w : nullptr;
    a->ckpt_every = x->ckpt_every;
    a->min_expansions = x->min_expansions;
    *num_sms = x->num_sms;
    *device = x->device;
    return SONG_OK;
}

int index_pq_size(const song_index* x) { return x ? x->p.pq_size : 0; }
bool index_model_staged(const song_index* x) { return x && x->has_model && x->model_staged; }
cudaError_t index_entry(song_index* x, const float* d_q, int qld, int nq, int32_t* d_ids,
                        float* d_d, cudaStream_t st, void* split_scratch, size_t split_bytes) {
    return song::launch_entry(d_q, qld, nq, x->dim, x->d_entry_tiles, x->d_entry_norm,
                              x->d_entry_ids, x->entry_hpad, d_ids, d_d, x->d_err, st,
                              split_scratch, split_bytes, x->num_sms);
}
int index_dim(const song_index* x) { return x ? x->dim : 0; }
bool index_has_model(const song_index* x) { return x && x->has_model; }

BaseRange scan_base_range(const float* rows, int64_t n, int dim) {
    BaseRange r;
    const int64_t total = n * (int64_t)dim;
    if (total <= 0) return r;
    float lo = rows[0], hi = rows[0];
    bool integral = true;
    for (int64_t i = 0; i < total; ++i) {
        const float v = rows[i];
        if (!(v == std::nearbyint(v)) || !(std::fabs(v) < 16777216.0f)) {
            integral = false;
            break;
        }
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    r.int_base = integral ? 1 : 0;
    r.lo = lo;
    r.hi = hi;
    return r;
}
}  // namespace song

extern "C" {

void song_params_default(song_params* p) {
    if (!p) return;
    p->block_size = 32;        // config.h:9
    p->fixed_degree = 31;      // config.h:12
    p->search_degree = 15;     // config.h:17
    p->ef_construction = 150;  // config.h:24
    p->pq_size = 50;           // config.h:28
    p->topk = 10;              // config.h:31
    p->n_multiprobe = 4;       // config.h:34
    p->n_multiquery = 512;     // config.h:38
    p->hash_bits = 256;        // config.h:41
    p->bf_words = 256;         // config.h:56
    p->bf_nhash = 4;           // config.h:58
}

const char* song_last_error(void) { return g_err.c_str(); }

const char* song_version(void) { return "song_b200 0.1 (sm_100a)"; }

song_status song_index_create_l2(const float* data, int64_t n, int dim, const int32_t* adj,
                                 const song_params* params, song_index** out) {
    return create_common(SONG_KIND_L2, data, n, dim, adj, params, out);
}

song_status song_index_create_hamming(const uint32_t* codes, int64_t n, int hash_words,
                                      const int32_t* adj, const song_params* params,
                                      song_index** out) {
    return create_common(SONG_KIND_HAMMING, codes, n, hash_words, adj, params, out);
}

song_status song_index_destroy(song_index* index) {
    free_index(index);
    return SONG_OK;
}

song_status song_index_info(const song_index* x, int64_t* n, int* dim, int* kind) {
    if (!x) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (n) *n = x->n;
    if (dim) *dim = x->dim;
    if (kind) *kind = x->kind;
    return SONG_OK;
}

song_status song_index_u8_rows(const song_index* x, int* has_u8, int* row_bytes) {
    if (!x) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (has_u8) *has_u8 = x->d_u8 != nullptr ? 1 : 0;
    if (row_bytes) *row_bytes = x->u8_ld;
    return SONG_OK;
}

song_status song_gpu_search(song_index* index, const float* queries, int nq, int k,
                            int n_multiquery, int ef_search, int32_t* ids,
                            song_query_trace* traces, song_timing* timing) {
    return host_search(index, SONG_KIND_L2, queries, nq, k, n_multiquery, ef_search, ids, traces,
                       timing);
}

song_status song_gpu_search_hamming(song_index* index, const uint32_t* queries, int nq, int k,
                                    int n_multiquery, int ef_search, int32_t* ids,
                                    song_query_trace* traces, song_timing* timing) {
    return host_search(index, SONG_KIND_HAMMING, queries, nq, k, n_multiquery, ef_search, ids,
                       traces, timing);
}

song_status song_search_device(song_index* x, const void* d_queries, int nq, int k, int ef_search,
                               int32_t* d_ids, song_query_trace* d_traces, void* stream) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (nq < 0 || k < 0) return fail(SONG_ERR_INVALID_ARG, "nq and k must be >= 0");
    if (nq == 0) return SONG_OK;
    if (d_queries == nullptr || (k > 0 && d_ids == nullptr))
        return fail(SONG_ERR_INVALID_ARG, "queries or ids is NULL");
    const int ef = clamp_ef(ef_search, k, x->p.pq_size);
    std::lock_guard<std::mutex> lock(x->mu);
    song::SearchArgs a;
    if (song_status s = make_args(x, d_queries, nq, k, ef, d_ids, d_traces, &a)) return s;
    return launch(x, a, (cudaStream_t)stream);
}

song_status song_build_graph(int kind, const void* rows, int64_t n, int dim,
                             const song_params* params, int batch_ratio, int build_bf_words,
                             int32_t* adj_out) {
    if (song_status s = check_params(params)) return s;
    if (rows == nullptr || adj_out == nullptr) return fail(SONG_ERR_INVALID_ARG, "rows or adj_out is NULL");
    if (kind != SONG_KIND_L2 && kind != SONG_KIND_HAMMING) return fail(SONG_ERR_INVALID_ARG, "bad kind");
    if (n < 1 || n > (int64_t)INT32_MAX - 1) return fail(SONG_ERR_INVALID_ARG, "n must be in [1, 2^31-1)");
    if (dim < 1 || (kind == SONG_KIND_HAMMING && dim > 32))
        return fail(SONG_ERR_INVALID_ARG, "dim out of range");
    if (params->fixed_degree < 1 || params->fixed_degree > 32 ||
        params->fixed_degree > params->block_size || params->search_degree < 1 ||
        params->ef_construction < 1)
        return fail(SONG_ERR_UNSUPPORTED, "GPU build needs 1 <= fixed_degree <= min(32, block_size)");
    const int ratio = batch_ratio > 0 ? batch_ratio : 32;
    const int bfw = build_bf_words > 0 ? build_bf_words : 1024;
    const int ld = song::search_row_stride(kind, dim);
    const song::BaseRange range =
        kind == SONG_KIND_L2 ? song::scan_base_range((const float*)rows, n, dim) : song::BaseRange();
    int dev = 0, sms = 0;
    SONG_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    SONG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
    void* d_rows = nullptr;
    int32_t* d_adj = nullptr;
    cudaStream_t st = nullptr;
    const size_t row_bytes = (size_t)ld * 4;
    cudaError_t e = cudaMalloc(&d_rows, (size_t)n * row_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d_adj, (size_t)n * params->block_size * 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess && ld != dim) e = cudaMemset(d_rows, 0, (size_t)n * row_bytes);
    if (e == cudaSuccess)
        e = cudaMemcpy2D(d_rows, row_bytes, rows, (size_t)dim * 4, (size_t)dim * 4, (size_t)n,
                         cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = song::build_graph_device(kind, d_rows, n, dim, ld, *params, ratio, bfw, d_adj,
                                     sms, st, range);
    if (e == cudaSuccess)
        e = cudaMemcpy(adj_out, d_adj, (size_t)n * params->block_size * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_rows);
    cudaFree(d_adj);
    if (st) cudaStreamDestroy(st);
    if (e != cudaSuccess) return cuda_fail(e, "graph build");
    return SONG_OK;
}

song_status song_index_set_precision(song_index* x, int precision) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (x->kind != SONG_KIND_L2) return fail(SONG_ERR_UNSUPPORTED, "the precision form applies to L2 indexes");
    if (precision != SONG_PREC_BF16 && precision != SONG_PREC_FP8)
        return fail(SONG_ERR_INVALID_ARG, "precision must be SONG_PREC_BF16 or SONG_PREC_FP8");
    std::lock_guard<std::mutex> lock(x->mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != x->device) SONG_CUDA(cudaSetDevice(x->device), "cudaSetDevice");
    const int pd = song::lowp_padded_dim(precision, x->dim);
    const int row_bytes = precision == SONG_PREC_BF16 ? pd * 2 : pd;
    void** dst = precision == SONG_PREC_BF16 ? &x->d_bf16 : &x->d_fp8;
    cudaFree(*dst);
    *dst = nullptr;
    SONG_CUDA(cudaMalloc(dst, (size_t)x->n * row_bytes), "compressed rows alloc");
    if (precision == SONG_PREC_FP8) {
        cudaFree(x->d_fp8_scale);
        x->d_fp8_scale = nullptr;
        SONG_CUDA(cudaMalloc(&x->d_fp8_scale, (size_t)x->n * sizeof(float)), "scale alloc");
    }
    SONG_CUDA(song::quantize_rows(precision, (const float*)x->d_base, x->n, x->dim, x->ld, *dst,
                                  row_bytes, x->d_fp8_scale, x->stream),
              "quantize");
    SONG_CUDA(cudaStreamSynchronize(x->stream), "quantize sync");
    if (precision == SONG_PREC_BF16) x->bf16_ld = row_bytes; else x->fp8_ld = row_bytes;
    return SONG_OK;
}

song_status song_search_device_ex(song_index* x, const song_search_opts* opts,
                                  const void* d_queries, int nq, int k, int ef_search,
                                  int32_t* d_ids, float* d_dists, song_query_trace* d_traces,
                                  void* stream) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (nq < 0 || k < 0) return fail(SONG_ERR_INVALID_ARG, "nq and k must be >= 0");
    if (nq == 0) return SONG_OK;
    if (d_queries == nullptr || (k > 0 && d_ids == nullptr))
        return fail(SONG_ERR_INVALID_ARG, "queries or ids is NULL");
    const int ef = clamp_ef(ef_search, k, x->p.pq_size);
    std::lock_guard<std::mutex> lock(x->mu);
    song::SearchArgs a;
    if (song_status s = make_args(x, d_queries, nq, k, ef, d_ids, d_traces, &a, opts, d_dists)) return s;
    return launch(x, a, (cudaStream_t)stream);
}

song_status song_search_device_seeded(song_index* x, const song_search_opts* opts,
                                      const void* d_queries, int nq, int k, int ef_search,
                                      const int32_t* d_seeds, int n_seeds, int32_t* d_ids,
                                      float* d_dists, song_query_trace* d_traces, void* stream) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (nq < 0 || k < 0) return fail(SONG_ERR_INVALID_ARG, "nq and k must be >= 0");
    if (nq == 0) return SONG_OK;
    if (d_queries == nullptr || d_seeds == nullptr || (k > 0 && d_ids == nullptr))
        return fail(SONG_ERR_INVALID_ARG, "queries, seeds or ids is NULL");
    if (n_seeds < 1 || n_seeds > 32) return fail(SONG_ERR_INVALID_ARG, "n_seeds must be 1..32");
    const int ef = clamp_ef(ef_search, k, x->p.pq_size);
    std::lock_guard<std::mutex> lock(x->mu);
    song::SearchArgs a;
    if (song_status s = make_args(x, d_queries, nq, k, ef, d_ids, d_traces, &a, opts, d_dists)) return s;
    a.qseeds = d_seeds;
    a.n_qseeds = n_seeds;
    return launch(x, a, (cudaStream_t)stream);
}

// Graph::search on the GPU (see song_graphsearch.cu); ef_search raised to k
// as graph.h:36 does.  Stream-ordered.
song_status graph_search_launch(song_index* x, const float* d_q, int nq, int k, int ef_search,
                                int32_t* d_ids, song_query_trace* d_tr, cudaStream_t st) {
    if (x->kind != SONG_KIND_L2) return fail(SONG_ERR_UNSUPPORTED, "Graph::search is the L2 search");
    const int ef = ef_search < k ? k : ef_search;
    if (ef < 1 || ef > 1024) return fail(SONG_ERR_UNSUPPORTED, "Graph::search mode: ef must be 1..1024");
    if (ef < x->p.n_multiprobe)
        return fail(SONG_ERR_UNSUPPORTED, "Graph::search mode: ef must be >= N_MULTIPROBE");
    const int64_t warps = song::graph_search_resident_warps(x->dim, ef, x->num_sms, x->device);
    if (warps < 4) return fail(SONG_ERR_UNSUPPORTED, "Graph::search mode: per-query state does not fit");
    const int64_t vwords = (x->n + 31) / 32;
    CallScratch cs(x, st);
    uint32_t* visited = nullptr;
    SONG_CUDA(cs.get(&visited, (size_t)warps * vwords * 4), "visited bitmaps");
    unsigned* ctr = x->d_counter + 2 * (x->counter_next++ % kCounterRing);
    SONG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned), st), "counter reset");
    cudaError_t e = song::launch_graph_search((const float*)x->d_base, x->ld, x->dim, x->d_adj,
                                              x->p.block_size, x->n, d_q, nq, k, ef,
                                              x->p.n_multiprobe, d_ids, d_tr, ctr, x->d_err,
                                              visited, warps, x->num_sms, st);
    if (e != cudaSuccess) return cuda_fail(e, "Graph::search launch");
    // this kernel does not return its counter to zero itself: the ring slot
    // must be zero for the search launch that takes it next
    SONG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned), st), "counter reset");
    return SONG_OK;
}

song_status song_index_set_entry_hubs(song_index* x, const int32_t* hub_ids, int count) {
    if (x == nullptr || hub_ids == nullptr || count < 1)
        return fail(SONG_ERR_INVALID_ARG, "index or hub ids missing");
    std::lock_guard<std::mutex> lock(x->mu);
    return attach_entry_hubs(x, std::vector<int32_t>(hub_ids, hub_ids + count));
}

song_status song_index_entry_candidates(song_index* x, const float* d_queries, int nq,
                                        int32_t* d_ids, float* d_dists, void* stream) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (nq < 0) return fail(SONG_ERR_INVALID_ARG, "nq must be >= 0");
    if (nq == 0) return SONG_OK;
    if (d_queries == nullptr || d_ids == nullptr || d_dists == nullptr)
        return fail(SONG_ERR_INVALID_ARG, "queries, ids or dists is NULL");
    std::lock_guard<std::mutex> lock(x->mu);
    if (x->entry_hpad == 0) return fail(SONG_ERR_INVALID_ARG, "no entry hub set attached");
    return run_entry(x, d_queries, nq, d_ids, d_dists, (cudaStream_t)stream);
}

song_status song_graph_search_device(song_index* x, const float* d_queries, int nq, int k,
                                     int ef_search, int32_t* d_ids, song_query_trace* d_traces,
                                     void* stream) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (nq < 0 || k < 1) return fail(SONG_ERR_INVALID_ARG, "nq must be >= 0 and k >= 1");
    if (nq == 0) return SONG_OK;
    if (d_queries == nullptr || d_ids == nullptr) return fail(SONG_ERR_INVALID_ARG, "queries or ids is NULL");
    std::lock_guard<std::mutex> lock(x->mu);
    return graph_search_launch(x, d_queries, nq, k, ef_search, d_ids, d_traces, (cudaStream_t)stream);
}

song_status song_graph_search(song_index* x, const float* queries, int nq, int k, int ef_search,
                              int32_t* ids, song_query_trace* traces) {
    if (x == nullptr) return fail(SONG_ERR_INVALID_ARG, "index is NULL");
    if (nq < 0 || k < 1) return fail(SONG_ERR_INVALID_ARG, "nq must be >= 0 and k >= 1");
    if (nq == 0) return SONG_OK;
    if (queries == nullptr || ids == nullptr) return fail(SONG_ERR_INVALID_ARG, "queries or ids is NULL");
    std::lock_guard<std::mutex> lock(x->mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != x->device) SONG_CUDA(cudaSetDevice(x->device), "cudaSetDevice");
    cudaStream_t st = x->stream;
    SONG_CUDA(grow(&x->d_q, &x->q_cap, (size_t)nq * x->dim * 4), "query alloc");
    SONG_CUDA(grow(&x->d_ids, &x->ids_cap, (size_t)nq * k * 4), "ids alloc");
    if (traces) SONG_CUDA(grow(&x->d_tr, &x->tr_cap, (size_t)nq * sizeof(song_query_trace)), "trace alloc");
    SONG_CUDA(cudaMemsetAsync(x->d_err, 0, 4, st), "error reset");
    SONG_CUDA(cudaMemcpyAsync(x->d_q, queries, (size_t)nq * x->dim * 4, cudaMemcpyHostToDevice, st),
              "query copy");
    if (song_status s = graph_search_launch(x, (const float*)x->d_q, nq, k, ef_search, x->d_ids,
                                            traces ? x->d_tr : nullptr, st))
        return s;
    SONG_CUDA(cudaMemcpyAsync(ids, x->d_ids, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st), "ids copy");
    if (traces)
        SONG_CUDA(cudaMemcpyAsync(traces, x->d_tr, (size_t)nq * sizeof(song_query_trace),
                                  cudaMemcpyDeviceToHost, st), "trace copy");
    int err = 0;
    SONG_CUDA(cudaMemcpyAsync(&err, x->d_err, 4, cudaMemcpyDeviceToHost, st), "error word");
    SONG_CUDA(cudaStreamSynchronize(st), "Graph::search");
    if (err == 3)
        return fail(SONG_ERR_UNSUPPORTED, "Graph::search mode: more distance ties at the top-ef "
                                          "maximum than the frontier holds");
    if (err != 0) return fail(SONG_ERR_CUDA, "Graph::search: the kernel reported an error");
    return SONG_OK;
}

song_status song_gpu_search_ex(song_index* index, const song_search_opts* opts,
                               const float* queries, int nq, int k, int n_multiquery,
                               int ef_search, int32_t* ids, float* dists,
                               song_query_trace* traces, song_timing* timing) {
    return host_search(index, index ? index->kind : SONG_KIND_L2, queries, nq, k, n_multiquery,
                       ef_search, ids, traces, timing, opts, dists);
}

void song_learn_params_default(song_learn_params* p) {
    if (!p) return;
    p->k = 10;
    p->ef = 128;
    p->ckpt_every = 8;
    p->min_expansions = 8;
    p->max_ckpt = 256;
    p->entry_steps = 1500;
    p->stop_steps = 3000;
    p->batch = 4096;
    p->lr = 2e-3f;
    p->entry_hubs = 8192;
    p->seed = 2020;
}

static song_status attach_model(song_index* x) {
    cudaFree(x->d_hubs);
    x->d_hubs = nullptr;
    SONG_CUDA(cudaMalloc(&x->d_hubs, std::max<size_t>(1, x->hubs.size()) * 4), "hub alloc");
    SONG_CUDA(cudaMemcpy(x->d_hubs, x->hubs.data(), x->hubs.size() * 4, cudaMemcpyHostToDevice), "hubs");
    SONG_CUDA(song::upload_half(x->entry_p, &x->d_entry_w), "entry weights");
    SONG_CUDA(song::upload_half(x->stop_p, &x->d_stop_w), "stop weights");
    x->has_model = true;
    return SONG_OK;
}

song_status song_index_learn(song_index* x, const song_learn_params* lp,
                             const float* d_train_queries, int nq, const int32_t* d_train_nn1,
                             song_learn_report* report) {
    if (x == nullptr || lp == nullptr) return fail(SONG_ERR_INVALID_ARG, "index or params is NULL");
    if (x->kind != SONG_KIND_L2) return fail(SONG_ERR_UNSUPPORTED, "learned models apply to L2 indexes");
    if (nq < 1 || d_train_queries == nullptr || d_train_nn1 == nullptr)
        return fail(SONG_ERR_INVALID_ARG, "training queries / nearest neighbours missing");
    if (lp->k < 1 || lp->ef < 1 || lp->ckpt_every < 1 || lp->max_ckpt < 1 || lp->batch < 1)
        return fail(SONG_ERR_INVALID_ARG, "bad learn parameters");
    std::lock_guard<std::mutex> lock(x->mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != x->device) SONG_CUDA(cudaSetDevice(x->device), "cudaSetDevice");
    const int ef = clamp_ef(lp->ef, lp->k, x->p.pq_size);
    int32_t* d_ids = nullptr;
    SONG_CUDA(cudaMalloc(&d_ids, (size_t)nq * lp->k * 4), "train ids alloc");
    song::SearchArgs a;
    song_status s = make_args(x, d_train_queries, nq, lp->k, ef, d_ids, nullptr, &a);
    if (s != SONG_OK) {
        cudaFree(d_ids);
        return s;
    }
    unsigned* ctr = x->d_counter + 2 * (x->counter_next++ % kCounterRing);
    a.counter = ctr;
    a.done = ctr + 1;
    a.ckpt_every = lp->ckpt_every;
    a.min_expansions = lp->min_expansions;
    // The entry stage: a hub set of entry_hubs nodes (a seeded sample) laid out
    // for the tensor cores; the training queries' candidates feed the traces.
    const bool staged = lp->entry_hubs > 0 && x->dim <= song::kEntryMaxDim;
    int32_t* d_tc = nullptr;
    float* d_td = nullptr;
    if (staged) {
        const int64_t H = std::min<int64_t>(lp->entry_hubs, x->n);
        std::vector<int32_t> perm((size_t)x->n);
        for (int64_t i = 0; i < x->n; ++i) perm[(size_t)i] = (int32_t)i;
        std::mt19937_64 rng(lp->seed * 0x9E3779B97F4A7C15ull + 17u);
        for (int64_t i = 0; i < H; ++i) {  // partial Fisher-Yates
            std::uniform_int_distribution<int64_t> pick(i, x->n - 1);
            std::swap(perm[(size_t)i], perm[(size_t)pick(rng)]);
        }
        perm.resize((size_t)H);
        std::sort(perm.begin(), perm.end());
        song_status s3 = attach_entry_hubs(x, perm);
        cudaError_t e3 = cudaSuccess;
        if (s3 == SONG_OK) {
            e3 = cudaMalloc(&d_tc, (size_t)nq * song::kEntryK * 4);
            if (e3 == cudaSuccess) e3 = cudaMalloc(&d_td, (size_t)nq * song::kEntryK * 4);
            if (e3 != cudaSuccess) s3 = cuda_fail(e3, "entry candidates alloc");
        }
        if (s3 == SONG_OK) s3 = run_entry(x, d_train_queries, nq, d_tc, d_td, x->stream);
        if (s3 != SONG_OK) {
            cudaFree(d_ids);
            cudaFree(d_tc);
            cudaFree(d_td);
            return s3;
        }
        a.ecand = d_tc;
        a.edist = d_td;
    }
    song::LearnInputs in{};
    in.args = a;
    in.base = x->d_base;
    in.n = x->n;
    in.dim = x->dim;
    in.ld = x->ld;
    in.nn1 = d_train_nn1;
    in.nq = nq;
    in.max_ckpt = lp->max_ckpt;
    in.entry_steps = lp->entry_steps;
    in.stop_steps = lp->stop_steps;
    in.batch = lp->batch;
    in.lr = lp->lr;
    in.seed = lp->seed;
    in.num_sms = x->num_sms;
    in.stream = x->stream;
    song::LearnOutputs out;
    cudaError_t e = song::learn_models(in, &out);
    cudaFree(d_ids);
    cudaFree(d_tc);
    cudaFree(d_td);
    if (e != cudaSuccess) return cuda_fail(e, "learn");
    x->hubs = out.hubs;
    x->model_staged = staged;
    x->entry_p = out.entry;
    x->stop_p = out.stop;
    x->ckpt_every = lp->ckpt_every;
    x->min_expansions = lp->min_expansions;
    x->model_k = lp->k;
    if (song_status s2 = attach_model(x)) return s2;
    if (report) {
        report->n_hubs = staged ? (int)x->entry_hubs.size() : (int)out.hubs.size();
        report->stop_samples = out.stop_samples;
        report->entry_loss_first = out.entry_loss_first;
        report->entry_loss_last = out.entry_loss_last;
        report->stop_loss_first = out.stop_loss_first;
        report->stop_loss_last = out.stop_loss_last;
        report->stop_pos_frac = out.stop_pos_frac;
    }
    return SONG_OK;
}

static const uint32_t kModelMagic = 0x534f4e47u;  // "SONG"

song_status song_index_get_model(const song_index* x, float* blob, int capacity, int* length) {
    if (x == nullptr || length == nullptr) return fail(SONG_ERR_INVALID_ARG, "index or length is NULL");
    if (!x->has_model) return fail(SONG_ERR_INVALID_ARG, "no learned model attached");
    std::vector<float> v;
    auto put_u = [&](uint32_t u) { float f; std::memcpy(&f, &u, 4); v.push_back(f); };
    // version 1: [magic 1 n_hubs ckpt min_exp k n_entry n_stop] hubs entry stop
    // version 2 (entry stage): [magic 2 n_out ckpt min_exp k n_entry n_stop n_set] set entry stop
    put_u(kModelMagic);
    put_u(x->model_staged ? 2u : 1u);
    put_u(x->model_staged ? (uint32_t)song::kEntryK : (uint32_t)x->hubs.size());
    put_u((uint32_t)x->ckpt_every);
    put_u((uint32_t)x->min_expansions);
    put_u((uint32_t)x->model_k);
    put_u((uint32_t)x->entry_p.size());
    put_u((uint32_t)x->stop_p.size());
    if (x->model_staged) {
        put_u((uint32_t)x->entry_hubs.size());
        for (int32_t h : x->entry_hubs) put_u((uint32_t)h);
    } else {
        for (int32_t h : x->hubs) put_u((uint32_t)h);
    }
    v.insert(v.end(), x->entry_p.begin(), x->entry_p.end());
    v.insert(v.end(), x->stop_p.begin(), x->stop_p.end());
    *length = (int)v.size();
    if (blob != nullptr) {
        if (capacity < (int)v.size()) return fail(SONG_ERR_INVALID_ARG, "blob capacity too small");
        std::memcpy(blob, v.data(), v.size() * 4);
    }
    return SONG_OK;
}

song_status song_index_set_model(song_index* x, const float* blob, int length) {
    if (x == nullptr || blob == nullptr || length < 8) return fail(SONG_ERR_INVALID_ARG, "bad model blob");
    auto get_u = [&](int i) { uint32_t u; std::memcpy(&u, blob + i, 4); return u; };
    const uint32_t ver = get_u(1);
    if (get_u(0) != kModelMagic || (ver != 1 && ver != 2)) return fail(SONG_ERR_INVALID_ARG, "not a model blob");
    const int nh = (int)get_u(2), ne = (int)get_u(6), ns = (int)get_u(7);
    const int hdr = ver == 2 ? 9 : 8;
    const int nset = ver == 2 ? (length >= 9 ? (int)get_u(8) : -1) : nh;
    if (nh < 1 || nh > song::kFeat || (ver == 2 && nh != song::kEntryK) || nset < 1 ||
        ne != song::mlp_param_count(nh) || ns != song::mlp_param_count(1) ||
        length != hdr + nset + ne + ns)
        return fail(SONG_ERR_INVALID_ARG, "model blob sizes do not match");
    std::lock_guard<std::mutex> lock(x->mu);
    std::vector<int32_t> ids((size_t)nset);
    for (int i = 0; i < nset; ++i) {
        ids[(size_t)i] = (int32_t)get_u(hdr + i);
        if (ids[(size_t)i] < 0 || ids[(size_t)i] >= x->n) return fail(SONG_ERR_INVALID_ARG, "hub id out of range");
    }
    if (ver == 2) {
        if (song_status s2 = attach_entry_hubs(x, ids)) return s2;
        x->hubs.clear();
    } else {
        x->hubs = ids;
    }
    x->model_staged = ver == 2;
    x->ckpt_every = (int)get_u(3);
    x->min_expansions = (int)get_u(4);
    x->model_k = (int)get_u(5);
    x->entry_p.assign(blob + hdr + nset, blob + hdr + nset + ne);
    x->stop_p.assign(blob + hdr + nset + ne, blob + hdr + nset + ne + ns);
    return attach_model(x);
}

song_status song_mlp_grad(int out, int loss_kind, const float* params, const float* x,
                          const float* y, const float* sample_weight, int batch, float* grad,
                          double* loss) {
    if (out < 1 || out > 64 || (loss_kind == 0 && out != 1) || loss_kind < 0 || loss_kind > 1 ||
        batch < 1 || !params || !x || !y || !grad || !loss)
        return fail(SONG_ERR_INVALID_ARG, "bad mlp_grad arguments");
    cudaError_t e = song::mlp_grad(params, out, loss_kind, x, y, sample_weight, batch, grad, loss);
    if (e != cudaSuccess) return cuda_fail(e, "mlp_grad");
    return SONG_OK;
}

int64_t song_kernel_launch_count(void) { return song::g_launches.load(); }

}  // extern "C"
