// song_kernels.cuh -- launch interface of the sm_100a search kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include <vector>

#include "song_b200.h"

namespace song {

// Everything one search launch needs.  All pointers are device pointers.
struct SearchArgs {
    const void* base;        // FP32 [n x ld] (L2) or u32 [n x ld] (Hamming)
    const int32_t* adj;      // [n x block_size], -1 = empty slot
    const void* queries;     // [nq x qld], same element type as base
    int32_t* out;            // [nq x k], best-first, -1 padded
    song_query_trace* trace; // [nq] or nullptr
    unsigned* counter;       // work counter: must be 0 at launch
    unsigned* done;          // nullable: CTAs past their loop; the last one zeroes counter and done
    int* err;                // set non-zero if an adjacency entry is out of range
    int64_t n;
    int dim;                 // elements compared per row (floats or u32 words)
    int ld;                  // row stride of base, elements (multiple of 4)
    int qld;                 // row stride of queries, elements
    int block_size;          // BLOCK_SIZE
    int k;
    int nq;
    int cap;                 // queue capacity = clamp(ef, 1, pq_size)
    int bf_words;            // BF_WORDS
    int bf_nhash;            // BF_NHASH (1..4)
    int n_multiprobe;        // N_MULTIPROBE
    const int32_t* qseeds;   // [nq x n_qseeds] entry points per query (-1 = none), or nullptr
    int n_qseeds;            // 1..32
    int warp_smem;           // bytes of shared memory per warp (multiple of 16)
    int q_off, rows_off, cd_off, ci_off, rd_off, ri_off, bl_off;  // per-warp carve-up, bytes
    int tm_cols;             // TMEM columns one CTA allocates (set by launch_search)
    int tm_warp_cols;        // TMEM columns of one warp's queue ids (set by launch_search)
    int int_base;            // 1: every base value is an integer in [base_min, base_max]
    float base_min, base_max;
    const uint8_t* u8;       // base values as bytes [n x u8_ld] when all are integers in [0, 255]
    int u8_ld;               // bytes per byte row (multiple of 16)
    // precision form (prec != SONG_PREC_FP32)
    int prec;                // SONG_PREC_FP32 / SONG_PREC_BF16 / SONG_PREC_FP8
    const void* lowp;        // compressed rows [n x lowp_ld bytes]
    const float* scales;     // FP8: per-vector scale [n]
    int lowp_ld;             // bytes per compressed row (multiple of 128)
    int qdim;                // floats of the query kept in shared memory (padded dim)
    int rerank;              // 1: exact FP32 re-rank of the final results queue
    float* out_dist;         // [nq x k] distance of each output id (nullable)
    // learned entry / stop (lm: 0 off, 1 collect traces of the full search, 2 infer)
    int lm;
    int no_entry_stage;      // learned searches: 1 = skip the entry stage (reference seeds)
    const int32_t* ecand;    // [nq x kEntryK] entry-stage candidates (hub node ids, -1 = none), or nullptr
    const float* edist;      // [nq x kEntryK] their squared distances
    const int32_t* hubs;     // [n_hubs] entry hub node ids (n_hubs <= kFeat)
    int n_hubs;
    const __half* entry_w;   // packed entry MLP (kFeat -> kHid -> kHid -> n_hubs), nullable
    const __half* stop_w;    // packed stop MLP (kFeat -> kHid -> kHid -> 1), nullable
    int beam;                // learned searches: candidates expanded per step (1 to 4)
    int ckpt_every;          // expansions between stop checkpoints
    int min_expansions;      // no learned stop before this many expansions
    float stop_thr;          // stop when sigmoid(stop logit) >= stop_thr
    int max_ckpt;            // checkpoints per query in the trace buffers
    float* tr_feat;          // [nq x max_ckpt x kFeat] stop features
    float* tr_kth;           // [nq x max_ckpt] k-th best distance at each checkpoint
    int* tr_count;           // [nq] checkpoints written
    float* tr_final_kth;     // [nq] k-th best distance at the end of the search
    float* tr_entry_feat;    // [nq x kFeat] entry features (hub distances)
};

// Learned model geometry: kFeat inputs, two hidden layers of kHid (ReLU).
constexpr int kFeat = 24;
constexpr int kHid = 64;
// Packed FP16 / FP32 parameter layout: W1[kHid][kFeat] b1[kHid] W2[kHid][kHid] b2[kHid]
// W3[out][kHid] b3[out].
constexpr int mlp_param_count(int out) { return kHid * kFeat + kHid + kHid * kHid + kHid + out * kHid + out; }

// Entry points of the learned search (song_entry.cu): every query's
// kEntryK nearest hubs from a hub set laid out as BF16 tensor-core tiles.
constexpr int kEntryK = kFeat;
constexpr int kEntryMaxDim = 288;
int entry_padded_dim(int dim);
int entry_tile_hubs();
size_t entry_smem_bytes(int dim);
// Lay out hubs (node ids, -1 = padding; hpad a multiple of entry_tile_hubs())
// of FP32 base rows as BF16 tiles [hpad x entry_padded_dim(dim)] and their
// squared norms (+inf for padding).  Stream-ordered.
cudaError_t build_entry_tables(const float* d_base, int ld, int dim, const int32_t* d_ids,
                               int hpad, __nv_bfloat16* d_tiles, float* d_norm, cudaStream_t st);
// out_ids / out_d [nq x kEntryK]: each query's nearest hubs (node ids, -1 if
// none) and squared distances, nearest first.  err is set to 2 if a bounded
// wait gives up.
// split_scratch (nullable, split_bytes long; entry_split_scratch_bytes(nq,
// num_sms) is enough for the widest split) lets the hub tiles of each 128
// queries spread over several CTAs; the last CTA of each 128 queries merges
// their lists (the scratch also holds the arrival counters, zeroed by an
// asynchronous memset on the stream before each launch).
constexpr int kEntrySplits = 16;
size_t entry_split_scratch_bytes(int nq, int num_sms);
// overlap: the scratch's arrival counters are zero (the kernel leaves them
// so) and the launch may start while the previous search launch on the stream
// finishes its tail; it ends after that launch.  Otherwise a memset zeroes the
// counters first and the launch is ordinary.
// keep: how many of the nearest hubs the caller reads (the rest of each
// kEntryK row is -1 / +inf); the first `keep` entries are those of the full
// list.  kEntryK for the entry model's features.
cudaError_t launch_entry(const float* d_queries, int qld, int nq, int dim,
                         const __nv_bfloat16* d_tiles, const float* d_norm, const int32_t* d_ids,
                         int hpad, int32_t* d_out_ids, float* d_out_d, int* d_err,
                         cudaStream_t st, void* split_scratch, size_t split_bytes, int num_sms,
                         bool overlap = false, int keep = kEntryK);

// Graph::search (graph.h:33-115) bit for bit (song_graphsearch.cu).
int graph_search_frontier_cap(int ef);
size_t graph_search_warp_smem(int dim, int ef);
int64_t graph_search_resident_warps(int dim, int ef, int num_sms, int dev);
cudaError_t launch_graph_search(const float* d_base, int ld, int dim, const int32_t* d_adj, int bs,
                                int64_t n, const float* d_queries, int nq, int k, int ef, int nmp,
                                int32_t* d_out, song_query_trace* d_trace, unsigned* d_counter,
                                int* d_err, uint32_t* d_visited, int64_t visited_slots,
                                int num_sms, cudaStream_t st);

// Padded element count of a compressed row (a whole number of 128-byte
// lines per 8-lane group) and its byte stride.
int lowp_padded_dim(int prec, int dim);

// Fill the compressed copy of the FP32 rows: BF16 (round to nearest even) or
// FP8 e4m3 with a per-vector scale amax/448.  Stream-ordered.
cudaError_t quantize_rows(int prec, const float* d_rows, int64_t n, int dim, int ld, void* d_out,
                          int out_ld, float* d_scales, cudaStream_t st);

// Integer range of FP32 rows (0 in int_base if any value is not an integer).
struct BaseRange {
    int int_base = 0;
    float lo = 0.0f, hi = 0.0f;
};
BaseRange scan_base_range(const float* rows, int64_t n, int dim);

// Byte rows of integer-valued vectors: at most kU8MaxDim elements, each row
// zero padded to u8_row_bytes(dim) (a multiple of 16) -- the exact-integer
// distance path then reads whole 16-byte chunks.
constexpr int kU8MaxDim = 256;
int u8_row_bytes(int dim);
cudaError_t convert_rows_u8(const float* d_rows, int64_t n, int dim, int ld, uint8_t* d_out,
                            int out_ld, cudaStream_t st);

// Row stride (elements) the kernels use for `dim` elements of `kind`.
int search_row_stride(int kind, int dim);

// Per-warp shared-memory layout for (kind, query floats, cap, bf_words).
int search_warp_smem(int kind, int dim, int cap, int bf_words, SearchArgs* a);

// Launch the plain search on `stream`: chooses the kernel instance for
// (kind, dim), the warps per CTA and a persistent grid.  Returns a CUDA error.
cudaError_t launch_search(int kind, const SearchArgs& a, int num_sms, cudaStream_t stream);

// Batched-insertion NSW build over device rows (song_build.cu).
cudaError_t build_graph_device(int kind, const void* d_base, int64_t n, int dim, int ld,
                               const song_params& p, int ratio, int bf_words, int32_t* d_adj,
                               int num_sms, cudaStream_t st, BaseRange range = BaseRange());

// Scratch bytes build_graph_with_scratch needs for (n, params, ratio).
size_t build_scratch_bytes(int64_t n, const song_params& p, int ratio);

// build_graph_device with all temporaries carved from caller scratch; no
// allocation, stream-ordered, does not wait.
cudaError_t build_graph_with_scratch(int kind, const void* d_base, int64_t n, int dim, int ld,
                                     const song_params& p, int ratio, int bf_words,
                                     int32_t* d_adj, int num_sms, cudaStream_t st, void* scratch,
                                     size_t scratch_bytes);

// Serving ring (song_serve.cu): slot = 32-byte header {long long ticket; int k;
// int cap; int flags; ...} then the query (dim floats).
constexpr int kServeHeader = 32;
constexpr int kServeLearned = 1;  // request flag: learned entry/stop
struct ServeArgs {
    SearchArgs base;            // index-wide arguments (per-warp layout sized for max_cap)
    const unsigned char* ring;  // device [slots x slot_bytes]
    int slot_bytes, slots, max_k;
    long long* head;            // device: next ticket to claim
    const volatile long long* tail;  // device: tickets published (written by host copies)
    const volatile long long* stop;  // device: non-zero = shut down (set by a host copy)
    int32_t* res_ids;           // mapped host [slots x max_k]
    float* res_dist;            // mapped host [slots x max_k]
    song_query_trace* res_trace;  // mapped host [slots]
    long long* res_done;        // mapped host [slots]: ticket completed in the slot
    long long* last_claim;      // device: %globaltimer (ns) of the latest claim
    long long* exits;           // device [3]: warps that left idle, at the poll cap, at the stop word
    const int32_t* scand;       // device [slots x kEntryK]: entry-stage candidates per slot, or nullptr
    const float* sdist;         // device [slots x kEntryK]: their squared distances
    long long idle_ns;          // a warp leaves once no request was claimed for this long
    int max_idle_polls, sleep_ns;  // hard bound on consecutive empty polls; poll backoff cap
};
// reserve_sms > 0: one CTA per SM on num_sms - reserve_sms SMs, leaving the
// rest to the entry stage (a learned model with a hub set).
cudaError_t launch_serve(const ServeArgs& s, int num_sms, int max_ctas, int reserve_sms,
                         cudaStream_t st, int* warps_out);

// Training of the learned entry / stop models (song_learn.cu).
struct LearnInputs {
    SearchArgs args;         // plain full-budget search over the training queries (cap = ef, k)
    const void* base;        // FP32 rows [n x ld]
    int64_t n;
    int dim, ld;
    const int32_t* nn1;      // [nq] exact nearest neighbour of each training query
    int nq, max_ckpt, entry_steps, stop_steps, batch;
    float lr;
    uint64_t seed;
    int num_sms;
    cudaStream_t stream;
};
struct LearnOutputs {
    std::vector<int32_t> hubs;
    std::vector<float> entry, stop;  // FP32 master parameters (packed layout)
    double entry_loss_first = 0, entry_loss_last = 0, stop_loss_first = 0, stop_loss_last = 0;
    double stop_pos_frac = 0;
    int64_t stop_samples = 0;
};
cudaError_t learn_models(const LearnInputs& in, LearnOutputs* out);
cudaError_t upload_half(const std::vector<float>& P, __half** d);
cudaError_t mlp_grad(const float* hP, int out, int loss_kind, const float* hX, const float* hY,
                     const float* hW, int B, float* hG, double* loss);

// Index accessors used by the server (song_capi.cu).
song_status server_args(song_index* x, const song_search_opts* opts, int max_k, int max_cap,
                        SearchArgs* a, int* num_sms, int* device);
int index_pq_size(const song_index* x);
int index_dim(const song_index* x);
bool index_has_model(const song_index* x);
// The learned model scores the entry stage's candidates (song_index_learn
// with entry_hubs > 0); index_entry runs that stage on nq queries that are
// qld floats apart.
bool index_model_staged(const song_index* x);
cudaError_t index_entry(song_index* x, const float* d_q, int qld, int nq, int32_t* d_ids,
                        float* d_d, cudaStream_t st, void* split_scratch, size_t split_bytes);

// Records a failure message for song_last_error() on the calling thread.
song_status set_error(song_status status, const char* message);

}  // namespace song
