/*
 * song_b200.h -- C ABI of the B200-native SONG graph search.
 *
 * Drop-in boundary for the reference's search path (lrlorry/2020_song_ex):
 * plain pointers and sizes, no C++ or torch types.  Every entry point
 * returns a song_status; song_last_error() gives the message of the last
 * failure on the calling thread.  The reference checks no errors at all
 * (its CUDA calls are unchecked, kernalGraph.h:39-45, :326-380).
 *
 * Semantics follow the reference GPU search exactly: for the same graph,
 * queries and parameters the plain search returns the same top-k ids, in the
 * same order including ties, and the same per-query QueryTrace counters as
 * kg_search_kernel (kernalGraph.h:184-299) / hkg_search_kernel
 * (hashKernelGraph.h:238-352).
 */
#ifndef SONG_B200_H
#define SONG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int song_status;
#define SONG_OK                0
#define SONG_ERR_INVALID_ARG   1  /* bad size, pointer, parameter or graph entry   */
#define SONG_ERR_OOM           2  /* device allocation failed                       */
#define SONG_ERR_CUDA          3  /* a CUDA call failed (message has the reason)    */
#define SONG_ERR_TIMEOUT       4  /* a bounded wait gave up                          */
#define SONG_ERR_BUDGET        5  /* request exceeds a memory budget                 */
#define SONG_ERR_UNSUPPORTED   6  /* parameters outside what the kernels implement   */

/* Distance precision of a search (song_search_opts.precision). */
#define SONG_PREC_FP32  0        /* the plain search: bit-exact with the reference             */
#define SONG_PREC_BF16  1        /* traversal on BF16 rows, FP32 accumulation                  */
#define SONG_PREC_FP8   2        /* traversal on FP8 e4m3 rows with a per-vector FP32 scale    */

/* Index kinds. */
#define SONG_KIND_L2       0     /* FP32 vectors, squared L2 (kernalGraph.h)          */
#define SONG_KIND_HAMMING  1     /* packed u32 sign codes, Hamming (hashKernelGraph.h) */

/*
 * Search/build parameters: the compile-time constants of config.h:9-58 as
 * runtime values.  song_params_default() fills the reference defaults.
 */
typedef struct song_params {
    int block_size;       /* BLOCK_SIZE      config.h:9   adjacency slots per node      */
    int fixed_degree;     /* FIXED_DEGREE    config.h:12  (graph builder)               */
    int search_degree;    /* SEARCH_DEGREE   config.h:17  (graph builder)               */
    int ef_construction;  /* EF_CONSTRUCTION config.h:24  (graph builder)               */
    int pq_size;          /* pq_size         config.h:28  queue capacity cap            */
    int topk;             /* TOPK            config.h:31                                */
    int n_multiprobe;     /* N_MULTIPROBE    config.h:34  entry points p*n/N            */
    int n_multiquery;     /* N_MULTIQUERY    config.h:38  queries staged per batch      */
    int hash_bits;        /* hash_bits       config.h:41  sign-projection code length   */
    int bf_words;         /* BF_WORDS        config.h:56  Bloom filter 64-bit words     */
    int bf_nhash;         /* BF_NHASH        config.h:58  Bloom hashes (1..4)           */
} song_params;

/* QueryTrace (telemetry.h:5-18): 12 int counters, same order and layout. */
typedef struct song_query_trace {
    int seed_count;
    int visited_nodes;
    int expanded_nodes;
    int neighbor_slots_scanned;
    int candidate_nodes;
    int distance_evals;
    int frontier_pushes;
    int result_updates;
    int peak_frontier;
    int peak_results;
    int result_count;
    int early_stopped;
} song_query_trace;

/* The scalar part of GpuSearchTrace (telemetry.h:30-41). Times in ms. */
typedef struct song_timing {
    double alloc_ms;      /* host time of staging-buffer growth */
    double h2d_ms;        /* CUDA-event time of the query copies */
    double memset_ms;
    double kernel_ms;     /* CUDA-event time of the search kernels */
    double d2h_ms;        /* CUDA-event time of the result copies */
    double total_ms;      /* host time of the call after allocation */
    int ef_search;        /* ef after the reference clamp */
    int batch_limit;      /* n_multiquery as passed */
    int n_batches;
} song_timing;

typedef struct song_index song_index;

/*
 * Options of the extended searches (no counterpart in the reference, whose
 * only search is the plain one).  A zeroed struct selects the plain search.
 */
typedef struct song_search_opts {
    int precision;        /* SONG_PREC_*; BF16/FP8 need song_index_set_precision()      */
    int rerank;           /* 1: re-rank the final results queue with exact FP32 distances */
    int learned;          /* 1: use the index's learned entry/stop model                 */
    float stop_threshold; /* learned stop: stop when P(converged) >= threshold           */
    int beam;             /* learned search: 2..4 = expand that many best candidates per
                             step (their adjacency rows in one round trip; BLOCK_SIZE
                             <= 32; values above 4 act as 4); 0 or 1 = one per step,
                             the reference's order                                     */
    int bloom_hashes;     /* learned search: Bloom hashes per id (1..4) in place of the
                             index's bf_nhash (BF_NHASH); 0 = the index's value.  Plain
                             searches reject it: they keep the reference's visited set */
    int entry;            /* learned search, entry points (SONG_ENTRY_*): 0 = the entry
                             model's top N_MULTIPROBE hubs; 1 = the N_MULTIPROBE nearest
                             hubs of the entry stage, no model; 2 = the reference's seeds
                             p*n/N_MULTIPROBE, no entry stage.  1 and 2 measure what the
                             entry model and the entry stage contribute              */
    int reserved;
} song_search_opts;

#define SONG_ENTRY_MODEL   0
#define SONG_ENTRY_NEAREST 1
#define SONG_ENTRY_SEEDS   2

/* Reference defaults of config.h:9-58. */
void song_params_default(song_params* p);

/* Message of the last failed call on this thread ("" if none). */
const char* song_last_error(void);

/* Library version string. */
const char* song_version(void);

/*
 * Create an L2 index: uploads data[n x dim] (FP32, row-major) and
 * adj[n x block_size] (int32, -1 = empty slot) to the current CUDA device.
 * Replaces KernelGraph + upload_to_gpu (kernalGraph.h:20-43).  Every adj
 * entry must be -1 or a node id in [0, n).
 */
song_status song_index_create_l2(const float* data, int64_t n, int dim, const int32_t* adj,
                                 const song_params* params, song_index** out);

/*
 * Create a Hamming index over packed codes[n x hash_words] (u32).
 * Replaces HashKernelGraph + upload_to_gpu (hashKernelGraph.h:22-98).
 * hash_words must be a multiple of 4 and at most 32.
 */
song_status song_index_create_hamming(const uint32_t* codes, int64_t n, int hash_words,
                                      const int32_t* adj, const song_params* params,
                                      song_index** out);

/* Frees the device copies (the KernelGraph destructor, kernalGraph.h:45). */
song_status song_index_destroy(song_index* index);

/* n, dim (floats or code words) and kind of an index. */
song_status song_index_info(const song_index* index, int64_t* n, int* dim, int* kind);

/*
 * Whether an L2 index keeps a byte copy of its rows (no counterpart in the
 * reference).  When every base value is an integer in [0, 255] (and dim <=
 * 256) the index stores the rows also as bytes, row_bytes each; the plain and
 * learned searches then compute the distances of queries whose values are
 * integers in [0, 255] from those bytes, exactly (the same FP32 distances as
 * the reference's float arithmetic, which is exact for such vectors), and
 * gather a quarter of the bytes.
 */
song_status song_index_u8_rows(const song_index* index, int* has_u8, int* row_bytes);

/*
 * gpu_search (kernalGraph.h:307-382): host queries[nq x dim] in, host
 * ids[nq x k] out (best-first, -1 padded).  ef_search is clamped exactly as
 * the reference does (raise to k, then cap at pq_size).  traces (host,
 * nq entries) and timing may be NULL.  Synchronous, like the reference.
 */
song_status song_gpu_search(song_index* index, const float* queries, int nq, int k,
                            int n_multiquery, int ef_search, int32_t* ids,
                            song_query_trace* traces, song_timing* timing);

/* gpu_search overload of hashKernelGraph.h:360-435 on u32 query codes. */
song_status song_gpu_search_hamming(song_index* index, const uint32_t* queries, int nq, int k,
                                    int n_multiquery, int ef_search, int32_t* ids,
                                    song_query_trace* traces, song_timing* timing);

/*
 * The reference's CPU search, Graph::search (graph.h:33-115), on the GPU:
 * exact visited set, unbounded frontier and top-ef ordered by (distance,
 * id), distances summed in dimension order.  For the same graph, queries
 * and ef the ids (worst-first, as Graph::search returns them, -1 padded to
 * k) and all twelve QueryTrace counters equal the reference's bit for bit.
 * ef_search is raised to k (graph.h:36); it must be 1..1024 and at least
 * N_MULTIPROBE.  L2 indexes.  Host buffers, synchronous; the device form is
 * asynchronous on `stream`.
 */
song_status song_graph_search(song_index* index, const float* queries, int nq, int k,
                              int ef_search, int32_t* ids, song_query_trace* traces);
song_status song_graph_search_device(song_index* index, const float* d_queries, int nq, int k,
                                     int ef_search, int32_t* d_ids, song_query_trace* d_traces,
                                     void* stream);

/*
 * Device-resident search: d_queries (FP32 or u32 codes, by index kind),
 * d_ids[nq x k] and d_traces (nullable) are device pointers; the call is
 * asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream).
 * Same clamp and results as song_gpu_search.  Searches of one index may
 * run on different streams at the same time: each launch takes its own work
 * counter (a ring of 1024 per index), its own entry-stage lists (learned
 * searches: a ring of 16 slots per index, so at most 16 learned searches of
 * one index may be in flight at once) and its own Graph::search bitmaps
 * (from the index's stream-ordered memory pool, freed on the launching
 * stream).  Consecutive plain searches on one stream, and a learned search's
 * entry stage after the previous search on its stream, may overlap that
 * launch's tail; each writes its results only after the launch before it
 * has finished.  Host calls on one index are serialised by a lock.  One thing is shared: the index's error word.  A kernel that meets
 * an out-of-range id (a corrupted graph or caller seed) sets it instead of
 * reading out of range, and every host call clears it before its own
 * launches and reports it after them, so with searches of one index running
 * on several streams at once an error is reported by whichever host call
 * reads the word next, not necessarily by the call whose launch set it.
 */
song_status song_search_device(song_index* index, const void* d_queries, int nq, int k,
                               int ef_search, int32_t* d_ids, song_query_trace* d_traces,
                               void* stream);

/*
 * Build an NSW graph on the current GPU: the reference's insertion algorithm
 * (kernalGraph.h:140-149 / hashKernelGraph.h:196-207 -- beam search from
 * node 0 with EF_CONSTRUCTION, SEARCH_DEGREE forward edges, reverse edges
 * with farthest-eviction up to FIXED_DEGREE) run in batches of
 * max(1, inserted/batch_ratio) nodes.  Same graph shape and rules, not
 * byte-identical to the reference's sequential build.
 * rows: FP32 [n x dim] (kind SONG_KIND_L2) or u32 codes [n x dim]
 * (SONG_KIND_HAMMING), host.  adj_out: host [n x block_size].
 * batch_ratio <= 0 selects 32; build_bf_words <= 0 selects 1024.  A small
 * graph of high-dimensional points may want a larger ratio (smaller
 * batches): on 8,000 x 960 points 128 gave recall@10 0.79 against 0.61 for
 * 32 (reference builder 0.75), while on 1,000,000 x 960 points 32 gave the
 * better graph.
 * fixed_degree must be <= 32 and <= block_size.
 */
song_status song_build_graph(int kind, const void* rows, int64_t n, int dim,
                             const song_params* params, int batch_ratio, int build_bf_words,
                             int32_t* adj_out);

/*
 * Allocation-free song_build_graph (no counterpart in the reference).
 * For callers that cannot call cudaMalloc while they build a graph: a
 * serving process whose device memory is owned by its own pool, or one that
 * must not let an allocation synchronise the device under live traffic.
 * d_rows ([n x ld] FP32 or u32 codes, ld a multiple of 4, 16-byte aligned)
 * and d_adj ([n x block_size], written) are the caller's device buffers; all
 * temporaries live in one fixed 16 MiB device array inside this library,
 * which every GPU that loads the library holds until the process exits.  A
 * build whose temporaries do not fit is rejected with SONG_ERR_BUDGET (the
 * message gives the bytes needed; a larger batch_ratio needs less).
 * Asynchronous on `stream` (a cudaStream_t).  The first call on a device
 * looks up the array's device address, so make that first call before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race with each other.  The library must not be used on a device after a
 * cudaDeviceReset (the looked-up address would be stale).  Row words or
 * floats past dim (ld > dim) are ignored, whatever they hold.  Produces the
 * same graph as song_build_graph.
 */
song_status song_build_graph_noalloc(int kind, const void* d_rows, int64_t n, int dim, int ld,
                                     const song_params* params, int batch_ratio,
                                     int build_bf_words, int32_t* d_adj, void* stream);

/*
 * BitHash (bitHash.h:17-56): sign-random-projection codes for the Hamming
 * index.  song_bithash_matrix is the constructor BitHash(dim, seed)
 * (bitHash.h:23-27): R[hash_bits x dim] (host, row-major) drawn from
 * std::mt19937(seed) and std::normal_distribution<float>(0, 1), the same
 * generator calls as the reference.  song_bithash_project is project_all
 * (bitHash.h:51-56) on the GPU: codes[n x hash_bits/32] (host) with bit b of
 * word w set when the FP32 dot of R[w*32+b] with x[i] is > 0, summed in
 * increasing d with a separate multiply and add per step exactly as the
 * reference's -O3 host build computes it, so the codes are bit-identical.
 * hash_bits must be a positive multiple of 32 (HASH_WORDS = hash_bits/32,
 * config.h:44).  Synchronous.
 */
song_status song_bithash_matrix(int dim, int hash_bits, unsigned seed, float* R);
song_status song_bithash_project(const float* R, int dim, int hash_bits, const float* x,
                                 int64_t n, uint32_t* codes);
/* Device-pointer project_all: x[n x ldx] FP32 (ldx >= dim elements), R as
 * above, codes[n x ldc] u32 (ldc >= hash_bits/32 words; words beyond
 * hash_bits/32 are left untouched).  Asynchronous on `stream`. */
song_status song_bithash_project_device(const float* d_R, int dim, int hash_bits,
                                        const float* d_x, int64_t n, int64_t ldx,
                                        uint32_t* d_codes, int64_t ldc, void* stream);

/*
 * Exact k nearest neighbours by squared L2 (the ground truth recall is
 * measured against).  Replaces the reference's brute force
 * (bench_cpu.cpp:158-175, main.cpp:14-49; numpy in run_compare.py:199-213).
 * Distances are |q|^2 - 2 q.b + |b|^2 with the cross term from 3xBF16
 * split products on the tensor cores (FP32 accumulation; exact for integer
 * data in [0, 255] with dim <= 128).  Output per query: k ids ascending by
 * (distance, id), -1 / +inf when n < k.  1 <= k <= 128.
 * The device form takes device buffers (row strides ldb, ldq in floats) and
 * returns when the result is on the device (it synchronises `stream`).
 */
song_status song_exact_knn_device(const float* d_base, int64_t n, int64_t ldb, int dim,
                                  const float* d_queries, int nq, int64_t ldq, int k,
                                  int32_t* d_ids, float* d_dists, void* stream);
song_status song_exact_knn(const float* base, int64_t n, int dim, const float* queries, int nq,
                           int k, int32_t* ids, float* dists);

/*
 * Attach a compressed copy of an L2 index's vectors for the precision form
 * (SONG_PREC_BF16 or SONG_PREC_FP8), converted on the GPU from the FP32
 * copy, which stays resident for the exact re-rank.  Replaces an earlier
 * compressed copy.
 */
song_status song_index_set_precision(song_index* index, int precision);

/*
 * The extended search on device pointers: opts selects precision, FP32
 * re-rank and the learned model; d_dists (nullable) receives the distance
 * of every output id (the FP32 distance after a re-rank).  With a zeroed
 * opts (or NULL) it is song_search_device plus distances.
 */
song_status song_search_device_ex(song_index* index, const song_search_opts* opts,
                                  const void* d_queries, int nq, int k, int ef_search,
                                  int32_t* d_ids, float* d_dists, song_query_trace* d_traces,
                                  void* stream);

/*
 * The extended search from caller-chosen entry points (no counterpart in the
 * reference, whose entry points are always p*n/N_MULTIPROBE,
 * kernalGraph.h:214-231): d_seeds [nq x n_seeds] (device int32, 1 <= n_seeds
 * <= 32, -1 = no entry) replaces the N_MULTIPROBE seeds of each query; the
 * rest is song_search_device_ex.  An id >= n is skipped and reported through
 * the index's error word.
 */
song_status song_search_device_seeded(song_index* index, const song_search_opts* opts,
                                      const void* d_queries, int nq, int k, int ef_search,
                                      const int32_t* d_seeds, int n_seeds, int32_t* d_ids,
                                      float* d_dists, song_query_trace* d_traces, void* stream);

/* The extended search with host buffers (gpu_search-style, synchronous). */
song_status song_gpu_search_ex(song_index* index, const song_search_opts* opts,
                               const float* queries, int nq, int k, int n_multiquery,
                               int ef_search, int32_t* ids, float* dists,
                               song_query_trace* traces, song_timing* timing);

/*
 * Learned entry and stop models (no counterpart in the reference).  Two
 * MLPs of 24 inputs and two hidden layers of 64 with FP16 weights: the entry
 * model scores 24 hub nodes from the query's distances to them (its top
 * N_MULTIPROBE hubs become the entry points); the stop model reads running
 * queue statistics every ckpt_every expansions and stops the search once
 * P(top-k final) >= song_search_opts.stop_threshold.  Both are trained on
 * the GPU by this library's kernels from traces of the plain full-budget
 * search; without a confident stop the search runs to its natural end.
 */
typedef struct song_learn_params {
    int k;               /* top-k the stop model watches (the first min(k,32) are tracked) */
    int ef;              /* queue size of the full-budget plain search the traces come from */
    int ckpt_every;      /* expansions between stop checkpoints (default 8)                */
    int min_expansions;  /* no learned stop before this many expansions (default 8)        */
    int max_ckpt;        /* checkpoints kept per training query (default 256)              */
    int entry_steps;     /* Adam steps of the entry model (default 1500)                   */
    int stop_steps;      /* Adam steps of the stop model (default 3000)                    */
    int batch;           /* minibatch (default 4096)                                       */
    float lr;            /* Adam learning rate (default 2e-3)                              */
    unsigned seed;
    int entry_hubs;      /* hub set of the tensor-core entry stage (default 8192; dim <= 288).
                            0: the entry model scores 24 farthest-point hubs instead   */
} song_learn_params;

typedef struct song_learn_report {
    int n_hubs;
    long long stop_samples;
    double entry_loss_first, entry_loss_last;
    double stop_loss_first, stop_loss_last;
    double stop_pos_frac;  /* fraction of checkpoints whose top-k was already final */
} song_learn_report;

void song_learn_params_default(song_learn_params* p);

/*
 * Train both models for an L2 index from nq training queries (device FP32
 * [nq x dim]) and their exact nearest neighbours (device int32 [nq]).
 * Synchronous.  The models stay attached to the index.
 */
song_status song_index_learn(song_index* index, const song_learn_params* params,
                             const float* d_train_queries, int nq, const int32_t* d_train_nn1,
                             song_learn_report* report);

/*
 * Hub set of the learned entry stage (no counterpart in the reference).
 * song_index_set_entry_hubs attaches `count` hub node ids to an L2 index
 * (dim <= 288): their rows are laid out once as BF16 tensor-core tiles.
 * song_index_learn chooses and attaches a hub set itself.
 * song_index_entry_candidates runs the entry stage alone: for each query
 * (device FP32 [nq x dim]) the 24 nearest hubs by BF16 tensor-core distance,
 * nearest first (ties: earlier hub first), as node ids (-1 when the set has
 * fewer hubs) and squared distances (device [nq x 24] each); exact for
 * integer vectors in [0, 255] with dim <= 128.  Asynchronous on `stream`.
 */
song_status song_index_set_entry_hubs(song_index* index, const int32_t* hub_ids, int count);
song_status song_index_entry_candidates(song_index* index, const float* d_queries, int nq,
                                        int32_t* d_ids, float* d_dists, void* stream);

/* Flat FP32 copy of the attached models (*length floats; blob may be NULL to query). */
song_status song_index_get_model(const song_index* index, float* blob, int capacity, int* length);
/* Attach models saved by song_index_get_model. */
song_status song_index_set_model(song_index* index, const float* blob, int length);

/*
 * Gradient check entry point: mean loss and gradient of the packed MLP
 * parameters (FP32, layout W1 b1 W2 b2 W3 b3) over a batch, computed by the
 * training kernels.  loss_kind 0 = binary cross-entropy with logits (y in
 * [0,1], out = 1), 1 = softmax cross-entropy (y = class index).  Host buffers.
 */
song_status song_mlp_grad(int out, int loss_kind, const float* params, const float* x,
                          const float* y, const float* sample_weight, int batch, float* grad,
                          double* loss);

/*
 * Serving loop with continuous batching (no counterpart in the reference,
 * whose gpu_search is a synchronous batch call).  A persistent kernel keeps
 * one request per warp; requests published while others run are claimed as
 * soon as a warp (shared-memory slot) frees up, so their work overlaps on
 * the device.  Requests wait in a device-resident ring sized by hbm_budget;
 * results land in pinned host memory.  Each request carries its own k (<=
 * max_k) and queue size (clamped like gpu_search to min(max_ef, pq_size)).
 */
typedef struct song_server song_server;

#define SONG_REQ_LEARNED 1   /* request flag: learned entry/stop (full search if not confident) */

typedef struct song_server_config {
    int max_k;             /* largest k of a request (default 100)                          */
    int max_ef;            /* largest queue size of a request; sizes each slot (default 256) */
    int precision;         /* SONG_PREC_* used by every request                             */
    float stop_threshold;  /* learned stop threshold for requests flagged SONG_REQ_LEARNED  */
    int ring_slots;        /* requests queued or running at once (default 4096)             */
    long long hbm_budget;  /* device bytes the request ring may take (0 = no cap)           */
    int max_ctas;          /* persistent CTAs (0 = as many as fit)                          */
    int idle_exit_us;      /* idle warps exit after about this long (default 200000)        */
} song_server_config;

void song_server_config_default(song_server_config* c);
song_status song_server_create(song_index* index, const song_server_config* config,
                               song_server** out);
/* Queue n requests (host queries [n x dim], per-request k, ef, flags).  All
 * or nothing: SONG_ERR_BUDGET if the ring has no room.  *first_ticket gets
 * the ticket of the first request; the rest follow consecutively.  Poll a
 * ticket's results before ring_slots later requests reuse its slot. */
song_status song_server_submit(song_server* s, const float* queries, int n, const int* ks,
                               const int* efs, const int* flags, long long* first_ticket);
/* *done = 1 and ids/dists/trace (host, nullable) filled when the ticket finished. */
song_status song_server_poll(song_server* s, long long ticket, int32_t* ids, float* dists,
                             song_query_trace* trace, int* done);
/* Wait for a ticket at most timeout_us microseconds (host-side, bounded):
 * SONG_OK with ids/dists/trace filled, or SONG_ERR_TIMEOUT if it has not
 * finished by then (it may still finish; wait or poll again). */
song_status song_server_wait(song_server* s, long long ticket, long long timeout_us, int32_t* ids,
                             float* dists, song_query_trace* trace);

/* The persistent kernel's state: how often it was launched, whether it is
 * running, and why its warps left -- the server-wide idle time ran out
 * (idle_exit_us), the cap on empty polls was reached, or the stop word.
 * Every wait of the kernel is bounded; a later submit relaunches it. */
typedef struct song_server_stats {
    long long launches;
    long long idle_exits;      /* warps that left because nothing was claimed for idle_exit_us */
    long long poll_cap_exits;  /* warps that left at the cap on consecutive empty polls         */
    long long stop_exits;      /* warps that left at the stop word                              */
    int running;               /* 1 while the last launch has not finished                      */
} song_server_stats;
song_status song_server_get_stats(song_server* s, song_server_stats* out);
/* Native Poisson driver: nq requests arriving at rate_qps (exponential gaps,
 * seeded), submitted as they arrive, completions observed by polling.
 * latency_ms[i] = completion - arrival of request i.  ids_out (nullable)
 * [nq x max_k]; *wall_s = first arrival to last completion. */
song_status song_server_run_poisson(song_server* s, const float* queries, int nq, const int* ks,
                                    const int* efs, const int* flags, double rate_qps,
                                    unsigned seed, double* latency_ms, int32_t* ids_out,
                                    double* wall_s);
/* Stops the kernel (each warp exits at its next poll) and frees the server. */
song_status song_server_destroy(song_server* s);

/* Number of search-kernel launches issued by this library since load. */
int64_t song_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* SONG_B200_H */
