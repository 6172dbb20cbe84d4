// song_b200.hpp -- the reference's C++ host interface over the song_b200 C ABI.
//
// Drop-in for code written against lrlorry/2020_song_ex's headers:
//   KernelGraph      kernalGraph.h:20-71   (data + adj, add_vertex, upload_to_gpu)
//   HashKernelGraph  hashKernelGraph.h:22-126 (codes + adj)
//   gpu_search       kernalGraph.h:307-382 and hashKernelGraph.h:360-435
//   build_kernel_graph kernalGraph.h:140-149 (here: the batched GPU build)
//   graph_search     graph.h:33-115 (Graph::search's results, on the GPU)
//   BitHash          bitHash.h:17-56 (projection on the GPU)
//   GpuSearchTrace / QueryTrace telemetry.h:5-41
// The compile-time constants of config.h become a song_params value (the
// reference defaults unless given).  Results, tie order and QueryTrace
// counters are those of the reference's gpu_search for the same graph.
// Errors throw std::runtime_error carrying song_last_error().
#ifndef SONG_B200_HPP
#define SONG_B200_HPP

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "song_b200.h"

namespace song_b200 {

using QueryTrace = song_query_trace;

struct BatchTiming {  // telemetry.h:20-28 (one entry per staged batch)
    int batch_index = 0;
    int batch_offset = 0;
    int batch_size = 0;
    double h2d_ms = 0.0, memset_ms = 0.0, kernel_ms = 0.0, d2h_ms = 0.0;
};

struct GpuSearchTrace {  // telemetry.h:30-41
    int ef_search = 0;
    int batch_limit = 0;
    double alloc_ms = 0.0, h2d_ms = 0.0, memset_ms = 0.0, kernel_ms = 0.0, d2h_ms = 0.0,
           total_ms = 0.0;
    std::vector<BatchTiming> batches;
    std::vector<QueryTrace> queries;
};

inline void check(song_status s) {
    if (s != SONG_OK) throw std::runtime_error(std::string("song_b200: ") + song_last_error());
}

inline song_params default_params() {
    song_params p;
    song_params_default(&p);
    return p;
}

// KernelGraph (kernalGraph.h:20-71): host copies plus a device index.
class KernelGraph {
public:
    int num_nodes;
    int dim;
    std::vector<float> data;
    std::vector<int> adj;
    song_params params;

    KernelGraph(int n, int d, std::vector<float> data_, const song_params& p = default_params())
        : num_nodes(n), dim(d), data(std::move(data_)),
          adj((size_t)n * p.block_size, -1), params(p) {}
    KernelGraph(const KernelGraph&) = delete;
    KernelGraph& operator=(const KernelGraph&) = delete;
    KernelGraph(KernelGraph&& o) noexcept
        : num_nodes(o.num_nodes), dim(o.dim), data(std::move(o.data)), adj(std::move(o.adj)),
          params(o.params), index_(o.index_) {
        o.index_ = nullptr;
    }
    ~KernelGraph() {
        if (index_) song_index_destroy(index_);
    }

    void add_vertex(int u, const std::vector<int>& neighbors) {  // kernalGraph.h:32-35
        const int m = std::min((int)neighbors.size(), params.fixed_degree);
        for (int j = 0; j < m; ++j) adj[(size_t)u * params.block_size + j] = neighbors[j];
    }

    void upload_to_gpu() {  // kernalGraph.h:38-43
        if (index_) {
            song_index_destroy(index_);
            index_ = nullptr;
        }
        check(song_index_create_l2(data.data(), num_nodes, dim, adj.data(), &params, &index_));
    }

    song_index* index() const { return index_; }

private:
    song_index* index_ = nullptr;
};

// HashKernelGraph (hashKernelGraph.h:22-126) over packed sign codes.
class HashKernelGraph {
public:
    int num_nodes;
    int hash_words;
    std::vector<uint32_t> hashed;
    std::vector<int> adj;
    song_params params;

    HashKernelGraph(int n, std::vector<uint32_t> codes, int words,
                    const song_params& p = default_params())
        : num_nodes(n), hash_words(words), hashed(std::move(codes)),
          adj((size_t)n * p.block_size, -1), params(p) {}
    HashKernelGraph(const HashKernelGraph&) = delete;
    HashKernelGraph& operator=(const HashKernelGraph&) = delete;
    ~HashKernelGraph() {
        if (index_) song_index_destroy(index_);
    }

    void upload_to_gpu() {
        if (index_) {
            song_index_destroy(index_);
            index_ = nullptr;
        }
        check(song_index_create_hamming(hashed.data(), num_nodes, hash_words, adj.data(), &params,
                                        &index_));
    }

    song_index* index() const { return index_; }

private:
    song_index* index_ = nullptr;
};

namespace detail {
inline void fill_trace(GpuSearchTrace* trace, const song_timing& t, int nq, int n_multiquery) {
    trace->ef_search = t.ef_search;
    trace->batch_limit = n_multiquery;
    trace->alloc_ms = t.alloc_ms;
    trace->h2d_ms = t.h2d_ms;
    trace->memset_ms = t.memset_ms;
    trace->kernel_ms = t.kernel_ms;
    trace->d2h_ms = t.d2h_ms;
    trace->total_ms = t.total_ms;
    trace->batches.assign(1, BatchTiming{0, 0, nq, t.h2d_ms, t.memset_ms, t.kernel_ms, t.d2h_ms});
}
}  // namespace detail

// gpu_search (kernalGraph.h:307-382): flat [nq*k] ids, best-first, -1 padded.
// ef_search < 0 selects pq_size, the reference's default argument.
inline std::vector<int> gpu_search(const KernelGraph& g, const float* queries, int nq, int k,
                                   int N_MULTIQUERY = 512, int ef_search = -1,
                                   GpuSearchTrace* trace = nullptr) {
    if (!g.index()) throw std::runtime_error("song_b200: graph not uploaded");
    std::vector<int> ids((size_t)nq * k);
    song_timing t{};
    if (trace) trace->queries.resize(nq);
    check(song_gpu_search(g.index(), queries, nq, k, N_MULTIQUERY,
                          ef_search < 0 ? g.params.pq_size : ef_search, ids.data(),
                          trace ? trace->queries.data() : nullptr, &t));
    if (trace) detail::fill_trace(trace, t, nq, N_MULTIQUERY);
    return ids;
}

// gpu_search overload on u32 query codes (hashKernelGraph.h:360-435).
inline std::vector<int> gpu_search(const HashKernelGraph& g, const uint32_t* queries, int nq,
                                   int k, int N_MULTIQUERY = 512, int ef_search = -1,
                                   GpuSearchTrace* trace = nullptr) {
    if (!g.index()) throw std::runtime_error("song_b200: graph not uploaded");
    std::vector<int> ids((size_t)nq * k);
    song_timing t{};
    if (trace) trace->queries.resize(nq);
    check(song_gpu_search_hamming(g.index(), queries, nq, k, N_MULTIQUERY,
                                  ef_search < 0 ? g.params.pq_size : ef_search, ids.data(),
                                  trace ? trace->queries.data() : nullptr, &t));
    if (trace) detail::fill_trace(trace, t, nq, N_MULTIQUERY);
    return ids;
}

// Graph::search (graph.h:33-115) for nq queries, computed on the GPU with the
// reference's CPU results: each entry is what Graph::search returns for that
// query (the best min(k, found) ids, worst first).  ef_search <= 0 selects k.
inline std::vector<std::vector<int>> graph_search(const KernelGraph& g, const float* queries,
                                                  int nq, int k, int ef_search = 0,
                                                  std::vector<QueryTrace>* traces = nullptr) {
    if (!g.index()) throw std::runtime_error("song_b200: graph not uploaded");
    std::vector<int32_t> ids((size_t)nq * k);
    std::vector<QueryTrace> tr((size_t)nq);
    check(song_graph_search(g.index(), queries, nq, k, ef_search, ids.data(), tr.data()));
    std::vector<std::vector<int>> out((size_t)nq);
    for (int i = 0; i < nq; ++i)
        out[(size_t)i].assign(ids.begin() + (size_t)i * k, ids.begin() + (size_t)i * k + tr[(size_t)i].result_count);
    if (traces) *traces = std::move(tr);
    return out;
}

// BitHash (bitHash.h:17-56): the projection matrix drawn as the reference's
// constructor draws it; project / project_all run on the GPU and return the
// reference's codes bit for bit.  hash_bits is config.h's hash_bits.
struct BitHash {
    int dim;
    int hash_bits;
    std::vector<float> R;  // [hash_bits x dim]

    explicit BitHash(int dim_, unsigned seed = 42, int hash_bits_ = 256)
        : dim(dim_), hash_bits(hash_bits_), R((size_t)hash_bits_ * dim_) {
        check(song_bithash_matrix(dim, hash_bits, seed, R.data()));
    }
    void project(const float* vec, uint32_t* out) const {
        check(song_bithash_project(R.data(), dim, hash_bits, vec, 1, out));
    }
    std::vector<uint32_t> project_all(const float* data, int n) const {
        std::vector<uint32_t> out((size_t)n * (hash_bits / 32));
        check(song_bithash_project(R.data(), dim, hash_bits, data, n, out.data()));
        return out;
    }
};

// build_kernel_graph (kernalGraph.h:140-149), built on the GPU in batches.
inline KernelGraph build_kernel_graph(std::vector<float> data, int n, int dim,
                                      const song_params& p = default_params(),
                                      int batch_ratio = 32) {
    KernelGraph g(n, dim, std::move(data), p);
    check(song_build_graph(SONG_KIND_L2, g.data.data(), n, dim, &g.params, batch_ratio, 0,
                           g.adj.data()));
    return g;
}

}  // namespace song_b200

#endif  // SONG_B200_HPP
