// C-ABI harness over the reference's CPU path, compiled against a configured
// copy of the reference headers by oracle/build_ref.py.
//
// TEST INFRASTRUCTURE ONLY: it exposes the reference's own code unchanged --
//   * build_graph     (graph.h:190-199): sequential NSW insertion;
//   * Graph::search   (graph.h:33-115) : the bench_cpu search path
//                                        (bench_cpu.cpp:444-451),
// so that tests can build graphs exactly as the reference does and so that
// bench.py can time the reference CPU search on the host cores.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "graph.h"

static_assert(sizeof(QueryTrace) == 12 * sizeof(int), "QueryTrace layout");

extern "C" {

// The compile-time constants of this variant (config.h:9-58), in this order:
// BLOCK_SIZE FIXED_DEGREE SEARCH_DEGREE EF_CONSTRUCTION pq_size TOPK
// N_MULTIPROBE N_MULTIQUERY hash_bits HASH_WORDS BF_WORDS BF_NHASH
void ref_config(int* out12) {
    const int v[12] = {BLOCK_SIZE, FIXED_DEGREE, SEARCH_DEGREE, EF_CONSTRUCTION, pq_size, TOPK,
                       N_MULTIPROBE, N_MULTIQUERY, hash_bits, HASH_WORDS, BF_WORDS, BF_NHASH};
    std::memcpy(out12, v, sizeof v);
}

// build_graph(data, n, dim) -> adj[n * BLOCK_SIZE]
int ref_cpu_build_graph(const float* data, int n, int dim, int32_t* adj_out) {
    if (n <= 0 || dim <= 0) return -1;
    Graph g = build_graph(std::vector<dist_t>(data, data + (size_t)n * dim), n, dim);
    std::memcpy(adj_out, g.adj.data(), (size_t)n * BLOCK_SIZE * sizeof(int32_t));
    return 0;
}

// A Graph whose adjacency is supplied by the caller (graph.h:11-20).
void* ref_cpu_graph_create(const float* data, int n, int dim, const int32_t* adj) {
    Graph* g = new Graph(n, dim, std::vector<dist_t>(data, data + (size_t)n * dim));
    std::memcpy(g->adj.data(), adj, (size_t)n * BLOCK_SIZE * sizeof(int32_t));
    return g;
}

void ref_cpu_graph_destroy(void* h) { delete static_cast<Graph*>(h); }

// Graph::search for nq queries on `nthreads` threads (Graph::search is const
// and touches only locals, graph.h:33-45).  ids_out[nq*k] receives each
// result exactly as Graph::search returns it (worst-first, graph.h:108-112),
// padded with -1; trace_out[nq*12] (nullable) receives the QueryTrace.
int ref_cpu_graph_search(void* h, const float* queries, int nq, int k, int ef, int nthreads,
                         int32_t* ids_out, int32_t* trace_out) {
    const Graph* g = static_cast<const Graph*>(h);
    if (nthreads < 1) nthreads = 1;
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= nq) break;
            QueryTrace tr;
            std::vector<idx_t> r = g->search(queries + (size_t)i * g->dim, k, ef, &tr);
            for (int j = 0; j < k; ++j) ids_out[(size_t)i * k + j] = j < (int)r.size() ? r[j] : -1;
            if (trace_out) std::memcpy(trace_out + (size_t)i * 12, &tr, sizeof tr);
        }
    };
    if (nthreads == 1) {
        work();
    } else {
        std::vector<std::thread> ts;
        for (int t = 0; t < nthreads; ++t) ts.emplace_back(work);
        for (auto& t : ts) t.join();
    }
    return 0;
}

}  // extern "C"
