// C-ABI harness over the reference's GPU path and builders, compiled by nvcc
// against a configured copy of the reference headers (oracle/build_ref.py).
//
// TEST INFRASTRUCTURE ONLY: it exposes the reference's own code unchanged --
//   * build_kernel_graph (kernalGraph.h:140-149) and build_hashed_graph
//     (hashKernelGraph.h:196-207): the graphs bench_gpu searches;
//   * BitHash (bitHash.h:17-56): the 1-bit random projection;
//   * gpu_search (kernalGraph.h:307-382, hashKernelGraph.h:360-435) with
//     kg_search_kernel / hkg_search_kernel: the bit-exact target, run on a
//     B200 to pin the CPU restatement in oracle/song_oracle.cpp.
// The builders run on any host; the searches need a GPU.
#include <cstdint>
#include <cstring>
#include <vector>

#include "kernalGraph.h"
#include "hashKernelGraph.h"

static_assert(sizeof(QueryTrace) == 12 * sizeof(int), "QueryTrace layout");

extern "C" {

int ref_build_kernel_graph(const float* data, int n, int dim, int32_t* adj_out) {
    if (n <= 0 || dim <= 0) return -1;
    KernelGraph g = build_kernel_graph(std::vector<dist_t>(data, data + (size_t)n * dim), n, dim);
    std::memcpy(adj_out, g.adj.data(), (size_t)n * BLOCK_SIZE * sizeof(int32_t));
    return 0;
}

// codes_out[n * HASH_WORDS]: BitHash(dim) (seed 42) projection of the data;
// adj_out[n * BLOCK_SIZE]: the Hamming NSW graph over those codes.
int ref_build_hashed_graph(const float* data, int n, int dim, int32_t* adj_out, uint32_t* codes_out) {
    if (n <= 0 || dim <= 0) return -1;
    HashKernelGraph g = build_hashed_graph(data, n, dim);
    std::memcpy(adj_out, g.adj.data(), (size_t)n * BLOCK_SIZE * sizeof(int32_t));
    std::memcpy(codes_out, g.hashed.data(), (size_t)n * HASH_WORDS * sizeof(uint32_t));
    return 0;
}

// BitHash(dim, seed).project_all(data, n) -> codes_out[n * HASH_WORDS];
// R_out (nullable) receives the [hash_bits x dim] projection matrix.
int ref_bithash_project(const float* data, int n, int dim, unsigned seed, uint32_t* codes_out, float* R_out) {
    BitHash bh(dim, seed);
    if (R_out) std::memcpy(R_out, bh.R.data(), bh.R.size() * sizeof(float));
    if (n > 0) {
        std::vector<uint32_t> c = bh.project_all(data, n);
        std::memcpy(codes_out, c.data(), c.size() * sizeof(uint32_t));
    }
    return 0;
}

static int fill_outputs(const std::vector<int>& ids, const GpuSearchTrace& tr, int nq, int k,
                        int32_t* ids_out, int32_t* trace_out, double* timing_out) {
    std::memcpy(ids_out, ids.data(), (size_t)nq * k * sizeof(int32_t));
    if (trace_out)
        for (int i = 0; i < nq; ++i) std::memcpy(trace_out + (size_t)i * 12, &tr.queries[i], sizeof(QueryTrace));
    if (timing_out) {
        timing_out[0] = tr.alloc_ms; timing_out[1] = tr.h2d_ms; timing_out[2] = tr.kernel_ms;
        timing_out[3] = tr.d2h_ms; timing_out[4] = tr.total_ms; timing_out[5] = tr.ef_search;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

// gpu_search(KernelGraph, ...) on a graph whose adjacency is supplied.
int ref_gpu_search_l2(const float* data, int n, int dim, const int32_t* adj, const float* queries,
                      int nq, int k, int n_multiquery, int ef, int32_t* ids_out, int32_t* trace_out,
                      double* timing_out) {
    KernelGraph g(n, dim, std::vector<dist_t>(data, data + (size_t)n * dim));
    std::memcpy(g.adj.data(), adj, (size_t)n * BLOCK_SIZE * sizeof(int32_t));
    g.upload_to_gpu();
    GpuSearchTrace tr;
    std::vector<int> ids = gpu_search(g, queries, nq, k, n_multiquery, ef, &tr);
    return fill_outputs(ids, tr, nq, k, ids_out, trace_out, timing_out);
}

// gpu_search(HashKernelGraph, ...) on supplied codes and adjacency.
int ref_gpu_search_hamming(const uint32_t* codes, int n, const int32_t* adj, const uint32_t* qcodes,
                           int nq, int k, int n_multiquery, int ef, int32_t* ids_out, int32_t* trace_out,
                           double* timing_out) {
    HashKernelGraph g(n, BitHash(1), std::vector<uint32_t>(codes, codes + (size_t)n * HASH_WORDS));
    std::memcpy(g.adj.data(), adj, (size_t)n * BLOCK_SIZE * sizeof(int32_t));
    g.upload_to_gpu();
    GpuSearchTrace tr;
    std::vector<int> ids = gpu_search(g, qcodes, nq, k, n_multiquery, ef, &tr);
    return fill_outputs(ids, tr, nq, k, ids_out, trace_out, timing_out);
}

}  // extern "C"
