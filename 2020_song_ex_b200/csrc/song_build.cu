// song_build.cu -- NSW graph construction on the GPU (batched insertion).
//
// The reference builds the graph on one CPU thread, inserting u = 1..n-1 in
// order (kernalGraph.h:140-149, graph.h:190-199; 13 minutes for 1M x 128):
//   1. beam search from node 0 over the nodes inserted so far, beam
//      EF_CONSTRUCTION (kg_search_layer, kernalGraph.h:77-110);
//   2. keep the SEARCH_DEGREE nearest as u's row (kg_select_neighbors,
//      add_vertex, :112-120, :32-35);
//   3. add the reverse edge v -> u for each of them: first empty slot of v's
//      FIXED_DEGREE, else replace v's farthest neighbour when u is closer
//      (kg_add_reverse_edge, :123-137).
// Here the nodes are inserted in batches [s, s + B) with B = max(1, s/ratio):
// the whole batch searches the graph of nodes < s at once with the plain
// search kernel (one entry point = node 0, queue = EF_CONSTRUCTION), then the
// batch's reverse edges are grouped by target with a stable radix sort and
// applied by one warp per target in increasing u order with the reference's
// rule.  Nodes of one batch do not see each other, so the graph is an NSW
// graph of the same shape but not byte-identical to the reference's; it is
// deterministic for a given (data, params, ratio).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "song_kernels.cuh"

namespace song {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// Writes the batch's rows (the first min(sd, fd) found ids, the rest -1) and
// the reverse-edge list (key = target v, value = u; key 0xffffffff = none).
__global__ void scatter_forward(const int32_t* __restrict__ fwd, int sd, int fd, int bs,
                                int64_t s, int B, int32_t* __restrict__ adj,
                                uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)B * bs) return;
    const int b = (int)(t / bs), j = (int)(t % bs);
    const int m = sd < fd ? sd : fd;
    const int32_t v = j < sd ? fwd[(int64_t)b * sd + j] : -1;
    adj[(s + b) * bs + j] = (j < m) ? v : -1;
    if (j < sd) {
        const bool edge = j < m && v >= 0;
        keys[(int64_t)b * sd + j] = edge ? (uint32_t)v : 0xffffffffu;
        vals[(int64_t)b * sd + j] = (uint32_t)(s + b);
    }
}

// Distance between two stored rows, summed over the warp (all lanes get it).
template <int KIND>
__device__ __forceinline__ float warp_row_dist(const void* base, int ld, int dim, int64_t a,
                                               int64_t b, int lane) {
    float s = 0.0f;
    if constexpr (KIND == SONG_KIND_L2) {
        const float* ra = reinterpret_cast<const float*>(base) + a * ld;
        const float* rb = reinterpret_cast<const float*>(base) + b * ld;
        for (int i = lane; i < dim; i += 32) {
            const float t = ra[i] - rb[i];
            s = fmaf(t, t, s);
        }
    } else {
        const uint32_t* ra = reinterpret_cast<const uint32_t*>(base) + a * ld;
        const uint32_t* rb = reinterpret_cast<const uint32_t*>(base) + b * ld;
        int c = 0;
        for (int i = lane; i < dim; i += 32) c += __popc(ra[i] ^ rb[i]);
        s = (float)c;
    }
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) s += __shfl_xor_sync(FULL, s, w);
    return s;
}

// One warp per run of equal keys: applies that target's reverse edges in
// increasing u with kg_add_reverse_edge's rule (first empty slot among the
// first `fd`, else evict the first farthest if strictly closer).  fd <= 32.
template <int KIND>
__global__ void reverse_edges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                              int E, const void* __restrict__ base, int ld, int dim,
                              int32_t* __restrict__ adj, int bs, int fd) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= E) return;
    const uint32_t v = keys[i];
    if (v == 0xffffffffu) return;
    if (i > 0 && keys[i - 1] == v) return;  // not the head of its run
    int32_t* row = adj + (int64_t)v * bs;
    int nbr = lane < fd ? row[lane] : -1;
    float dl = 0.0f;  // distance v -> nbr of this lane (valid when have_dist)
    bool have_dist = false;
    for (int64_t t = i; t < E && keys[t] == v; ++t) {
        const int u = (int)vals[t];
        const unsigned empty = __ballot_sync(FULL, lane < fd && nbr < 0);
        if (empty) {
            const int j = __ffs(empty) - 1;
            if (lane == j) {
                nbr = u;
                row[j] = u;
            }
            have_dist = false;
            continue;
        }
        if (!have_dist) {
            for (int j = 0; j < fd; ++j) {
                const int nj = __shfl_sync(FULL, nbr, j);
                const float d = warp_row_dist<KIND>(base, ld, dim, v, nj, lane);
                if (lane == j) dl = d;
            }
            have_dist = true;
        }
        const float du = warp_row_dist<KIND>(base, ld, dim, v, u, lane);
        const unsigned bits = lane < fd ? __float_as_uint(dl) : 0u;
        const unsigned m = __reduce_max_sync(FULL, bits);
        const int fj = (int)__reduce_min_sync(FULL, (lane < fd && bits == m) ? lane : 32);
        if (du < __uint_as_float(m) && lane == fj) {
            nbr = u;
            dl = du;
            row[fj] = u;
        }
    }
}

}  // namespace

// Builds the adjacency [n x bs] in d_adj (device) over d_base rows
// ([n x ld], kind L2 or Hamming).  Stream-ordered; returns a CUDA error.
cudaError_t build_graph_device(int kind, const void* d_base, int64_t n, int dim, int ld,
                               const song_params& p, int ratio, int bf_words, int32_t* d_adj,
                               int num_sms, cudaStream_t st, BaseRange range) {
    if (ratio < 1) ratio = 32;
    const int bs = p.block_size, fd = p.fixed_degree, sd = p.search_degree;
    if (fd > 32 || fd > bs || sd < 1) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(d_adj, 0xff, (size_t)n * bs * sizeof(int32_t), st);
    if (e != cudaSuccess) return e;
    if (n < 2) return cudaSuccess;
    const int64_t maxB = std::max<int64_t>(1, (n - 1) / ratio + 1);
    const int64_t maxE = maxB * sd;
    int32_t* d_fwd = nullptr;
    uint32_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr;
    unsigned* ctr = nullptr;
    int* err = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    auto cleanup = [&]() {
        cudaFree(d_fwd); cudaFree(k0); cudaFree(k1); cudaFree(v0); cudaFree(v1);
        cudaFree(ctr); cudaFree(err); cudaFree(tmp);
    };
    if ((e = cudaMalloc(&d_fwd, maxB * sd * sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMalloc(&k0, maxE * 4)) != cudaSuccess || (e = cudaMalloc(&k1, maxE * 4)) != cudaSuccess ||
        (e = cudaMalloc(&v0, maxE * 4)) != cudaSuccess || (e = cudaMalloc(&v1, maxE * 4)) != cudaSuccess ||
        (e = cudaMalloc(&ctr, 4)) != cudaSuccess || (e = cudaMalloc(&err, 4)) != cudaSuccess) {
        cleanup();
        return e;
    }
    // Sort on the low key_bits bits: every valid key is < n < 2^key_bits and
    // the "no edge" key 0xffffffff reads as 2^key_bits - 1, so it sorts last.
    int key_bits = 1;
    while (key_bits < 32 && ((int64_t)1 << key_bits) <= n) ++key_bits;
    e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, k0, k1, v0, v1, (int)maxE, 0, key_bits, st);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, 4, st);
    int64_t s = 1;
    while (e == cudaSuccess && s < n) {
        const int B = (int)std::min<int64_t>(n - s, std::max<int64_t>(1, s / ratio));
        SearchArgs a{};
        a.base = d_base;
        a.adj = d_adj;
        a.queries = static_cast<const char*>(d_base) + (size_t)s * ld * 4;
        a.out = d_fwd;
        a.trace = nullptr;
        a.counter = ctr;
        a.err = err;
        a.n = s;
        a.dim = dim;
        a.ld = ld;
        a.qld = ld;
        a.qdim = dim;  // the generic (dim > 256) instance stages this many query floats
        a.block_size = bs;
        a.k = sd;
        a.nq = B;
        a.cap = std::max(1, p.ef_construction);
        a.bf_words = bf_words;
        a.bf_nhash = 4;
        a.n_multiprobe = 1;  // the reference build search starts from node 0 alone
        a.int_base = range.int_base;
        a.base_min = range.lo;
        a.base_max = range.hi;
        search_warp_smem(kind, dim, a.cap, bf_words, &a);
        e = cudaMemsetAsync(ctr, 0, 4, st);
        if (e == cudaSuccess) e = launch_search(kind, a, num_sms, st);
        if (e != cudaSuccess) break;
        const int64_t cells = (int64_t)B * bs;
        scatter_forward<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(d_fwd, sd, fd, bs, s, B,
                                                                          d_adj, k0, v0);
        const int E = B * sd;
        e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0, k1, v0, v1, E, 0, key_bits, st);
        if (e != cudaSuccess) break;
        const int64_t threads = (int64_t)E * 32;
        if (kind == SONG_KIND_L2)
            reverse_edges<SONG_KIND_L2><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
                k1, v1, E, d_base, ld, dim, d_adj, bs, fd);
        else
            reverse_edges<SONG_KIND_HAMMING><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
                k1, v1, E, d_base, ld, dim, d_adj, bs, fd);
        e = cudaGetLastError();
        s += B;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cleanup();
    return e;
}

}  // namespace song

namespace song {

namespace {

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct BuildScratch {
    unsigned* ctr;
    int* err;
    int32_t* fwd;
    uint32_t *k0, *k1, *v0, *v1;
    void* tmp;
    size_t tmp_bytes;
    size_t total;
};

// Carves the build temporaries out of one region starting at `base` (or, for
// base == nullptr, only computes the layout and the total size).
cudaError_t carve_build_scratch(int64_t n, const song_params& p, int ratio, char* base,
                                BuildScratch* s, int* key_bits) {
    const int64_t maxB = std::max<int64_t>(1, (n - 1) / ratio + 1);
    const int64_t maxE = maxB * p.search_degree;
    if (maxE > (int64_t)INT32_MAX / 2) return cudaErrorInvalidValue;  // far beyond any scratch
    int kb = 1;
    while (kb < 32 && ((int64_t)1 << kb) <= n) ++kb;
    *key_bits = kb;
    size_t tmp_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (uint32_t*)nullptr,
                                                    (uint32_t*)nullptr, (uint32_t*)nullptr,
                                                    (uint32_t*)nullptr, (int)maxE, 0, kb);
    if (e != cudaSuccess) return e;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += align256(bytes); return base ? base + o : nullptr; };
    s->ctr = reinterpret_cast<unsigned*>(take(8));
    s->err = s->ctr ? reinterpret_cast<int*>(s->ctr + 1) : nullptr;
    s->fwd = reinterpret_cast<int32_t*>(take((size_t)maxE * 4));
    s->k0 = reinterpret_cast<uint32_t*>(take((size_t)maxE * 4));
    s->k1 = reinterpret_cast<uint32_t*>(take((size_t)maxE * 4));
    s->v0 = reinterpret_cast<uint32_t*>(take((size_t)maxE * 4));
    s->v1 = reinterpret_cast<uint32_t*>(take((size_t)maxE * 4));
    s->tmp = take(tmp_bytes);
    s->tmp_bytes = tmp_bytes;
    s->total = off;
    return cudaSuccess;
}

}  // namespace

size_t build_scratch_bytes(int64_t n, const song_params& p, int ratio) {
    if (ratio < 1) ratio = 32;
    BuildScratch s{};
    int kb = 0;
    if (carve_build_scratch(n, p, ratio, nullptr, &s, &kb) != cudaSuccess) return (size_t)-1;
    return s.total;
}

// The batched build of build_graph_device with every temporary taken from
// the caller's device region `scratch` (build_scratch_bytes(n, p, ratio)
// bytes) instead of cudaMalloc.  Stream-ordered on `st`; does not wait.
cudaError_t build_graph_with_scratch(int kind, const void* d_base, int64_t n, int dim, int ld,
                                     const song_params& p, int ratio, int bf_words,
                                     int32_t* d_adj, int num_sms, cudaStream_t st, void* scratch,
                                     size_t scratch_bytes) {
    if (ratio < 1) ratio = 32;
    const int bs = p.block_size, fd = p.fixed_degree, sd = p.search_degree;
    if (fd > 32 || fd > bs || sd < 1) return cudaErrorInvalidValue;
    BuildScratch s{};
    int key_bits = 0;
    cudaError_t e = carve_build_scratch(n, p, ratio, static_cast<char*>(scratch), &s, &key_bits);
    if (e != cudaSuccess) return e;
    if (s.total > scratch_bytes) return cudaErrorInvalidValue;
    e = cudaMemsetAsync(d_adj, 0xff, (size_t)n * bs * sizeof(int32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.ctr, 0, 8, st);  // counter and error word
    int64_t u = 1;
    while (e == cudaSuccess && u < n) {
        const int B = (int)std::min<int64_t>(n - u, std::max<int64_t>(1, u / ratio));
        SearchArgs a{};
        a.base = d_base;
        a.adj = d_adj;
        a.queries = static_cast<const char*>(d_base) + (size_t)u * ld * 4;
        a.out = s.fwd;
        a.counter = s.ctr;
        a.err = s.err;
        a.n = u;
        a.dim = dim;
        a.ld = ld;
        a.qld = ld;
        a.qdim = dim;  // the generic (dim > 256) instance stages this many query floats
        a.block_size = bs;
        a.k = sd;
        a.nq = B;
        a.cap = std::max(1, p.ef_construction);
        a.bf_words = bf_words;
        a.bf_nhash = 4;
        a.n_multiprobe = 1;
        search_warp_smem(kind, dim, a.cap, bf_words, &a);
        e = cudaMemsetAsync(s.ctr, 0, 4, st);
        if (e == cudaSuccess) e = launch_search(kind, a, num_sms, st);
        if (e != cudaSuccess) break;
        const int64_t cells = (int64_t)B * bs;
        scatter_forward<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(s.fwd, sd, fd, bs, u, B,
                                                                          d_adj, s.k0, s.v0);
        const int E = B * sd;
        size_t tb = s.tmp_bytes;
        e = cub::DeviceRadixSort::SortPairs(s.tmp, tb, s.k0, s.k1, s.v0, s.v1, E, 0, key_bits, st);
        if (e != cudaSuccess) break;
        const int64_t threads = (int64_t)E * 32;
        if (kind == SONG_KIND_L2)
            reverse_edges<SONG_KIND_L2><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
                s.k1, s.v1, E, d_base, ld, dim, d_adj, bs, fd);
        else
            reverse_edges<SONG_KIND_HAMMING><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
                s.k1, s.v1, E, d_base, ld, dim, d_adj, bs, fd);
        e = cudaGetLastError();
        u += B;
    }
    return e;
}

}  // namespace song
