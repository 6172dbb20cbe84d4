// song_noalloc.cu -- graph build that allocates no device memory.
//
// Why this exists: some callers cannot call cudaMalloc at the moment they
// build a graph.  A serving process whose device memory is handed out by
// its own pool (or reserved up front by another framework) has no spare
// allocation to give, and a cudaMalloc/cudaFree pair can synchronise the
// device and stall the streams that are answering queries.  For them,
// song_build_graph_noalloc takes the rows and the output adjacency as device
// pointers the caller already owns and runs every temporary of the batched
// build -- the search results of each batch, the reverse-edge keys and
// values, the radix-sort workspace and the work counter -- inside one fixed
// device array that belongs to this library.
//
// The array is a file-scope __device__ variable of kScratchBytes (16 MiB):
// every GPU that loads this library holds it until the process exits.  In
// host code its name stands for a host-side shadow, not a device address, so
// the device address is looked up once per device with cudaGetSymbolAddress
// (the first call on a device does that set-up; make that first call before
// any stream capture) and the kernels receive that pointer.
//
// All calls share the array and it keeps whatever the last call left there:
// the counter and error words are cleared on the stream before each build,
// everything else is written before it is read.  Two calls whose work
// overlaps on the GPU (different streams, or different host threads on one
// device) race on the array; serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "song_b200.h"
#include "song_kernels.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;

static __device__ __align__(256) unsigned char g_build_scratch[kScratchBytes];

constexpr int kMaxDevices = 256;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_build_scratch on the current device (looked up once).
song_status scratch_address(int dev, void** out) {
    if (dev < 0 || dev >= kMaxDevices)
        return song::set_error(SONG_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_build_scratch);
        if (e != cudaSuccess) {
            char buf[200];
            std::snprintf(buf, sizeof buf, "cudaGetSymbolAddress(build scratch): %s",
                          cudaGetErrorString(e));
            return song::set_error(SONG_ERR_CUDA, buf);
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return SONG_OK;
}

}  // namespace

extern "C" {

song_status song_build_graph_noalloc(int kind, const void* d_rows, int64_t n, int dim, int ld,
                                     const song_params* params, int batch_ratio,
                                     int build_bf_words, int32_t* d_adj, void* stream) {
    if (params == nullptr) return song::set_error(SONG_ERR_INVALID_ARG, "params is NULL");
    if (d_rows == nullptr || d_adj == nullptr)
        return song::set_error(SONG_ERR_INVALID_ARG, "d_rows or d_adj is NULL");
    if (kind != SONG_KIND_L2 && kind != SONG_KIND_HAMMING)
        return song::set_error(SONG_ERR_INVALID_ARG, "bad kind");
    if (n < 1 || n > (int64_t)INT32_MAX - 1)
        return song::set_error(SONG_ERR_INVALID_ARG, "n must be in [1, 2^31-1)");
    if (dim < 1 || ld < dim || ld % 4 != 0 || (kind == SONG_KIND_HAMMING && dim > 32))
        return song::set_error(SONG_ERR_INVALID_ARG,
                               "need 1 <= dim <= ld, ld a multiple of 4 (and dim <= 32 for codes)");
    if (kind == SONG_KIND_HAMMING && ld != song::search_row_stride(kind, dim))
        return song::set_error(SONG_ERR_INVALID_ARG,
                               "for codes, ld must be 4, 8, 16 or 32 words (the smallest >= dim)");
    if (((uintptr_t)d_rows & 15u) != 0)
        return song::set_error(SONG_ERR_INVALID_ARG, "d_rows must be 16-byte aligned");
    if (params->block_size < 1 || params->fixed_degree < 1 || params->fixed_degree > 32 ||
        params->fixed_degree > params->block_size || params->search_degree < 1 ||
        params->ef_construction < 1)
        return song::set_error(SONG_ERR_UNSUPPORTED,
                               "GPU build needs 1 <= fixed_degree <= min(32, block_size)");
    const int ratio = batch_ratio > 0 ? batch_ratio : 32;
    const int bfw = build_bf_words > 0 ? build_bf_words : 1024;
    const size_t need = song::build_scratch_bytes(n, *params, ratio);
    if (need == (size_t)-1) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "build of n=%lld (search_degree %d, batch_ratio %d) needs far more scratch "
                      "than the fixed %zu-byte array holds (raise batch_ratio or use "
                      "song_build_graph)",
                      (long long)n, params->search_degree, ratio, kScratchBytes);
        return song::set_error(SONG_ERR_BUDGET, buf);
    }
    if (need > kScratchBytes) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "build of n=%lld (search_degree %d, batch_ratio %d) needs %zu bytes of "
                      "scratch; the fixed scratch array holds %zu bytes (raise batch_ratio or "
                      "use song_build_graph)",
                      (long long)n, params->search_degree, ratio, need, kScratchBytes);
        return song::set_error(SONG_ERR_BUDGET, buf);
    }
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return song::set_error(SONG_ERR_CUDA, cudaGetErrorString(e));
    void* scratch = nullptr;
    if (song_status s = scratch_address(dev, &scratch)) return s;
    e = song::build_graph_with_scratch(kind, d_rows, n, dim, ld, *params, ratio, bfw, d_adj, sms,
                                       (cudaStream_t)stream, scratch, kScratchBytes);
    if (e != cudaSuccess) return song::set_error(SONG_ERR_CUDA, cudaGetErrorString(e));
    return SONG_OK;
}

}  // extern "C"
