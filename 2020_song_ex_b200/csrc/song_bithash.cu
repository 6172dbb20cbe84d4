// song_bithash.cu -- sign-random-projection codes (BitHash) on the GPU.
//
// The reference projects every base vector and every query on one CPU
// thread (BitHash::project / project_all, bitHash.h:32-56): bit b of word w
// is set when the FP32 dot product of hyperplane R[w*32+b] with the vector is
// > 0, the dot being summed in increasing d as `dot += R[row*dim+d] * x[d]`.
// The reference is built with plain -O3 for x86-64, so each step is an FP32
// multiply rounded to nearest, then an FP32 add rounded to nearest (no fused
// multiply-add).  This kernel performs exactly those two roundings per step
// (__fmul_rn, __fadd_rn: never contracted) in the same d order, so every
// code is bit-identical to the reference's, including the signs of dot
// products that land near zero.
//
// Layout of one CTA (128 threads): 64 vectors x 4 code words (128
// hyperplanes).  Warp w owns code word blockIdx.y*4 + w; lane l owns vectors
// l and l+32 and keeps all 32 dot products of its word for both, so the sign
// bits pack in registers with no cross-lane step.  d advances in chunks of
// 32: the chunk of the 64 vectors is staged in shared memory (padded rows:
// lane l reads its own vector without bank conflicts) and the chunk of the
// 128 hyperplanes is staged transposed (d-major, float4 groups swizzled by d)
// so that the 32 hyperplanes of a word are read as 8 broadcast float4 loads.
// Work is n * hash_bits * dim multiply-add pairs on the CUDA cores; R
// (hash_bits * dim * 4 bytes) stays in L2.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "song_b200.h"
#include "song_kernels.cuh"

namespace song {
extern std::atomic<int64_t> g_launches;
}

namespace {

constexpr int kTV = 64;     // vectors per CTA
constexpr int kWords = 4;   // code words per CTA (one per warp)
constexpr int kRows = kWords * 32;
constexpr int kDC = 32;     // d per staged chunk

// Position of hyperplane `row` at chunk offset d in the transposed R tile:
// float4 group (row / 4) is XOR-swizzled by d so that the transposing stores
// of one warp (32 consecutive d, one row) spread over 8 banks.
__device__ __forceinline__ int rs_pos(int d, int row) {
    return d * kRows + ((((row >> 2) ^ d) & 31) << 2) + (row & 3);
}

__global__ void __launch_bounds__(128) bithash_kernel(const float* __restrict__ R, int dim,
                                                      int words, const float* __restrict__ x,
                                                      int64_t n, int64_t ldx,
                                                      uint32_t* __restrict__ codes, int64_t ldc) {
    __shared__ __align__(16) float xs[kTV][kDC + 1];
    __shared__ __align__(16) float rs[kDC * kRows];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t v0 = (int64_t)blockIdx.x * kTV;
    const int w0 = blockIdx.y * kWords;
    const int row0 = w0 * 32;
    const int rows_here = min(kRows, words * 32 - row0);
    const int my_word = w0 + warp;

    float acc0[32], acc1[32];
#pragma unroll
    for (int b = 0; b < 32; ++b) {
        acc0[b] = 0.0f;
        acc1[b] = 0.0f;
    }

    for (int d0 = 0; d0 < dim; d0 += kDC) {
        const int cl = min(kDC, dim - d0);
        __syncthreads();  // the previous chunk is consumed
        // vectors: 64 x 32 floats, coalesced along d
#pragma unroll
        for (int i = 0; i < (kTV * kDC) / 128; ++i) {
            const int idx = i * 128 + t;
            const int v = idx >> 5, d = idx & 31;
            const int64_t gv = v0 + v;
            float val = 0.0f;
            if (gv < n && d < cl) val = __ldg(x + gv * ldx + d0 + d);
            xs[v][d] = val;
        }
        // hyperplanes: 128 x 32 floats, coalesced along d, stored transposed
#pragma unroll
        for (int i = 0; i < (kRows * kDC) / 128; ++i) {
            const int idx = i * 128 + t;
            const int row = idx >> 5, d = idx & 31;
            float val = 0.0f;
            if (row < rows_here && d < cl) val = __ldg(R + (int64_t)(row0 + row) * dim + d0 + d);
            rs[rs_pos(d, row)] = val;
        }
        __syncthreads();
        if (my_word < words) {
            for (int d = 0; d < cl; ++d) {
                const float xa = xs[lane][d];
                const float xb = xs[lane + 32][d];
                const float* rrow = rs + d * kRows;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int grp = warp * 8 + c;  // float4 group of hyperplanes 4*grp .. 4*grp+3
                    const float4 r = *reinterpret_cast<const float4*>(rrow + (((grp ^ d) & 31) << 2));
                    const float rv[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int b = 4 * c + e;
                        acc0[b] = __fadd_rn(acc0[b], __fmul_rn(rv[e], xa));
                        acc1[b] = __fadd_rn(acc1[b], __fmul_rn(rv[e], xb));
                    }
                }
            }
        }
    }
    if (my_word >= words) return;
    uint32_t c0 = 0, c1 = 0;
#pragma unroll
    for (int b = 0; b < 32; ++b) {
        c0 |= (acc0[b] > 0.0f ? 1u : 0u) << b;
        c1 |= (acc1[b] > 0.0f ? 1u : 0u) << b;
    }
    const int64_t va = v0 + lane, vb = v0 + lane + 32;
    if (va < n) codes[va * ldc + my_word] = c0;
    if (vb < n) codes[vb * ldc + my_word] = c1;
}

song_status fail(song_status s, const char* msg) { return song::set_error(s, msg); }

song_status cuda_fail(cudaError_t e, const char* what) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    return song::set_error(SONG_ERR_CUDA, buf);
}

song_status check_shape(int dim, int hash_bits, int64_t n) {
    if (dim < 1) return fail(SONG_ERR_INVALID_ARG, "dim must be >= 1");
    if (hash_bits < 32 || hash_bits % 32 != 0)
        return fail(SONG_ERR_INVALID_ARG, "hash_bits must be a positive multiple of 32");
    if (n < 0) return fail(SONG_ERR_INVALID_ARG, "n must be >= 0");
    return SONG_OK;
}

}  // namespace

namespace song {

cudaError_t launch_bithash(const float* d_R, int dim, int hash_bits, const float* d_x, int64_t n,
                           int64_t ldx, uint32_t* d_codes, int64_t ldc, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const int words = hash_bits / 32;
    const dim3 grid((unsigned)((n + kTV - 1) / kTV), (unsigned)((words + kWords - 1) / kWords));
    bithash_kernel<<<grid, 128, 0, st>>>(d_R, dim, words, d_x, n, ldx, d_codes, ldc);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError();
}

}  // namespace song

extern "C" {

song_status song_bithash_matrix(int dim, int hash_bits, unsigned seed, float* R) {
    if (song_status s = check_shape(dim, hash_bits, 0)) return s;
    if (R == nullptr) return fail(SONG_ERR_INVALID_ARG, "R is NULL");
    // The reference's generator and distribution (bitHash.h:23-27), called,
    // not restated: the same standard library gives the same matrix.
    std::mt19937 rng(seed);
    std::normal_distribution<float> gauss(0.0f, 1.0f);
    const size_t total = (size_t)hash_bits * (size_t)dim;
    for (size_t i = 0; i < total; ++i) R[i] = gauss(rng);
    return SONG_OK;
}

song_status song_bithash_project_device(const float* d_R, int dim, int hash_bits,
                                        const float* d_x, int64_t n, int64_t ldx,
                                        uint32_t* d_codes, int64_t ldc, void* stream) {
    if (song_status s = check_shape(dim, hash_bits, n)) return s;
    if (n == 0) return SONG_OK;
    if (d_R == nullptr || d_x == nullptr || d_codes == nullptr)
        return fail(SONG_ERR_INVALID_ARG, "R, x or codes is NULL");
    if (ldx < dim) return fail(SONG_ERR_INVALID_ARG, "ldx must be >= dim");
    if (ldc < hash_bits / 32) return fail(SONG_ERR_INVALID_ARG, "ldc must be >= hash_bits / 32");
    if ((n + kTV - 1) / kTV > (int64_t)INT32_MAX)
        return fail(SONG_ERR_INVALID_ARG, "n too large for one launch");
    cudaError_t e = song::launch_bithash(d_R, dim, hash_bits, d_x, n, ldx, d_codes, ldc,
                                         (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "bithash launch");
    return SONG_OK;
}

song_status song_bithash_project(const float* R, int dim, int hash_bits, const float* x,
                                 int64_t n, uint32_t* codes) {
    if (song_status s = check_shape(dim, hash_bits, n)) return s;
    if (n == 0) return SONG_OK;
    if (R == nullptr || x == nullptr || codes == nullptr)
        return fail(SONG_ERR_INVALID_ARG, "R, x or codes is NULL");
    const int words = hash_bits / 32;
    float* d_R = nullptr;
    float* d_x = nullptr;
    uint32_t* d_c = nullptr;
    cudaStream_t st = nullptr;
    const size_t rb = (size_t)hash_bits * dim * 4, xb = (size_t)n * dim * 4,
                 cb = (size_t)n * words * 4;
    cudaError_t e = cudaMalloc(&d_R, rb);
    if (e == cudaSuccess) e = cudaMalloc(&d_x, xb);
    if (e == cudaSuccess) e = cudaMalloc(&d_c, cb);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_R, R, rb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_x, x, xb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = song::launch_bithash(d_R, dim, hash_bits, d_x, n, dim, d_c, words, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(codes, d_c, cb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_R);
    cudaFree(d_x);
    cudaFree(d_c);
    if (st) cudaStreamDestroy(st);
    if (e == cudaErrorMemoryAllocation) return fail(SONG_ERR_OOM, "bithash: device allocation failed");
    if (e != cudaSuccess) return cuda_fail(e, "bithash");
    return SONG_OK;
}

}  // extern "C"
