// song_gt.cu -- exact k nearest neighbours on the tensor cores (the ground
// truth that recall is measured against).
//
// The reference computes ground truth by sequential brute force on the CPU
// (bench_cpu.cpp:158-175, a max-heap of the k smallest squared L2 distances
// per query) or in numpy (run_compare.py:199-213).  Here every distance is
// |q|^2 - 2 q.b + |b|^2 with the cross term from 3xBF16 split products on
// the tensor cores: x = hi + lo with hi = bf16(x) and lo = bf16(x - hi), and
// q.b ~= hi_q.hi_b + hi_q.lo_b + lo_q.hi_b accumulated in FP32 (lo.lo is
// below FP32 resolution).  A product whose lo operand is zero everywhere is
// skipped; for integer data in [0, 255] both lo parts are zero and, for
// dim <= 128, every sum stays an integer below 2^24, so distances are exact.
// The squared norms are FP64 sums rounded to FP32 and the distance is formed
// as (|q|^2 - 2 q.b) + |b|^2 in FP32.
//
// Layout in HBM: base and query rows are converted once into BF16 blocks of
// 128 rows x 32 dimensions (8 KB, the tensor cores' shared-memory operand
// layout: K-major, no swizzle, 8 x 16-byte core matrices; core matrices
// adjacent along K are 128 B apart, groups of 8 rows 512 B apart), hi and lo
// blocks side by side: [tile][chunk][hi, lo][128 x 32].
//
// One CTA (192 threads) owns 128 queries and a contiguous range of base
// tiles (a split); warps have fixed roles:
//   warp 4  copies, per (tile, chunk), the needed hi/lo blocks of the
//           queries and of the bases into a ring of shared-memory stages
//           (cp.async.bulk, completion counted on the stage's mbarrier);
//   warp 5  (one thread) issues tcgen05.mma kind::f16 (BF16 x BF16 -> FP32,
//           M = N = 128, K = 16) into one of two 128-column TMEM
//           accumulators, commits each stage back to the copier and each
//           finished tile to the epilogue;
//   warps 0-3 read the accumulator (tcgen05.ld, TMEM lane = query) while the
//           other accumulator is being filled, form the distances and keep
//           each query's k smallest (distance, id) keys in a max-heap in
//           shared memory.  A 32-column chunk is first reduced to the mask of
//           keys below the heap's top, so only those are inserted.
// Bases are visited in increasing id order inside a split, so a key that
// ties the heap's top distance never beats it (its id is larger): the
// comparison is on the distance alone.  Each split writes its k keys sorted;
// a merge kernel (one warp per query) takes the k smallest over the splits.
// The result -- ascending (distance, id), ties broken by the lower id -- does
// not depend on the split.
//
// Every wait is bounded (about two seconds): a role that gives up raises the
// CTA's abort flag and the error word, the others leave their loops, copies
// still in flight and MMAs still running are waited for (again bounded), and
// the tensor memory is freed before the CTA returns.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>

#include "song_b200.h"
#include "song_kernels.cuh"

namespace song {
extern std::atomic<int64_t> g_launches;
}

namespace {

constexpr int kM = 128;            // queries per CTA (MMA M, TMEM lanes)
constexpr int kN = 128;            // bases per tile (MMA N, columns of one accumulator)
constexpr int kKC = 32;            // dimensions per chunk
constexpr int kBlock = kM * kKC * 2;  // bytes of one 128 x 32 BF16 block
constexpr int kMaxStages = 8;
constexpr int kMaxK = 128;
constexpr int kMaxSplits = 32;
constexpr int kThreads = 192;
constexpr int kSmemLimit = 232448;  // opt-in shared memory per block on sm_100
constexpr long long kWaitNs = 2000000000LL;

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ long long now_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of parity `parity`; false after ~2 s, or as soon as
// another role has raised `abort` (when given).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const volatile int* abort) {
    const long long t0 = now_ns();
    for (;;) {
        if (mbar_test(bar, parity)) return true;
        if (abort != nullptr && *abort) return false;
        if (now_ns() - t0 > kWaitNs) return false;
    }
}

// Shared-memory matrix descriptor (tcgen05): start, leading and stride byte
// offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(tmem), "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc) : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(bar) : "memory");
}

// Byte offset of element (r, k) inside one 128 x 32 block.
__host__ __device__ __forceinline__ uint32_t blk_off(int r, int k) {
    return (uint32_t)((r >> 3) * 512 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Order-preserving map of an FP32 distance to an unsigned key (all finite
// values and +inf; -0 is folded into +0 by the caller).
__device__ __forceinline__ uint32_t ord32(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unord32(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// BF16 hi/lo blocks of `rows` FP32 rows (padding rows and dimensions are
// zero); `lo_any` gets 1 when some lo value is nonzero.  One thread per row
// and 8 dimensions.
__global__ void gt_tiles(const float* __restrict__ x, int64_t rows, int64_t ld, int dim, int nch,
                         int64_t rows_pad, unsigned char* __restrict__ tiles, int* __restrict__ lo_any) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int groups = nch * (kKC / 8);
    if (g >= rows_pad * groups) return;
    const int64_t r = g / groups;
    const int k0 = (int)(g % groups) * 8;
    __align__(16) __nv_bfloat16 hi[8];
    __align__(16) __nv_bfloat16 lo[8];
    bool nz = false;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int k = k0 + e;
        const float v = (r < rows && k < dim) ? x[r * ld + k] : 0.0f;
        hi[e] = __float2bfloat16_rn(v);
        lo[e] = __float2bfloat16_rn(v - __bfloat162float(hi[e]));
        nz |= __bfloat162float(lo[e]) != 0.0f;
    }
    const int64_t t = r / kM;
    const int c = k0 / kKC;
    unsigned char* blk = tiles + ((size_t)(t * nch + c) * 2) * kBlock;
    const uint32_t o = blk_off((int)(r % kM), k0 % kKC);
    *reinterpret_cast<uint4*>(blk + o) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(blk + kBlock + o) = *reinterpret_cast<const uint4*>(lo);
    if (nz) atomicOr(lo_any, 1);
}

// Squared norms: FP64 sums of the FP32 squares, rounded to FP32 (one warp
// per row); padding rows get +inf.
__global__ void gt_norms(const float* __restrict__ x, int64_t rows, int64_t ld, int dim,
                         int64_t rows_pad, float* __restrict__ norm) {
    const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows_pad) return;
    double s = 0.0;
    if (r < rows)
        for (int k = lane; k < dim; k += 32) {
            const double v = (double)x[r * ld + k];
            s += v * v;
        }
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) s += __shfl_xor_sync(0xffffffffu, s, w);
    if (lane == 0) norm[r] = r < rows ? (float)s : INFINITY;
}

struct GtArgs {
    const unsigned char* qtiles;  // [qtiles][nch][2][kBlock]
    const unsigned char* btiles;  // [btiles][nch][2][kBlock]
    const float* qnorm;           // [nq padded]
    const float* bnorm;           // [n padded]
    int nq, n, nch, ntiles, tiles_per_split, splits, k;
    int a_parts, b_parts;         // 1: hi only, 2: hi and lo
    int stages;
    unsigned long long* part;     // [nq][splits][k] keys, ascending
    int* err;                     // set to 2 when a bounded wait gives up
};

__global__ void __launch_bounds__(kThreads, 1) gt_kernel(const GtArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_full[kMaxStages];
    __shared__ __align__(8) uint64_t bar_empty[kMaxStages];
    __shared__ __align__(8) uint64_t bar_accf[2];
    __shared__ __align__(8) uint64_t bar_acce[2];
    __shared__ __align__(8) uint64_t bar_drain;
    __shared__ uint32_t tslot;
    __shared__ volatile int abort_flag;
    __shared__ int issued_s, consumed_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t stage_bytes = (uint32_t)(a.a_parts + a.b_parts) * kBlock;
    unsigned char* stages = smem;
    unsigned long long* heap =
        reinterpret_cast<unsigned long long*>(smem + (size_t)a.stages * stage_bytes);
    uint32_t* scratch = reinterpret_cast<uint32_t*>(heap + (size_t)kM * a.k);

    const int qt = blockIdx.x, y = blockIdx.y;
    const int t_begin = y * a.tiles_per_split;
    const int t_end = min(a.ntiles, t_begin + a.tiles_per_split);
    const int ntl = max(0, t_end - t_begin);
    const int loads = ntl * a.nch;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&tslot)), "r"(2 * kN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < a.stages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_empty[s])) : "memory");
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_accf[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(&bar_acce[b])), "r"(kM) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_drain)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
        issued_s = 0;
        consumed_s = 0;
    }
    if (tid < kM)
        for (int i = 0; i < a.k; ++i) heap[(size_t)i * kM + tid] = ~0ull;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tslot;

    if (warp == 4) {
        // ---- copier: (tile, chunk) i -> stage i % stages ----
        if (lane == 0) {
            int i = 0;
            for (; i < loads; ++i) {
                const int s = i % a.stages, u = i / a.stages;
                if (u > 0 && !mbar_wait(smem_addr(&bar_empty[s]), (uint32_t)((u - 1) & 1), &abort_flag)) {
                    abort_flag = 1;
                    break;
                }
                const int t = t_begin + i / a.nch, c = i % a.nch;
                const uint32_t bar = smem_addr(&bar_full[s]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                             :: "r"(bar), "r"(stage_bytes) : "memory");
                const uint32_t dst = smem_addr(stages + (size_t)s * stage_bytes);
                const unsigned char* qsrc = a.qtiles + ((size_t)(qt * a.nch + c) * 2) * kBlock;
                const unsigned char* bsrc = a.btiles + ((size_t)((int64_t)t * a.nch + c) * 2) * kBlock;
                for (int p = 0; p < a.a_parts + a.b_parts; ++p) {
                    const unsigned char* src = p < a.a_parts ? qsrc + (size_t)p * kBlock
                                                             : bsrc + (size_t)(p - a.a_parts) * kBlock;
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                        :: "r"(dst + (uint32_t)p * kBlock), "l"(src), "r"((uint32_t)kBlock), "r"(bar)
                        : "memory");
                }
            }
            issued_s = i;
        }
    } else if (warp == 5) {
        // ---- MMA issuer ----
        if (lane == 0) {
            int consumed = 0;
            bool ok = true;
            for (int j = 0; j < ntl && ok; ++j) {
                const int b = j & 1;
                if (j >= 2 && !mbar_wait(smem_addr(&bar_acce[b]), (uint32_t)(((j >> 1) - 1) & 1), &abort_flag)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_addr = tmem + (uint32_t)(b * kN);
                for (int c = 0; c < a.nch; ++c) {
                    const int i = j * a.nch + c, s = i % a.stages;
                    if (!mbar_wait(smem_addr(&bar_full[s]), (uint32_t)((i / a.stages) & 1), &abort_flag)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t s0 = smem_addr(stages + (size_t)s * stage_bytes);
                    const uint32_t ahi = s0, alo = s0 + kBlock;
                    const uint32_t bhi = s0 + (uint32_t)a.a_parts * kBlock, blo = bhi + kBlock;
#pragma unroll
                    for (int ks = 0; ks < kKC / 16; ++ks) {
                        const uint32_t off = (uint32_t)ks * 256u;
                        const uint64_t dah = umma_desc(ahi + off, 128u, 512u);
                        const uint64_t dbh = umma_desc(bhi + off, 128u, 512u);
                        mma_bf16(acc_addr, dah, dbh, (c > 0 || ks > 0) ? 1u : 0u);
                        if (a.b_parts == 2) mma_bf16(acc_addr, dah, umma_desc(blo + off, 128u, 512u), 1u);
                        if (a.a_parts == 2) mma_bf16(acc_addr, umma_desc(alo + off, 128u, 512u), dbh, 1u);
                    }
                    mma_commit(smem_addr(&bar_empty[s]));  // the stage is free once these MMAs ran
                    consumed = i + 1;
                }
                if (ok) mma_commit(smem_addr(&bar_accf[b]));
            }
            if (!ok) abort_flag = 1;
            consumed_s = consumed;
            // every MMA issued so far has completed before the memory goes away
            mma_commit(smem_addr(&bar_drain));
            if (!mbar_wait(smem_addr(&bar_drain), 0u, nullptr)) abort_flag = 1;
        }
    } else {
        // ---- epilogue: warps 0-3, thread = query row = TMEM lane ----
        const int q = qt * kM + tid;
        const float qn = q < a.nq ? a.qnorm[q] : 0.0f;
        unsigned long long top = ~0ull;
        uint32_t thr = 0xFFFFFFFFu;
        uint32_t* my = scratch + tid * 32;
        const int sw = lane;
        const uint32_t row = tmem + ((uint32_t)(warp * 32) << 16);
        for (int j = 0; j < ntl; ++j) {
            const int b = j & 1, t = t_begin + j;
            bool ok = mbar_wait(smem_addr(&bar_accf[b]), (uint32_t)((j >> 1) & 1), &abort_flag);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) {
                abort_flag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int64_t col0 = (int64_t)t * kN;
            for (int c0 = 0; c0 < kN; c0 += 32) {
                uint32_t r[32];
                __syncwarp();
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                    "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
                    "tcgen05.wait::ld.sync.aligned;"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                      "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                      "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                      "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                      "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                      "=r"(r[30]), "=r"(r[31])
                    : "r"(row + (uint32_t)(b * kN + c0))
                    : "memory");
                if (c0 + 32 == kN) {
                    // the accumulator has been read: the MMAs may overwrite it
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];"
                                 :: "r"(smem_addr(&bar_acce[b])) : "memory");
                }
                const int64_t cb = col0 + c0;
                const int64_t left = (int64_t)a.n - cb;
                const int nv = left <= 0 ? 0 : (left >= 32 ? 32 : (int)left);
                const float4* bn4 = reinterpret_cast<const float4*>(a.bnorm + cb);
                uint32_t o[32];
                unsigned m = 0u;
#pragma unroll
                for (int g = 0; g < 8; ++g) {
                    const float4 nb = __ldg(bn4 + g);
                    const float nbv[4] = {nb.x, nb.y, nb.z, nb.w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int jj = g * 4 + e;
                        const float cross2 = 2.0f * __uint_as_float(r[jj]);
                        const float d = __fadd_rn(__fadd_rn(__fsub_rn(qn, cross2), nbv[e]), 0.0f);
                        o[jj] = ord32(d);
                        m |= (o[jj] < thr && jj < nv ? 1u : 0u) << jj;
                    }
                }
                if (q >= a.nq) m = 0u;
                if (m) {
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) my[jj ^ sw] = o[jj];
                }
                while (m) {
                    const int jj = __ffs(m) - 1;
                    m &= m - 1u;
                    const uint32_t ov = my[jj ^ sw];
                    if (ov >= thr) continue;
                    // replace the heap's largest key and sift it down
                    const unsigned long long key = ((unsigned long long)ov << 32) | (uint32_t)(cb + jj);
                    int i = 0;
                    for (;;) {
                        const int l = 2 * i + 1;
                        if (l >= a.k) break;
                        int ch = l;
                        unsigned long long cv = heap[(size_t)l * kM + tid];
                        if (l + 1 < a.k) {
                            const unsigned long long rv = heap[(size_t)(l + 1) * kM + tid];
                            if (rv > cv) {
                                cv = rv;
                                ch = l + 1;
                            }
                        }
                        if (cv <= key) break;
                        heap[(size_t)i * kM + tid] = cv;
                        i = ch;
                    }
                    heap[(size_t)i * kM + tid] = key;
                    top = heap[tid];
                    thr = (uint32_t)(top >> 32);
                }
            }
        }
    }
    __syncthreads();

    // copies still in flight when a role gave up: wait for them (bounded)
    if (abort_flag && tid == kM) {
        for (int i = consumed_s; i < issued_s; ++i)
            mbar_wait(smem_addr(&bar_full[i % a.stages]), (uint32_t)((i / a.stages) & 1), nullptr);
    }
    const bool failed = abort_flag != 0;
    if (failed && tid == 0) atomicExch(a.err, 2);

    // each query's keys of this split, ascending (heap sort in place)
    if (!failed && tid < kM) {
        const int q = qt * kM + tid;
        if (q < a.nq) {
            for (int end = a.k - 1; end > 0; --end) {
                const unsigned long long mx = heap[tid];
                const unsigned long long key = heap[(size_t)end * kM + tid];
                heap[(size_t)end * kM + tid] = mx;
                int i = 0;
                for (;;) {
                    const int l = 2 * i + 1;
                    if (l >= end) break;
                    int ch = l;
                    unsigned long long cv = heap[(size_t)l * kM + tid];
                    if (l + 1 < end) {
                        const unsigned long long rv = heap[(size_t)(l + 1) * kM + tid];
                        if (rv > cv) {
                            cv = rv;
                            ch = l + 1;
                        }
                    }
                    if (cv <= key) break;
                    heap[(size_t)i * kM + tid] = cv;
                    i = ch;
                }
                heap[(size_t)i * kM + tid] = key;
            }
            unsigned long long* out = a.part + ((size_t)q * a.splits + y) * a.k;
            for (int i = 0; i < a.k; ++i) out[i] = heap[(size_t)i * kM + tid];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(2 * kN)
                     : "memory");
}

// The k smallest keys over a query's splits (one warp per query, lane = split).
__global__ void gt_merge(const unsigned long long* __restrict__ part, int nq, int splits, int k,
                         int32_t* __restrict__ ids, float* __restrict__ dists) {
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= nq) return;
    const unsigned long long* mine = part + ((size_t)q * splits + lane) * k;
    int p = 0;
    unsigned long long head = lane < splits ? mine[0] : ~0ull;
    for (int i = 0; i < k; ++i) {
        unsigned long long mn = head;
#pragma unroll
        for (int w = 16; w >= 1; w >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, mn, w);
            mn = o < mn ? o : mn;
        }
        if (lane == 0) {
            const bool v = mn != ~0ull;
            ids[(size_t)q * k + i] = v ? (int32_t)(uint32_t)(mn & 0xFFFFFFFFull) : -1;
            dists[(size_t)q * k + i] = v ? unord32((uint32_t)(mn >> 32)) : INFINITY;
        }
        if (mn != ~0ull && head == mn) {  // keys are unique: one lane advances
            ++p;
            head = p < k ? mine[p] : ~0ull;
        }
    }
}

// Splits per 128 queries: the count that minimises (waves of CTAs) x (tiles
// per split), the smaller one on ties.
int pick_splits(int qtiles, int ntiles, int num_sms) {
    int best = 1;
    int64_t best_cost = INT64_MAX;
    for (int s = 1; s <= std::min(kMaxSplits, ntiles); ++s) {
        const int64_t tps = (ntiles + s - 1) / s;
        const int used = (int)((ntiles + tps - 1) / tps);
        if (used != s) continue;
        const int64_t items = (int64_t)qtiles * s;
        const int64_t waves = (items + num_sms - 1) / num_sms;
        const int64_t cost = waves * tps;
        if (cost < best_cost) {
            best_cost = cost;
            best = s;
        }
    }
    return best;
}

}  // namespace

namespace song {

size_t gt_smem_bytes(int k, int a_parts, int b_parts, int stages) {
    return (size_t)stages * (a_parts + b_parts) * kBlock + (size_t)kM * k * 8 + (size_t)kM * 32 * 4;
}

int gt_stages(int k, int a_parts, int b_parts) {
    const size_t fixed = (size_t)kM * k * 8 + (size_t)kM * 32 * 4 + 1024;
    const size_t stage = (size_t)(a_parts + b_parts) * kBlock;
    if (fixed + 2 * stage > (size_t)kSmemLimit) return 0;
    return (int)std::min<size_t>(kMaxStages, ((size_t)kSmemLimit - fixed) / stage);
}

// Exact kNN of device rows.  Synchronous on `st` (the lo-part flags are read
// back to choose the products).  err: 0 ok, 2 a wait gave up.
cudaError_t exact_knn(const float* d_base, int64_t n, int64_t ldb, int dim, const float* d_q, int nq,
                      int64_t ldq, int k, int32_t* d_ids, float* d_dists, cudaStream_t st, int* err_out) {
    *err_out = 0;
    if (nq == 0) return cudaSuccess;
    int dev = 0, num_sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int nch = (dim + kKC - 1) / kKC;
    const int qtiles = (nq + kM - 1) / kM, ntiles = (int)((n + kN - 1) / kN);
    const int64_t qpad = (int64_t)qtiles * kM, npad = (int64_t)ntiles * kN;
    const int splits = pick_splits(qtiles, ntiles, num_sms);
    const size_t qt_bytes = (size_t)qtiles * nch * 2 * kBlock, bt_bytes = (size_t)ntiles * nch * 2 * kBlock;
    unsigned char *qtl = nullptr, *btl = nullptr;
    float *qn = nullptr, *bn = nullptr;
    int* flags = nullptr;  // [0] query lo, [1] base lo, [2] error word
    unsigned long long* part = nullptr;
    e = cudaMalloc(&qtl, qt_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&btl, bt_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&qn, (size_t)qpad * 4);
    if (e == cudaSuccess) e = cudaMalloc(&bn, (size_t)npad * 4);
    if (e == cudaSuccess) e = cudaMalloc(&flags, 3 * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&part, (size_t)nq * splits * k * 8);
    if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, 3 * sizeof(int), st);
    int h_flags[3] = {0, 0, 0};
    if (e == cudaSuccess) {
        const int groups = nch * (kKC / 8);
        gt_tiles<<<(unsigned)((qpad * groups + 255) / 256), 256, 0, st>>>(d_q, nq, ldq, dim, nch, qpad,
                                                                          qtl, flags + 0);
        gt_tiles<<<(unsigned)((npad * groups + 255) / 256), 256, 0, st>>>(d_base, n, ldb, dim, nch, npad,
                                                                          btl, flags + 1);
        gt_norms<<<(unsigned)((qpad + 7) / 8), 256, 0, st>>>(d_q, nq, ldq, dim, qpad, qn);
        gt_norms<<<(unsigned)((npad + 7) / 8), 256, 0, st>>>(d_base, n, ldb, dim, npad, bn);
        g_launches.fetch_add(4, std::memory_order_relaxed);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_flags, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) {
        GtArgs a;
        a.qtiles = qtl;
        a.btiles = btl;
        a.qnorm = qn;
        a.bnorm = bn;
        a.nq = nq;
        a.n = (int)n;
        a.nch = nch;
        a.ntiles = ntiles;
        a.tiles_per_split = (ntiles + splits - 1) / splits;
        a.splits = splits;
        a.k = k;
        a.a_parts = h_flags[0] ? 2 : 1;
        a.b_parts = h_flags[1] ? 2 : 1;
        a.stages = gt_stages(k, a.a_parts, a.b_parts);
        a.part = part;
        a.err = flags + 2;
        const size_t smem = gt_smem_bytes(k, a.a_parts, a.b_parts, a.stages);
        e = cudaFuncSetAttribute(gt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) {
            gt_kernel<<<dim3((unsigned)qtiles, (unsigned)splits), kThreads, smem, st>>>(a);
            gt_merge<<<(unsigned)((nq + 3) / 4), 128, 0, st>>>(part, nq, splits, k, d_ids, d_dists);
            g_launches.fetch_add(2, std::memory_order_relaxed);
            e = cudaGetLastError();
        }
    }
    int h_err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, flags + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    *err_out = h_err;
    cudaFree(qtl);
    cudaFree(btl);
    cudaFree(qn);
    cudaFree(bn);
    cudaFree(flags);
    cudaFree(part);
    return e;
}

}  // namespace song

extern "C" {

song_status song_exact_knn_device(const float* d_base, int64_t n, int64_t ldb, int dim,
                                  const float* d_queries, int nq, int64_t ldq, int k,
                                  int32_t* d_ids, float* d_dists, void* stream) {
    if (dim < 1) return song::set_error(SONG_ERR_INVALID_ARG, "dim must be >= 1");
    if (n < 1 || n > (int64_t)INT32_MAX - kN) return song::set_error(SONG_ERR_INVALID_ARG, "n out of range");
    if (nq < 0) return song::set_error(SONG_ERR_INVALID_ARG, "nq must be >= 0");
    if (k < 1 || k > kMaxK) return song::set_error(SONG_ERR_INVALID_ARG, "k must be in [1, 128]");
    if (ldb < dim || ldq < dim) return song::set_error(SONG_ERR_INVALID_ARG, "ldb and ldq must be >= dim");
    if (nq > 0 && (d_base == nullptr || d_queries == nullptr || d_ids == nullptr || d_dists == nullptr))
        return song::set_error(SONG_ERR_INVALID_ARG, "base, queries, ids or dists is NULL");
    if (song::gt_stages(k, 2, 2) < 2) return song::set_error(SONG_ERR_INVALID_ARG, "k too large");
    int err = 0;
    const cudaError_t e = song::exact_knn(d_base, n, ldb, dim, d_queries, nq, ldq, k, d_ids, d_dists,
                                          (cudaStream_t)stream, &err);
    if (e != cudaSuccess) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "exact kNN: %s", cudaGetErrorString(e));
        return song::set_error(SONG_ERR_CUDA, buf);
    }
    if (err != 0) return song::set_error(SONG_ERR_TIMEOUT, "exact kNN: a bounded wait gave up");
    return SONG_OK;
}

song_status song_exact_knn(const float* base, int64_t n, int dim, const float* queries, int nq, int k,
                           int32_t* ids, float* dists) {
    if (nq == 0) return SONG_OK;
    if (base == nullptr || queries == nullptr || ids == nullptr || dists == nullptr)
        return song::set_error(SONG_ERR_INVALID_ARG, "base, queries, ids or dists is NULL");
    if (dim < 1 || n < 1 || nq < 0) return song::set_error(SONG_ERR_INVALID_ARG, "bad shape");
    float *d_b = nullptr, *d_q = nullptr, *d_d = nullptr;
    int32_t* d_i = nullptr;
    cudaStream_t st = nullptr;
    const size_t bb = (size_t)n * dim * 4, qb = (size_t)nq * dim * 4, ob = (size_t)nq * k;
    cudaError_t e = cudaMalloc(&d_b, bb);
    if (e == cudaSuccess) e = cudaMalloc(&d_q, qb);
    if (e == cudaSuccess) e = cudaMalloc(&d_i, ob * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_d, ob * 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_b, base, bb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_q, queries, qb, cudaMemcpyHostToDevice, st);
    song_status s = SONG_OK;
    if (e == cudaSuccess) {
        s = song_exact_knn_device(d_b, n, dim, dim, d_q, nq, dim, k, d_i, d_d, st);
        if (s == SONG_OK) {
            e = cudaMemcpyAsync(ids, d_i, ob * 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dists, d_d, ob * 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        }
    }
    cudaFree(d_b);
    cudaFree(d_q);
    cudaFree(d_i);
    cudaFree(d_d);
    if (st) cudaStreamDestroy(st);
    if (s != SONG_OK) return s;
    if (e != cudaSuccess) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "exact kNN: %s", cudaGetErrorString(e));
        return song::set_error(SONG_ERR_CUDA, buf);
    }
    return SONG_OK;
}

}  // extern "C"
