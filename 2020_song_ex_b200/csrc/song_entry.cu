// song_entry.cu -- entry points of the learned search: the nearest hubs of
// every query, on the tensor cores.
//
// A hub set of H nodes (a few thousand) is laid out once, at learn time, as
// BF16 tiles of 128 hubs in the tensor cores' shared-memory operand layout.
// One CTA serves 128 queries: it converts their rows to BF16 into shared
// memory (operand A), then for each hub tile
//   * a bulk copy (cp.async.bulk, completion on an mbarrier) brings the tile
//     into shared memory (operand B), double buffered so that the next
//     tile's copy overlaps this tile's work;
//   * one thread issues K/16 tcgen05.mma (kind::f16, BF16 x BF16 -> FP32,
//     M = 128, N = 128) into one half of a 256-column TMEM accumulator and
//     commits them to that half's mbarrier, one tile ahead of the warps that
//     read the other half;
//   * every thread reads its query's row of the accumulator (tcgen05.ld,
//     lane = query) and keeps the kEntryK hubs of smallest |h|^2 - 2 q.h in
//     registers (|q|^2 is the same for every hub of a query).
// The output is, per query, those hubs' node ids nearest first (ties: lower
// hub index first) and their squared distances |q|^2 + |h|^2 - 2 q.h.  For
// integer vectors in [0, 255] with dim <= 128 every BF16 value, product sum
// and key stays an exact FP32 integer below 2^24, so the distances are
// exact; otherwise they carry BF16 rounding, which only matters for the
// choice of entry points.
//
// Shared-memory operand layout (no swizzle, K-major): 8 x 16-byte core
// matrices, one per 8 rows x 8 elements; core matrices adjacent along K are
// 128 bytes apart (the descriptor's leading byte offset), groups of 8 rows
// are (Kp / 8) * 128 bytes apart (its stride byte offset).
//
// Every wait is bounded: a barrier that does not complete within about two
// seconds sets the error word, the CTA stops issuing work, and it still
// frees its tensor memory before it returns.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>

#include "song_kernels.cuh"

namespace song {
extern std::atomic<int64_t> g_launches;

namespace {

constexpr int kM = 128;           // queries per CTA (MMA M)
constexpr int kN = 128;           // hubs per tile (MMA N), TMEM columns of the accumulator
constexpr int kK = kEntryK;       // nearest hubs kept per query
constexpr long long kWaitNs = 2000000000LL;

__device__ __forceinline__ int lane_of(int tid) { return tid & 31; }

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ long long now_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the mbarrier phase with parity `parity`; false after ~2 s.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = now_ns();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (now_ns() - t0 > kWaitNs) return false;
    }
}

// Shared-memory matrix descriptor (tcgen05): start, leading and stride byte
// offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kM >> 4) << 24);

// Byte offset of element (r, k) of a K-major operand tile with Kp columns.
__host__ __device__ __forceinline__ uint32_t tile_off(int r, int k, int kp) {
    return (uint32_t)((r >> 3) * (kp >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

struct EntryArgs {
    const float* queries;      // [nq x qld] FP32
    int qld, nq, dim, kp;      // kp = dim rounded up to 16
    const __nv_bfloat16* hub_tiles;  // [ntiles][kN x kp] in the operand layout
    const float* hub_norm;     // [ntiles * kN], +inf for padding
    const int32_t* hub_ids;    // [ntiles * kN], -1 for padding
    int ntiles;
    int tiles_per_split;       // blockIdx.y covers tiles [y * tps, (y + 1) * tps)
    int32_t* out_ids;          // [nq x kK]
    float* out_d;              // [nq x kK]
    float* part_key;           // splits > 1: [splits x nq x kK] keys |h|^2 - 2 q.h
    int32_t* part_idx;         // splits > 1: [splits x nq x kK] hub indices (-1 = none)
    int* tile_done;            // splits > 1: [query tiles] CTAs finished, zero at launch;
                               // the merging CTA returns its counter to zero
    int* err;                  // set to 2 when a bounded wait gives up
};

// KK: hubs kept per query (kK for the entry model's features; fewer when the
// search only takes the nearest few as entry points).  The first KK of the
// kK output entries are those of a kK-long list, the rest are -1: the same
// hubs in the same order, at a fraction of the insertion work.
template <int KK>
__global__ void __launch_bounds__(128, 1) entry_kernel(const EntryArgs a) {
    static_assert(KK >= 1 && KK <= kK, "KK in [1, kK]");
    extern __shared__ __align__(128) unsigned char smem[];
    // Each thread's 32 keys of the current accumulator chunk (XOR-swizzled by
    // thread, conflict-free), so that only the keys below its threshold are
    // visited by the insertion loop; and the current tile's hub norms.
    __shared__ float stage[kM * 32];
    __shared__ float hn_s[kN];
    __shared__ __align__(8) uint64_t bar_load[2];
    __shared__ __align__(8) uint64_t bar_mma[2];
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t a_bytes = (uint32_t)kM * a.kp * 2, b_bytes = (uint32_t)kN * a.kp * 2;
    unsigned char* As = smem;
    unsigned char* Bs[2] = {smem + a_bytes, smem + a_bytes + b_bytes};
    const uint32_t sbo = (uint32_t)(a.kp >> 3) * 128;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&tslot)), "r"(2 * kN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_load[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_load[1])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_mma[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar_mma[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tslot;

    const int t_begin = blockIdx.y * a.tiles_per_split;
    const int t_end = min(a.ntiles, t_begin + a.tiles_per_split);
    // first hub tiles in flight while the queries are converted
    auto issue_load = [&](int t, int buf) {
        const uint32_t bar = smem_addr(&bar_load[buf]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     :: "r"(bar), "r"(b_bytes) : "memory");
        const __nv_bfloat16* src = a.hub_tiles + (size_t)t * kN * a.kp;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
            :: "r"(smem_addr(Bs[buf])), "l"(src), "r"(b_bytes), "r"(bar) : "memory");
    };
    if (tid == 0) {
        if (t_begin < t_end) issue_load(t_begin, 0);
        if (t_begin + 1 < t_end) issue_load(t_begin + 1, 1);
    }

    // operand A: this thread's query as BF16, and its FP32 squared norm.  The
    // rows pass through `stage` 32 columns at a time: warp w loads its own 32
    // rows with one coalesced 128-byte read per row, then every thread converts
    // its row and sums its squares in increasing k (XOR-swizzled slots keep both
    // steps free of bank conflicts).
    const int q = blockIdx.x * kM + tid;
    float qn = 0.0f;
    {
        float* my = stage + tid * 32;
        const int sw = tid & 31;
        for (int k0 = 0; k0 < a.kp; k0 += 32) {
            const int k = k0 + lane_of(tid);
#pragma unroll 8
            for (int r = 0; r < 32; ++r) {
                const int row = warp * 32 + r;
                const int qr = blockIdx.x * kM + row;
                const float x = (qr < a.nq && k < a.dim) ? __ldg(a.queries + (size_t)qr * a.qld + k) : 0.0f;
                stage[row * 32 + (lane_of(tid) ^ r)] = x;
            }
            __syncwarp();
            for (int j0 = 0; j0 < 32 && k0 + j0 < a.kp; j0 += 8) {
                __align__(16) __nv_bfloat16 v[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const float x = my[(j0 + e) ^ sw];
                    qn = fmaf(x, x, qn);
                    v[e] = __float2bfloat16_rn(x);
                }
                *reinterpret_cast<uint4*>(As + tile_off(tid, k0 + j0, a.kp)) = *reinterpret_cast<const uint4*>(v);
            }
            __syncwarp();
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
    __syncthreads();

    float kd[KK];
    int ki[KK];
#pragma unroll
    for (int i = 0; i < KK; ++i) {
        kd[i] = INFINITY;
        ki[i] = -1;
    }
    // One tile ahead: the MMAs of tile u + 1 run into the other half of the
    // accumulator (TMEM columns kN * ((u + 1) % 2) ..) while the warps read
    // tile u; each half completes on its own mbarrier.  lw / mw: loads and MMA
    // groups waited for (uniform); li / mi: issued (thread 0).
    auto issue_mma = [&](int u) {
        const int buf = u & 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_addr(As), b0 = smem_addr(Bs[buf]);
        const uint32_t acc_t = tmem + (uint32_t)(buf * kN);
        for (int s = 0; s < a.kp / 16; ++s) {
            const uint64_t ad = umma_desc(a0 + (uint32_t)s * 256u, 128u, sbo);
            const uint64_t bd = umma_desc(b0 + (uint32_t)s * 256u, 128u, sbo);
            const uint32_t acc = s > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                :: "r"(acc_t), "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc) : "memory");
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
            :: "r"(smem_addr(&bar_mma[buf])) : "memory");
    };
    const int nt = t_end - t_begin;
    int lw = 0, mw = 0, li = nt < 2 ? nt : 2, mi = 0;
    bool ok = true;
    if (nt > 0) {  // a wait that gives up in any thread ends the work in every thread
        ok = __syncthreads_and(mbar_wait(smem_addr(&bar_load[0]), 0u));
        if (ok) {
            lw = 1;
            if (tid == 0) issue_mma(0);
            mi = 1;
        }
    }
    for (int u = 0; ok && u < nt; ++u) {
        const int t = t_begin + u;  // this CTA's u-th tile: buffers u % 2, their (u / 2)-th use
        if (u + 1 < nt) {
            ok = __syncthreads_and(mbar_wait(smem_addr(&bar_load[(u + 1) & 1]), (uint32_t)(((u + 1) >> 1) & 1)));
            if (!ok) break;
            lw = u + 2;
            if (tid == 0) issue_mma(u + 1);
            mi = u + 2;
        }
        hn_s[tid] = __ldg(a.hub_norm + (size_t)t * kN + tid);  // kN == blockDim.x
        ok = __syncthreads_and(mbar_wait(smem_addr(&bar_mma[u & 1]), (uint32_t)((u >> 1) & 1)));
        if (!ok) break;
        mw = u + 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // the MMAs of tile u have read its buffer: refill it with tile u + 2
        if (tid == 0 && u + 2 < nt) {
            issue_load(t + 2, u & 1);
            ++li;
        }
        const uint32_t row = tmem + (uint32_t)((u & 1) * kN) + ((uint32_t)(warp * 32) << 16);
        float* my = stage + tid * 32;
        const int sw = tid & 31;
        for (int c0 = 0; c0 < kN; c0 += 32) {
            uint32_t r[32];
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
                : "r"(row + (uint32_t)c0)
                : "memory");
            // keys below this thread's current 24th: a 32-bit mask, then the
            // insertion loop visits only those (the warp pays the largest count
            // among its threads, not one pass per key any thread wants)
            const float thr = kd[KK - 1];
            float dv[32];
            unsigned m = 0u;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                dv[j] = fmaf(-2.0f, __uint_as_float(r[j]), hn_s[c0 + j]);
                m |= (dv[j] < thr ? 1u : 0u) << j;
            }
            if (m) {
#pragma unroll
                for (int j = 0; j < 32; ++j) my[j ^ sw] = dv[j];
            }
            while (m) {
                const int j = __ffs(m) - 1;
                m &= m - 1u;
                const float d = my[j ^ sw];
                if (d < kd[KK - 1]) {  // sorted insertion; equal keys keep the earlier hub first
                    const int idx = t * kN + c0 + j;
#pragma unroll
                    for (int i = KK - 1; i > 0; --i) {
                        const bool shift = d < kd[i - 1];
                        const bool here = !shift && d < kd[i];
                        kd[i] = shift ? kd[i - 1] : (here ? d : kd[i]);
                        ki[i] = shift ? ki[i - 1] : (here ? idx : ki[i]);
                    }
                    if (d < kd[0]) {
                        kd[0] = d;
                        ki[0] = idx;
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();  // every warp has read this half before its next MMA
    }
    if (!ok) {
        // the copies and MMAs still in flight land before the CTA frees its
        // shared and tensor memory (each wait again bounded)
        if (tid == 0) {
            atomicExch(a.err, 2);
            for (int v = lw; v < li; ++v) mbar_wait(smem_addr(&bar_load[v & 1]), (uint32_t)((v >> 1) & 1));
            for (int v = mw; v < mi; ++v) mbar_wait(smem_addr(&bar_mma[v & 1]), (uint32_t)((v >> 1) & 1));
        }
        __syncthreads();
    }
    if (q < a.nq) {
        if (gridDim.y > 1) {  // partial list of this split, merged below by the tile's last CTA
            const size_t o = ((size_t)blockIdx.y * a.nq + q) * kK;
#pragma unroll
            for (int i = 0; i < KK; ++i) {
                const bool v = ok && ki[i] >= 0 && kd[i] < INFINITY;
                a.part_key[o + i] = v ? kd[i] : INFINITY;
                a.part_idx[o + i] = v ? ki[i] : -1;
            }
        } else {
#pragma unroll
            for (int i = 0; i < KK; ++i) {
                const bool v = ok && ki[i] >= 0 && kd[i] < INFINITY;
                a.out_ids[(size_t)q * kK + i] = v ? __ldg(a.hub_ids + ki[i]) : -1;
                a.out_d[(size_t)q * kK + i] = v ? fmaxf(qn + kd[i], 0.0f) : INFINITY;
            }
            for (int i = KK; i < kK; ++i) {
                a.out_ids[(size_t)q * kK + i] = -1;
                a.out_d[(size_t)q * kK + i] = INFINITY;
            }
        }
    }
    if (gridDim.y > 1) {
        // The last CTA of this query tile to finish merges the splits' lists: per
        // query the kK smallest (key, hub index), the order the unsplit kernel
        // keeps.  Each list is sorted that way (sorted insertion, hubs visited in
        // increasing index), so a merge of the list heads suffices.
        __shared__ int is_last;
        __threadfence();
        __syncthreads();
        if (tid == 0) is_last = atomicAdd(a.tile_done + blockIdx.x, 1) == (int)gridDim.y - 1;
        __syncthreads();
        if (is_last) {
            __threadfence();
            if (tid == 0) a.tile_done[blockIdx.x] = 0;  // every split has arrived: ready for the next launch
            if (q < a.nq) {
                // list heads in registers (every split's first entry loaded at once);
                // each step reloads only the winner's next entry
                const int S = (int)gridDim.y;
                float hk[kEntrySplits];
                int hx[kEntrySplits], pos[kEntrySplits];
#pragma unroll
                for (int sp = 0; sp < kEntrySplits; ++sp) {
                    pos[sp] = 0;
                    hx[sp] = -1;
                    hk[sp] = INFINITY;
                    if (sp < S) {
                        const size_t o = ((size_t)sp * a.nq + q) * kK;
                        hx[sp] = __ldcg(a.part_idx + o);
                        hk[sp] = __ldcg(a.part_key + o);
                    }
                }
                for (int i = 0; i < KK; ++i) {
                    float bk = INFINITY;
                    int bi = INT_MAX, bs = -1;
#pragma unroll
                    for (int sp = 0; sp < kEntrySplits; ++sp) {
                        if (hx[sp] >= 0 && (hk[sp] < bk || (hk[sp] == bk && hx[sp] < bi))) {
                            bk = hk[sp];
                            bi = hx[sp];
                            bs = sp;
                        }
                    }
                    a.out_ids[(size_t)q * kK + i] = bs >= 0 ? __ldg(a.hub_ids + bi) : -1;
                    a.out_d[(size_t)q * kK + i] = bs >= 0 ? fmaxf(qn + bk, 0.0f) : INFINITY;
#pragma unroll
                    for (int sp = 0; sp < kEntrySplits; ++sp) {
                        if (sp == bs) {
                            ++pos[sp];
                            hx[sp] = -1;
                            hk[sp] = INFINITY;
                            if (pos[sp] < KK) {
                                const size_t o = ((size_t)sp * a.nq + q) * kK + pos[sp];
                                hx[sp] = __ldcg(a.part_idx + o);
                                hk[sp] = __ldcg(a.part_key + o);
                            }
                        }
                    }
                }
                for (int i = KK; i < kK; ++i) {
                    a.out_ids[(size_t)q * kK + i] = -1;
                    a.out_d[(size_t)q * kK + i] = INFINITY;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(2 * kN)
                     : "memory");
    // Launched to overlap the previous search launch's tail: this launch ends
    // only after that one, so work queued after it on the stream also follows
    // the previous launch (a no-op for an ordinary launch).
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Hub tiles from FP32 base rows: hub i of the set is node ids[i] (-1 =
// padding: zero row, norm +inf).  One thread per 8-element chunk.
__global__ void make_hub_tiles(const float* __restrict__ base, int ld, int dim, int kp,
                               const int32_t* __restrict__ ids, int hpad,
                               __nv_bfloat16* __restrict__ tiles) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int chunks = kp / 8;
    if (c >= (int64_t)hpad * chunks) return;
    const int h = (int)(c / chunks), k0 = (int)(c % chunks) * 8;
    const int id = ids[h];
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int k = k0 + e;
        v[e] = __float2bfloat16_rn((id >= 0 && k < dim) ? base[(size_t)id * ld + k] : 0.0f);
    }
    const int t = h / kN, r = h % kN;
    unsigned char* dst = reinterpret_cast<unsigned char*>(tiles + (size_t)t * kN * kp) + tile_off(r, k0, kp);
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(v);
}

// Squared norms of the BF16 hub rows (the values the tensor cores multiply).
__global__ void hub_norms(const __nv_bfloat16* __restrict__ tiles, const int32_t* __restrict__ ids,
                          int hpad, int kp, float* __restrict__ norm) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= hpad) return;
    if (ids[h] < 0) {
        norm[h] = INFINITY;
        return;
    }
    const int t = h / kN, r = h % kN;
    const unsigned char* tile = reinterpret_cast<const unsigned char*>(tiles + (size_t)t * kN * kp);
    float s = 0.0f;
    for (int k = 0; k < kp; ++k) {
        const float x = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + tile_off(r, k, kp)));
        s = fmaf(x, x, s);
    }
    norm[h] = s;
}

}  // namespace

int entry_padded_dim(int dim) { return (dim + 15) / 16 * 16; }
int entry_tile_hubs() { return kN; }

cudaError_t build_entry_tables(const float* d_base, int ld, int dim, const int32_t* d_ids,
                               int hpad, __nv_bfloat16* d_tiles, float* d_norm, cudaStream_t st) {
    const int kp = entry_padded_dim(dim);
    const int64_t work = (int64_t)hpad * (kp / 8);
    make_hub_tiles<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(d_base, ld, dim, kp, d_ids, hpad,
                                                                    d_tiles);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    hub_norms<<<(hpad + 127) / 128, 128, 0, st>>>(d_tiles, d_ids, hpad, kp, d_norm);
    return cudaGetLastError();
}

size_t entry_smem_bytes(int dim) {
    const size_t kp = (size_t)entry_padded_dim(dim);
    return (size_t)kM * kp * 2 + 2 * (size_t)kN * kp * 2;
}

// Bytes of the per-tile arrival counters at the front of the split scratch.
static size_t tile_done_bytes(int nq) {
    const size_t qt = (size_t)(std::max(nq, 1) + kM - 1) / kM;
    return (qt * 4 + 255) / 256 * 256;
}

size_t entry_split_scratch_bytes(int nq, int num_sms) {
    const int qt = (nq + kM - 1) / kM;
    int splits = qt <= 1 ? kEntrySplits : (2 * num_sms) / qt;
    splits = std::max(1, std::min(kEntrySplits, splits));
    return tile_done_bytes(nq) + (size_t)splits * std::max(nq, 1) * kK * 8;
}

cudaError_t launch_entry(const float* d_queries, int qld, int nq, int dim,
                         const __nv_bfloat16* d_tiles, const float* d_norm, const int32_t* d_ids,
                         int hpad, int32_t* d_out_ids, float* d_out_d, int* d_err,
                         cudaStream_t st, void* split_scratch, size_t split_bytes, int num_sms,
                         bool overlap, int keep) {
    if (nq <= 0) return cudaSuccess;
    if (dim > kEntryMaxDim || hpad % kN != 0 || hpad <= 0) return cudaErrorInvalidValue;
    EntryArgs a;
    a.queries = d_queries;
    a.qld = qld;
    a.nq = nq;
    a.dim = dim;
    a.kp = entry_padded_dim(dim);
    a.hub_tiles = d_tiles;
    a.hub_norm = d_norm;
    a.hub_ids = d_ids;
    a.ntiles = hpad / kN;
    a.out_ids = d_out_ids;
    a.out_d = d_out_d;
    // The hub tiles are spread over `splits` CTAs per 128 queries (about two
    // CTAs per SM in all, up to kEntrySplits), as far as the caller's scratch
    // holds their partial lists and the per-tile arrival counters; the last CTA
    // of each query tile merges the lists.  The result does not depend on the
    // split.
    const int qt = (nq + kM - 1) / kM;
    int splits = qt <= 1 ? kEntrySplits : (2 * num_sms) / qt;
    splits = std::max(1, std::min(std::min(kEntrySplits, a.ntiles), splits));
    const size_t per_split = (size_t)nq * kK * 8, head = tile_done_bytes(nq);
    if (split_scratch == nullptr || split_bytes < head) splits = 1;
    else splits = (int)std::min<size_t>((size_t)splits, (split_bytes - head) / per_split);
    if (splits < 1) splits = 1;
    a.tiles_per_split = (a.ntiles + splits - 1) / splits;
    splits = (a.ntiles + a.tiles_per_split - 1) / a.tiles_per_split;
    a.tile_done = static_cast<int*>(split_scratch);
    a.part_key = reinterpret_cast<float*>(static_cast<char*>(split_scratch) + head);
    a.part_idx = reinterpret_cast<int32_t*>(static_cast<char*>(split_scratch) + head +
                                            (size_t)splits * nq * kK * 4);
    a.err = d_err;
    const size_t smem = entry_smem_bytes(dim);
    void (*kern)(const EntryArgs) = keep <= 4 ? entry_kernel<4> : (keep <= 8 ? entry_kernel<8> : entry_kernel<kK>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (splits > 1 && !overlap) {
        e = cudaMemsetAsync(a.tile_done, 0, head, st);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((nq + kM - 1) / kM), (unsigned)splits);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = overlap ? 1 : 0;
    e = cudaLaunchKernelEx(&cfg, kern, a);
    if (e != cudaSuccess) return e;
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError();
}

}  // namespace song
