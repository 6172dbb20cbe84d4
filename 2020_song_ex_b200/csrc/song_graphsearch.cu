// song_graphsearch.cu -- the reference's CPU search, Graph::search
// (graph.h:33-115), on the GPU with the same results bit for bit.
//
// Graph::search differs from the GPU kernel the reference benchmarks
// (kg_search_kernel): it keeps an exact visited set, an unbounded frontier
// ordered by (distance, id), a top-ef max-heap ordered by (distance, id),
// sums squared differences in dimension order (dist_t d = a - b; sum += d*d,
// each step rounded, no fused multiply-add in the reference's -O3 x86-64
// build), and returns the k best worst-first.  One warp runs one query:
//  * visited: a bitmap of n bits per resident warp in global memory, set
//    with atomicOr; duplicate ids within one adjacency row are resolved to
//    their first slot (__match_any_sync), as the sequential loop does;
//  * distances: lane j computes the j-th new neighbour's distance alone,
//    in dimension order with __fsub_rn / __fmul_rn / __fadd_rn;
//  * top-ef: slot arrays in shared memory; the (distance, id) maximum is
//    cached and recomputed by a warp scan after each change;
//  * frontier: slot arrays in shared memory, popped by a warp scan for the
//    (distance, id) minimum.  Once the top-ef holds exactly ef entries, an
//    entry with distance above the top-ef's maximum can never be expanded
//    (the maximum only decreases, and popping it ends the search), so such
//    entries are not stored and are dropped on overflow.  The frontier's
//    size and peak are still counted as the reference's unbounded heap's,
//    and when only dropped entries remain the search ends exactly as the
//    reference's does: one more expansion, then the early stop.  With the
//    top-ef full, stored entries are top-ef members or distance ties with
//    its maximum, so a capacity of 2 * ef + 64 holds them; more ties than
//    that set the error word instead.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>

#include "song_kernels.cuh"

namespace song {
extern std::atomic<int64_t> g_launches;

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct GsArgs {
    const float* base;        // [n x ld]
    const int32_t* adj;       // [n x bs]
    const float* queries;     // [nq x qld]
    int32_t* out;             // [nq x k], worst-first, -1 padded
    song_query_trace* trace;  // [nq] or nullptr
    unsigned* counter;        // work counter, 0 at launch
    int* err;                 // 3 = frontier overflow (ties), 1 = bad adjacency entry
    uint32_t* visited;        // [resident warps x vwords]
    int64_t n;
    int ld, dim, qld, bs, nq, k, ef, nmp, fcap, vwords;
    int warp_smem, fd_off, fi_off, td_off, ti_off;
};

// (d, id) < (e, jd) lexicographically; distances are compared as floats.
__device__ __forceinline__ bool less_pair(float d, int id, float e, int jd) {
    return d < e || (d == e && id < jd);
}

// Graph::search's l2 (distance.h:5-12): dimension order, each step rounded.
__device__ __forceinline__ float l2_seq(const float* __restrict__ q, const float* __restrict__ b,
                                        int dim) {
    float s = 0.0f;
    for (int i = 0; i < dim; ++i) {
        const float t = __fsub_rn(q[i], __ldg(b + i));
        s = __fadd_rn(s, __fmul_rn(t, t));
    }
    return s;
}

// Warp scan for the (distance, id) maximum (MAX) or minimum of sz slots;
// returns its slot (-1 if empty) and fills d / id.
template <bool MAX>
__device__ __forceinline__ int scan_extreme(const float* dv, const int* iv, int sz, float& d,
                                            int& id, int lane) {
    float bd = MAX ? -INFINITY : INFINITY;
    int bi = MAX ? INT_MIN : INT_MAX, bs = -1;
    for (int s = lane; s < sz; s += 32) {
        const float x = dv[s];
        const int y = iv[s];
        if (bs < 0 || (MAX ? less_pair(bd, bi, x, y) : less_pair(x, y, bd, bi))) {
            bd = x;
            bi = y;
            bs = s;
        }
    }
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) {
        const float od = __shfl_xor_sync(FULL, bd, w);
        const int oi = __shfl_xor_sync(FULL, bi, w);
        const int os = __shfl_xor_sync(FULL, bs, w);
        const bool take = os >= 0 && (bs < 0 || (MAX ? less_pair(bd, bi, od, oi) : less_pair(od, oi, bd, bi)));
        if (take) {
            bd = od;
            bi = oi;
            bs = os;
        }
    }
    d = bd;
    id = bi;
    return bs;
}

__global__ void __launch_bounds__(128) graph_search_kernel(const GsArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t slot_id = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    unsigned char* ws = smem + (size_t)wib * a.warp_smem;
    float* sq = reinterpret_cast<float*>(ws);
    float* fd = reinterpret_cast<float*>(ws + a.fd_off);
    int* fi = reinterpret_cast<int*>(ws + a.fi_off);
    float* td = reinterpret_cast<float*>(ws + a.td_off);
    int* ti = reinterpret_cast<int*>(ws + a.ti_off);
    uint32_t* vis = a.visited + slot_id * a.vwords;
    for (;;) {
        int qid = 0;
        if (lane == 0) qid = (int)atomicAdd(a.counter, 1u);
        qid = __shfl_sync(FULL, qid, 0);
        if (qid >= a.nq) break;
        const float* qg = a.queries + (int64_t)qid * a.qld;
        for (int i = lane; i < a.dim; i += 32) sq[i] = qg[i];
        for (int w = lane; w < a.vwords; w += 32) vis[w] = 0u;
        __threadfence();  // the cleared words are seen by this warp's atomics
        __syncwarp();
        song_query_trace tr = {};
        int ts = 0, fs = 0;
        long long fv = 0;  // size of the reference's unbounded frontier
        float tmd = -INFINITY;
        int tmi = INT_MIN, tms = -1;  // top-ef (distance, id) maximum and its slot
        bool overflow = false;

        // one candidate, in the reference's order (graph.h:47-62, :91-103)
        auto add = [&](float d, int v, bool seed) {
            fv += 1;
            tr.frontier_pushes += 1;
            tr.peak_frontier = (int)max((long long)tr.peak_frontier, fv);
            const bool prune = !seed && ts == a.ef && d > tmd;
            if (!prune) {
                if (fs == a.fcap && ts == a.ef) {  // drop entries that can never be expanded
                    int keep = 0;
                    for (int s0 = 0; s0 < fs; s0 += 32) {
                        const int s = s0 + lane;
                        const bool live = s < fs && !(fd[s] > tmd);
                        const float xd = s < fs ? fd[s] : 0.0f;
                        const int xi = s < fs ? fi[s] : 0;
                        const unsigned m = __ballot_sync(FULL, live);
                        __syncwarp();
                        if (live) {
                            const int p = keep + __popc(m & ((1u << lane) - 1u));
                            fd[p] = xd;
                            fi[p] = xi;
                        }
                        keep += __popc(m);
                        __syncwarp();
                    }
                    fs = keep;
                }
                if (fs < a.fcap) {
                    if (lane == 0) {
                        fd[fs] = d;
                        fi[fs] = v;
                    }
                    fs += 1;
                } else {
                    overflow = true;
                }
            }
            if (seed || ts < a.ef || d < tmd) {  // topk.push (+ pop of the maximum)
                if (lane == 0) {
                    if (!seed && ts >= a.ef) {
                        td[tms] = d;
                        ti[tms] = v;
                    } else {
                        td[ts] = d;
                        ti[ts] = v;
                    }
                }
                if (seed || ts < a.ef) ts += 1;
                __syncwarp();
                tms = scan_extreme<true>(td, ti, ts, tmd, tmi, lane);
                tr.result_updates += 1;
                tr.peak_results = max(tr.peak_results, ts);
            }
            __syncwarp();
        };

        // seeds p * n / N_MULTIPROBE (graph.h:47-62): duplicates keep the first p
        {
            int ep = -1;
            if (lane < a.nmp) ep = (int)((unsigned long long)lane * (unsigned long long)a.n /
                                         (unsigned long long)a.nmp);
            const unsigned same = __match_any_sync(FULL, ep);
            bool fresh = lane < a.nmp && (__ffs(same) - 1) == lane;
            if (fresh) {
                const uint32_t bit = 1u << (ep & 31);
                fresh = (atomicOr(vis + (ep >> 5), bit) & bit) == 0u;
            }
            const float d = fresh ? l2_seq(sq, a.base + (int64_t)ep * a.ld, a.dim) : 0.0f;
            unsigned N = __ballot_sync(FULL, fresh);
            while (N) {
                const int j = __ffs(N) - 1;
                N &= N - 1u;
                tr.seed_count += 1;
                tr.visited_nodes += 1;
                tr.distance_evals += 1;
                add(__shfl_sync(FULL, d, j), __shfl_sync(FULL, ep, j), true);
            }
        }
        for (;;) {
            if (fs == 0) {
                if (fv > 0) {  // only never-expandable entries remain: the reference pops one
                    tr.expanded_nodes += 1;
                    tr.early_stopped = 1;
                }
                break;
            }
            float cd;
            int cu;
            const int ms = scan_extreme<false>(fd, fi, fs, cd, cu, lane);
            __syncwarp();
            if (lane == 0) {  // remove: move the last slot into the hole
                fd[ms] = fd[fs - 1];
                fi[ms] = fi[fs - 1];
            }
            fs -= 1;
            fv -= 1;
            __syncwarp();
            tr.expanded_nodes += 1;
            if (ts == a.ef && cd > tmd) {
                tr.early_stopped = 1;
                break;
            }
            for (int c0 = 0; c0 < a.bs; c0 += 32) {  // graph.h:71-82, 32 slots at a time
                const int j = c0 + lane;
                int v = j < a.bs ? __ldg(a.adj + (int64_t)cu * a.bs + j) : -1;
                if (v >= a.n) {  // never read out of range
                    atomicExch(a.err, 1);
                    v = -1;
                }
                tr.neighbor_slots_scanned += min(32, a.bs - c0);
                const unsigned same = __match_any_sync(FULL, v);
                bool fresh = v >= 0 && (__ffs(same) - 1) == lane;
                if (fresh) {
                    const uint32_t bit = 1u << (v & 31);
                    fresh = (atomicOr(vis + (v >> 5), bit) & bit) == 0u;
                }
                unsigned N = __ballot_sync(FULL, fresh);
                const int c = __popc(N);
                tr.visited_nodes += c;
                tr.candidate_nodes += c;
                tr.distance_evals += c;
                const float d = fresh ? l2_seq(sq, a.base + (int64_t)v * a.ld, a.dim) : 0.0f;
                while (N) {  // graph.h:91-103, in slot order
                    const int jj = __ffs(N) - 1;
                    N &= N - 1u;
                    add(__shfl_sync(FULL, d, jj), __shfl_sync(FULL, v, jj), false);
                }
            }
        }
        if (overflow && lane == 0) atomicExch(a.err, 3);
        // graph.h:106-112: trim to k, then pop worst-first
        while (ts > a.k) {
            float md;
            int mi;
            const int s = scan_extreme<true>(td, ti, ts, md, mi, lane);
            __syncwarp();
            if (lane == 0) {
                td[s] = td[ts - 1];
                ti[s] = ti[ts - 1];
            }
            ts -= 1;
            __syncwarp();
        }
        int32_t* out = a.out + (int64_t)qid * a.k;
        const int cnt = ts;
        for (int i = 0; i < cnt; ++i) {
            float md;
            int mi;
            const int s = scan_extreme<true>(td, ti, ts, md, mi, lane);
            __syncwarp();
            if (lane == 0) {
                out[i] = mi;
                td[s] = td[ts - 1];
                ti[s] = ti[ts - 1];
            }
            ts -= 1;
            __syncwarp();
        }
        for (int i = cnt + lane; i < a.k; i += 32) out[i] = -1;
        tr.result_count = cnt;
        if (a.trace != nullptr && lane == 0) a.trace[qid] = tr;
        __syncwarp();
    }
}

int round_up16(int x) { return (x + 15) / 16 * 16; }

}  // namespace

int graph_search_frontier_cap(int ef) { return 2 * ef + 64; }

size_t graph_search_warp_smem(int dim, int ef) {
    const int fcap = graph_search_frontier_cap(ef);
    return (size_t)round_up16(dim * 4) + 2 * (size_t)round_up16(fcap * 4) +
           2 * (size_t)round_up16(ef * 4);
}

cudaError_t launch_graph_search(const float* d_base, int ld, int dim, const int32_t* d_adj, int bs,
                                int64_t n, const float* d_queries, int nq, int k, int ef, int nmp,
                                int32_t* d_out, song_query_trace* d_trace, unsigned* d_counter,
                                int* d_err, uint32_t* d_visited, int64_t visited_slots,
                                int num_sms, cudaStream_t st) {
    if (nq <= 0) return cudaSuccess;
    GsArgs a;
    a.base = d_base;
    a.adj = d_adj;
    a.queries = d_queries;
    a.out = d_out;
    a.trace = d_trace;
    a.counter = d_counter;
    a.err = d_err;
    a.visited = d_visited;
    a.n = n;
    a.ld = ld;
    a.dim = dim;
    a.qld = dim;
    a.bs = bs;
    a.nq = nq;
    a.k = k;
    a.ef = ef;
    a.nmp = nmp;
    a.fcap = graph_search_frontier_cap(ef);
    a.vwords = (int)((n + 31) / 32);
    a.fd_off = round_up16(dim * 4);
    a.fi_off = a.fd_off + round_up16(a.fcap * 4);
    a.td_off = a.fi_off + round_up16(a.fcap * 4);
    a.ti_off = a.td_off + round_up16(ef * 4);
    a.warp_smem = (int)graph_search_warp_smem(dim, ef);
    const int warps = 4;
    const size_t smem = (size_t)warps * a.warp_smem;
    cudaError_t e = cudaFuncSetAttribute(graph_search_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = (int)std::min<int64_t>(visited_slots / warps, ((int64_t)nq + warps - 1) / warps);
    if (grid < 1) return cudaErrorInvalidValue;
    (void)num_sms;
    graph_search_kernel<<<grid, warps * 32, smem, st>>>(a);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError();
}

int64_t graph_search_resident_warps(int dim, int ef, int num_sms, int dev) {
    const size_t smem = 4 * graph_search_warp_smem(dim, ef);
    int per_sm = 0;
    if (cudaFuncSetAttribute(graph_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, graph_search_kernel, 128, smem) !=
        cudaSuccess)
        return 0;
    (void)dev;
    return (int64_t)per_sm * num_sms * 4;
}

}  // namespace song
