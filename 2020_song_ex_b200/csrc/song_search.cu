// song_search.cu -- sm_100a kernels of the plain SONG graph search.
//
// One warp owns one query at a time; W warps share a CTA and a persistent
// grid pulls queries from a device work counter, so every SM keeps many
// independent traversals (and their neighbour gathers) in flight.  The
// reference runs one query per single-warp block with lane 0 doing all queue
// and Bloom work serially (kernalGraph.h:184-299).
//
// Results are bit-exact with the reference, including tie order and the
// QueryTrace counters, because the per-query state is the reference's own
// state and every step keeps its order:
//  * Candidates / Results (gpuHeap.h:8-108) stay unsorted slot arrays in
//    shared memory with the same slot moves.  Their O(cap) scans become
//    warp scans + redux.sync argmin/argmax that break ties by the lowest
//    slot, i.e. the reference's "first index" rule (strict < / strict >).
//  * A row of up to 32 neighbours is handled at once, lane j = slot j, but
//    the Bloom test of neighbour j sees the bits of neighbours < j exactly
//    as bf_test/bf_set in j order do (bloomFilter.h:34-48): see bloom_chunk.
//  * Distances follow warp_l2 (kernalGraph.h:157-170): lane l sums
//    (q_i - b_i)^2 over i = l (mod 32) with FMA, then a butterfly
//    transpose-reduce over 32 rows whose association is exactly the
//    reference's shfl_down tree (16,8,4,2,1), so FP32 sums match for any
//    data; lane j ends holding the distance of row j.
//  * Pushes are applied in lane (= j) order; a push into a full queue only
//    evicts when strictly closer than the current first maximum, and the
//    maximum never grows while a queue is full, so lanes that lose against
//    the running maximum drop out with one ballot.
#include <algorithm>
#include <atomic>
#include <climits>

#include "song_kernels.cuh"

namespace song {

std::atomic<int64_t> g_launches{0};

namespace {

constexpr unsigned FULL = 0xffffffffu;

// The mixing constants of bloomFilter.h:14-19: two per hash function.
__constant__ uint64_t kBloomMix[8] = {
    0x4bcb391f924ed183ULL, 0xa0ab69ccd854fc0aULL, 0x91086b9cecf5e3b7ULL, 0xc68e01641bead407ULL,
    0x3a7b976128a30449ULL, 0x6d122efabfc4d99fULL, 0xe6700ef8715030e2ULL, 0x80dd0c3bffcfb45bULL,
};

// A bounded slot queue in shared memory; the scalar fields are warp-uniform.
struct Queue {
    float* d;
    int* id;
    int sz;
    int cap;
    float maxv;   // first maximal slot (valid when max_ok)
    int maxi;
    bool max_ok;
};

struct BloomCfg {
    uint64_t nbits;     // BF_WORDS * 64
    uint32_t words;     // BF_WORDS
    uint32_t wmask;     // BF_WORDS - 1 when a power of two
    int shift;          // log2(BF_WORDS), or -1
    int nhash;          // BF_NHASH
};

__device__ __forceinline__ unsigned fbits(float x) { return __float_as_uint(x); }

// First slot holding the minimum over [0, sz).  Distances are non-negative,
// so their bit patterns order like the floats.
__device__ __forceinline__ void q_argmin(const Queue& q, int lane, float& v, int& idx) {
    unsigned best = 0xffffffffu, bi = 0xffffffffu;
    for (int s = lane; s < q.sz; s += 32) {
        const unsigned b = fbits(q.d[s]);
        if (b < best) { best = b; bi = (unsigned)s; }
    }
    const unsigned m = __reduce_min_sync(FULL, best);
    idx = (int)__reduce_min_sync(FULL, best == m ? bi : 0xffffffffu);
    v = __uint_as_float(m);
}

// First slot holding the maximum over [0, sz) (gpuHeap.h:29, :73, :83, :93).
__device__ __forceinline__ void q_argmax(Queue& q, int lane) {
    unsigned best = 0u, bi = 0xffffffffu;
    for (int s = lane; s < q.sz; s += 32) {
        const unsigned b = fbits(q.d[s]);
        if (bi == 0xffffffffu || b > best) { best = b; bi = (unsigned)s; }
    }
    const unsigned m = __reduce_max_sync(FULL, best);
    q.maxi = (int)__reduce_min_sync(FULL, (bi != 0xffffffffu && best == m) ? bi : 0xffffffffu);
    q.maxv = __uint_as_float(m);
    q.max_ok = true;
}

// Push (d, nb) of every lane in N, in lane order, with the semantics of
// Candidates::push / Results::try_push (gpuHeap.h:23-36, :68-77).
// Returns how many pushes were accepted.
__device__ __forceinline__ int q_push(Queue& q, unsigned N, float d, int nb, int lane) {
    if (N == 0u) return 0;
    const bool mine = (N >> lane) & 1u;
    const int rank = __popc(N & ((1u << lane) - 1u));
    const int nm = __popc(N);
    const int room = q.cap - q.sz;
    if (mine && rank < room) {
        q.d[q.sz + rank] = d;
        q.id[q.sz + rank] = nb;
    }
    int accepted = nm < room ? nm : room;
    if (accepted > 0) {
        q.sz += accepted;
        q.max_ok = false;
    }
    if (nm > room) {
        __syncwarp();
        if (!q.max_ok) q_argmax(q, lane);
        unsigned rest = __ballot_sync(FULL, mine && rank >= room && d < q.maxv);
        while (rest) {
            const int j = __ffs(rest) - 1;
            const float dj = __shfl_sync(FULL, d, j);
            const int nj = __shfl_sync(FULL, nb, j);
            if (lane == 0) {
                q.d[q.maxi] = dj;
                q.id[q.maxi] = nj;
            }
            __syncwarp();
            ++accepted;
            q_argmax(q, lane);
            rest &= ~(1u << j);
            rest &= __ballot_sync(FULL, d < q.maxv);
        }
    }
    __syncwarp();
    return accepted;
}

// bf_hash (bloomFilter.h:23-30) for a node id x >= 0.  The first x ^= x>>33
// of the reference is the identity for x < 2^33 and is left out.
__device__ __forceinline__ uint32_t bf_pos(int h, uint32_t x, const BloomCfg& bc) {
    uint64_t y = (uint64_t)x * kBloomMix[2 * h];
    y ^= y >> 33;
    y *= kBloomMix[2 * h + 1];
    y ^= y >> 33;
    return bc.shift >= 0 ? (uint32_t)(y & (bc.nbits - 1)) : (uint32_t)(y % bc.nbits);
}

// Bloom test-and-set of one chunk of up to 32 ids (lane j = j-th id of the
// row, nb < 0 = empty slot), equivalent to the reference's
//   for j: if (!bf_test(nb_j)) { bf_set(nb_j); new_j = true; }
// Returns the mask of lanes whose id is new.
//
// Reference order matters only through bits set by earlier ids of the same
// row: id j is skipped iff each of its positions is in B0 (the filter before
// the row) or is a position of an earlier valid id (an id that was itself
// skipped adds nothing new, so it may be counted too).  Lanes with all
// positions in B0 are skipped.  The others set their missing bits with
// atomicOr; if no atomicOr ever finds its bit already set, no missing
// position is shared by two lanes and the B0 test alone is exact.  Otherwise
// (rare with a large filter) every lane checks its missing positions against
// those of the lanes before it.  The final filter is B0 plus all positions of
// the new ids either way, as in the reference.
__device__ __forceinline__ unsigned bloom_chunk(uint64_t* bloom, int nb, const BloomCfg& bc,
                                                int lane) {
    uint32_t pos[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
    uint32_t wd[4] = {0, 0, 0, 0}, bt[4] = {0, 0, 0, 0};
    unsigned unc = 0;
    if (nb >= 0) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            if (h < bc.nhash) {
                const uint32_t p = bf_pos(h, (uint32_t)nb, bc);
                pos[h] = p;
                wd[h] = bc.shift >= 0 ? (p & bc.wmask) : (p % bc.words);
                bt[h] = bc.shift >= 0 ? (p >> bc.shift) : (p / bc.words);
                if (!((bloom[wd[h]] >> bt[h]) & 1ull)) unc |= 1u << h;
            }
        }
    }
    __syncwarp();
    bool event = false;
    if (unc) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            if ((unc >> h) & 1u) {
                const unsigned long long old =
                    atomicOr((unsigned long long*)&bloom[wd[h]], 1ull << bt[h]);
                if ((old >> bt[h]) & 1ull) event = true;
            }
        }
    }
    const unsigned fresh = __ballot_sync(FULL, unc != 0u);
    if (__ballot_sync(FULL, event) == 0u) {
        __syncwarp();
        return fresh;
    }
    unsigned cov = 0;
    unsigned src = fresh;
    while (src) {
        const int i = __ffs(src) - 1;
        src &= src - 1u;
        const uint32_t s0 = __shfl_sync(FULL, pos[0], i);
        const uint32_t s1 = __shfl_sync(FULL, pos[1], i);
        const uint32_t s2 = __shfl_sync(FULL, pos[2], i);
        const uint32_t s3 = __shfl_sync(FULL, pos[3], i);
        if (lane > i && unc) {
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const uint32_t p = pos[h];
                if (((unc >> h) & 1u) && (p == s0 || p == s1 || p == s2 || p == s3)) cov |= 1u << h;
            }
        }
    }
    __syncwarp();
    return __ballot_sync(FULL, (unc & ~cov) != 0u);
}

// Partial sum of lane `lane` for one row: sum over i = lane (mod 32) of
// (q_i - b_i)^2 with FMA, in increasing i (warp_l2's per-lane loop).
template <int NE>
__device__ __forceinline__ float row_partial(const float* __restrict__ row, int dim,
                                             const float (&qreg)[NE > 0 ? NE : 1],
                                             const float* sq, int lane) {
    float s = 0.0f;
    if constexpr (NE > 0) {
        float x[NE];
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int i = lane + 32 * e;
            x[e] = i < dim ? __ldg(row + i) : 0.0f;
        }
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int i = lane + 32 * e;
            if (i < dim) {
                const float t = qreg[e] - x[e];
                s = fmaf(t, t, s);
            }
        }
    } else {
        for (int i = lane; i < dim; i += 32) {
            const float t = sq[i] - __ldg(row + i);
            s = fmaf(t, t, s);
        }
    }
    return s;
}

// Squared L2 distances of the rows of the lanes in N; lane j returns the
// distance of its own row (meaningful when bit j of N is set).  Partial sums
// are combined by a butterfly transpose-reduce: step w (16,8,4,2,1) pairs
// lanes l and l^w, which is the reference tree's pairing of m and m+w.
template <int NE>
__device__ __forceinline__ float l2_chunk(const float* __restrict__ base, int ld, int dim,
                                          const float (&qreg)[NE > 0 ? NE : 1], const float* sq,
                                          int nb, unsigned N, int lane) {
    float v[16];
    const bool up16 = lane & 16;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const int id_lo = __shfl_sync(FULL, nb, r);
        const int id_hi = __shfl_sync(FULL, nb, r + 16);
        float s_lo = 0.0f, s_hi = 0.0f;
        if ((N >> r) & 1u) s_lo = row_partial<NE>(base + (size_t)id_lo * ld, dim, qreg, sq, lane);
        if ((N >> (r + 16)) & 1u) s_hi = row_partial<NE>(base + (size_t)id_hi * ld, dim, qreg, sq, lane);
        const float send = up16 ? s_lo : s_hi;
        const float keep = up16 ? s_hi : s_lo;
        v[r] = keep + __shfl_xor_sync(FULL, send, 16);
    }
#pragma unroll
    for (int w = 8; w >= 1; w >>= 1) {
        const bool up = lane & w;
#pragma unroll
        for (int i = 0; i < w; ++i) {
            const float send = up ? v[i] : v[i + w];
            const float keep = up ? v[i + w] : v[i];
            v[i] = keep + __shfl_xor_sync(FULL, send, w);
        }
    }
    return v[0];
}

// Hamming distance of this lane's own row: popcount(q ^ b) over W4 uint4
// (warp_hamming, hashKernelGraph.h:215-224; integer, so order-free).
template <int W4>
__device__ __forceinline__ float ham_lane(const uint32_t* __restrict__ base, int ld,
                                          const uint4 (&q)[W4], int nb, bool mine) {
    int s = 0;
    if (mine) {
        const uint4* row = reinterpret_cast<const uint4*>(base + (size_t)nb * ld);
#pragma unroll
        for (int e = 0; e < W4; ++e) {
            const uint4 x = __ldg(row + e);
            s += __popc(x.x ^ q[e].x) + __popc(x.y ^ q[e].y) + __popc(x.z ^ q[e].z) +
                 __popc(x.w ^ q[e].w);
        }
    }
    return (float)s;
}

// KIND 0 = L2 with NE query elements per lane in registers (0: shared
// memory); KIND 1 = Hamming with NE uint4 of code per row.
template <int KIND, int NE>
__device__ __forceinline__ void search_query(const SearchArgs& a, int qid, unsigned char* ws,
                                             int lane) {
    Queue cand{reinterpret_cast<float*>(ws + a.cd_off), reinterpret_cast<int*>(ws + a.ci_off), 0,
               a.cap, 0.0f, 0, false};
    Queue res{reinterpret_cast<float*>(ws + a.rd_off), reinterpret_cast<int*>(ws + a.ri_off), 0,
              a.cap, 0.0f, 0, false};
    uint64_t* bloom = reinterpret_cast<uint64_t*>(ws + a.bl_off);
    float* sq = reinterpret_cast<float*>(ws + a.q_off);

    BloomCfg bc;
    bc.words = (uint32_t)a.bf_words;
    bc.nbits = (uint64_t)a.bf_words * 64ull;
    bc.shift = (a.bf_words & (a.bf_words - 1)) == 0 ? __ffs(a.bf_words) - 1 : -1;
    bc.wmask = (uint32_t)a.bf_words - 1u;
    bc.nhash = a.bf_nhash;

    // Query: registers (and shared memory for the generic L2 path).
    float qreg[(KIND == 0 && NE > 0) ? NE : 1];
    uint4 qcode[KIND == 1 ? NE : 1];
    if constexpr (KIND == 0) {
        const float* qg = reinterpret_cast<const float*>(a.queries) + (int64_t)qid * a.qld;
        if constexpr (NE > 0) {
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                const int i = lane + 32 * e;
                qreg[e] = i < a.dim ? qg[i] : 0.0f;
            }
        } else {
            qreg[0] = 0.0f;
            for (int i = lane; i < a.dim; i += 32) sq[i] = qg[i];
        }
    } else {
        const uint32_t* qg = reinterpret_cast<const uint32_t*>(a.queries) + (int64_t)qid * a.qld;
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            uint32_t w[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) w[t] = (4 * e + t) < a.dim ? qg[4 * e + t] : 0u;
            qcode[e] = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    for (int w = lane; w < a.bf_words; w += 32) bloom[w] = 0ull;
    __syncwarp();

    auto dist = [&](int nb, unsigned N) -> float {
        if constexpr (KIND == 0) {
            return l2_chunk<NE>(reinterpret_cast<const float*>(a.base), a.ld, a.dim, qreg, sq, nb, N,
                                lane);
        } else {
            return ham_lane<NE>(reinterpret_cast<const uint32_t*>(a.base), a.ld, qcode, nb,
                                (N >> lane) & 1u);
        }
    };

    song_query_trace tr = {};

    // Seeds p*n/N_MULTIPROBE, 64-bit product (kernalGraph.h:214-231).
    for (int p0 = 0; p0 < a.n_multiprobe; p0 += 32) {
        const int p = p0 + lane;
        int ep = -1;
        if (p < a.n_multiprobe)
            ep = (int)((unsigned long long)p * (unsigned long long)a.n /
                       (unsigned long long)a.n_multiprobe);
        const unsigned N = bloom_chunk(bloom, ep, bc, lane);
        const float d = dist(ep, N);
        const int c = __popc(N);
        tr.seed_count += c;
        tr.visited_nodes += c;
        tr.distance_evals += c;
        tr.frontier_pushes += q_push(cand, N, d, ep, lane);
        tr.result_updates += q_push(res, N, d, ep, lane);
        if (N) {
            tr.peak_frontier = max(tr.peak_frontier, cand.sz);
            tr.peak_results = max(tr.peak_results, res.sz);
        }
    }

    // Expansion loop (kernalGraph.h:233-289).
    for (;;) {
        if (cand.sz == 0) break;
        float cmin;
        int mi;
        q_argmin(cand, lane, cmin, mi);
        const int cn = cand.id[mi];
        __syncwarp();
        if (lane == 0) {
            cand.d[mi] = cand.d[cand.sz - 1];
            cand.id[mi] = cand.id[cand.sz - 1];
        }
        cand.sz -= 1;
        cand.max_ok = false;
        __syncwarp();
        tr.expanded_nodes += 1;
        if (res.sz == res.cap) {  // early stop: full and strictly worse than the worst
            if (!res.max_ok) q_argmax(res, lane);
            if (cmin > res.maxv) {
                tr.early_stopped = 1;
                break;
            }
        }
        const int32_t* arow = a.adj + (int64_t)cn * a.block_size;
        for (int c0 = 0; c0 < a.block_size; c0 += 32) {
            const int j = c0 + lane;
            int nb = j < a.block_size ? __ldg(arow + j) : -1;
            if (nb >= a.n) {  // impossible for a validated graph; never read out of range
                atomicExch(a.err, 1);
                nb = -1;
            }
            tr.neighbor_slots_scanned += min(32, a.block_size - c0);
            const unsigned N = bloom_chunk(bloom, nb, bc, lane);
            const float d = dist(nb, N);
            const int c = __popc(N);
            tr.visited_nodes += c;
            tr.candidate_nodes += c;
            tr.distance_evals += c;
            tr.frontier_pushes += q_push(cand, N, d, nb, lane);
            tr.result_updates += q_push(res, N, d, nb, lane);
            if (N) {
                tr.peak_frontier = max(tr.peak_frontier, cand.sz);
                tr.peak_results = max(tr.peak_results, res.sz);
            }
        }
    }

    // Trim to k (Results::pop_worst), then k x drain_best (kernalGraph.h:292-296).
    while (res.sz > a.k) {
        q_argmax(res, lane);
        if (lane == 0) {
            res.d[res.maxi] = res.d[res.sz - 1];
            res.id[res.maxi] = res.id[res.sz - 1];
        }
        res.sz -= 1;
        __syncwarp();
    }
    const int cnt = res.sz < a.k ? res.sz : a.k;
    int32_t* out = a.out + (int64_t)qid * a.k;
    for (int i = 0; i < cnt; ++i) {
        float v;
        int m;
        q_argmin(res, lane, v, m);
        const int id = res.id[m];
        __syncwarp();
        if (lane == 0) {
            out[i] = id;
            res.d[m] = res.d[res.sz - 1];
            res.id[m] = res.id[res.sz - 1];
        }
        res.sz -= 1;
        __syncwarp();
    }
    for (int i = cnt + lane; i < a.k; i += 32) out[i] = -1;
    tr.result_count = cnt;
    if (a.trace != nullptr && lane == 0) a.trace[qid] = tr;
}

template <int KIND, int NE>
__global__ void __launch_bounds__(256) search_kernel(const SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    unsigned char* ws = smem + (size_t)(threadIdx.x >> 5) * a.warp_smem;
    for (;;) {
        int qid = 0;
        if (lane == 0) qid = (int)atomicAdd(a.counter, 1u);
        qid = __shfl_sync(FULL, qid, 0);
        if (qid >= a.nq) break;
        search_query<KIND, NE>(a, qid, ws, lane);
    }
}

using KernelFn = void (*)(const SearchArgs);

KernelFn pick_kernel(int kind, const SearchArgs& a) {
    if (kind == SONG_KIND_L2) {
        if (a.dim <= 32) return search_kernel<0, 1>;
        if (a.dim <= 64) return search_kernel<0, 2>;
        if (a.dim <= 128) return search_kernel<0, 4>;
        if (a.dim <= 256) return search_kernel<0, 8>;
        return search_kernel<0, 0>;
    }
    switch (a.ld / 4) {
        case 1: return search_kernel<1, 1>;
        case 2: return search_kernel<1, 2>;
        case 3: return search_kernel<1, 3>;
        case 4: return search_kernel<1, 4>;
        case 5: return search_kernel<1, 5>;
        case 6: return search_kernel<1, 6>;
        case 7: return search_kernel<1, 7>;
        case 8: return search_kernel<1, 8>;
        default: return nullptr;
    }
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace

int search_warp_smem(int kind, int dim, int cap, int bf_words, SearchArgs* a) {
    (void)kind;
    const int capr = round_up(cap, 4);
    a->q_off = 0;
    a->cd_off = round_up(dim * 4, 16);
    a->ci_off = a->cd_off + capr * 4;
    a->rd_off = a->ci_off + capr * 4;
    a->ri_off = a->rd_off + capr * 4;
    a->bl_off = round_up(a->ri_off + capr * 4, 16);
    a->warp_smem = round_up(a->bl_off + bf_words * 8, 16);
    return a->warp_smem;
}

cudaError_t launch_search(int kind, const SearchArgs& a, int num_sms, cudaStream_t stream) {
    if (a.nq <= 0) return cudaSuccess;
    KernelFn fn = pick_kernel(kind, a);
    if (fn == nullptr) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int smem_optin = 0;
    e = cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    // Up to 8 warps per CTA while the CTA's shared memory stays within a
    // quarter of the opt-in limit, so several CTAs can share an SM.
    int warps = 8;
    while (warps > 1 && (size_t)warps * a.warp_smem > (size_t)smem_optin / 4) warps >>= 1;
    const size_t smem = (size_t)warps * a.warp_smem;
    if (smem > (size_t)smem_optin) return cudaErrorInvalidConfiguration;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int64_t need = ((int64_t)a.nq + warps - 1) / warps;
    const int grid = (int)std::min<int64_t>((int64_t)per_sm * num_sms, need);
    fn<<<grid, warps * 32, smem, stream>>>(a);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError();
}

}  // namespace song
