// song_search.cu -- sm_100a kernels of the plain SONG graph search.
//
// One warp owns one query at a time; several warps share a CTA and a
// persistent grid pulls queries from a device work counter, so every SM
// keeps many independent traversals (and their neighbour gathers) in flight.
// The reference runs one query per single-warp block with lane 0 doing all
// queue and Bloom work serially (kernalGraph.h:184-299).
//
// Results are bit-exact with the reference, including tie order and the
// QueryTrace counters, because the per-query state is the reference's own
// state and every step keeps its order:
//  * Candidates / Results (gpuHeap.h:8-108) stay unsorted slot arrays in
//    shared memory with exactly the reference's slot moves.  The O(cap)
//    scans become a two-level tournament: slots are grouped 32 at a time
//    (one slot per lane), each group's (max, first slot) and (min, first
//    slot) summary lives in a register of lane g, and "first maximal slot"
//    or "first minimal slot" is two redux.sync over those summaries.  A slot
//    write refreshes only its group (one shared load per lane + redux).
//    Ties break on the lowest slot -- the reference's first-index rule.
//  * A row of up to 32 neighbours is handled at once, lane j = slot j, but
//    the Bloom test of neighbour j sees the bits of neighbours < j exactly as
//    bf_test/bf_set in j order do (bloomFilter.h:34-48): see bloom_chunk.
//  * Distances follow warp_l2 (kernalGraph.h:157-170): lane l sums
//    (q_i - b_i)^2 over i = l (mod 32) with FMA, then a butterfly
//    transpose-reduce whose association is the reference's shfl_down tree.
//    When every term and partial sum is an integer below 2^24 (integer
//    vectors, the SIFT-shaped case) every order gives the same FP32 value,
//    so those queries take a gather-only path instead: 8 lanes per row,
//    16-byte loads, only the rows that passed the Bloom test.
//  * Pushes are applied in lane (= j) order; a push into a full queue only
//    evicts when strictly closer than the current first maximum, and the
//    maximum never grows while a queue is full, so lanes that lose against
//    the running maximum drop out with one ballot.
//  * The final trim (pop_worst) and drain (drain_best) are replayed exactly;
//    when the k+1 smallest results have distinct distances their outcome is
//    simply those k in ascending order, which is taken directly.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <atomic>
#include <climits>

#include "song_kernels.cuh"

namespace song {

std::atomic<int64_t> g_launches{0};

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr unsigned NONE = 0xffffffffu;  // "no slot" / empty group

// The mixing constants of bloomFilter.h:14-19: two per hash function.
__constant__ uint64_t kBloomMix[8] = {
    0x4bcb391f924ed183ULL, 0xa0ab69ccd854fc0aULL, 0x91086b9cecf5e3b7ULL, 0xc68e01641bead407ULL,
    0x3a7b976128a30449ULL, 0x6d122efabfc4d99fULL, 0xe6700ef8715030e2ULL, 0x80dd0c3bffcfb45bULL,
};

__device__ __forceinline__ unsigned fbits(float x) { return __float_as_uint(x); }

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Read-only loads of base rows (the read-only data path; an L1 no-allocate
// variant measured slightly slower).
__device__ __forceinline__ float ld_row(const float* p) { return __ldg(p); }
__device__ __forceinline__ float4 ld_row(const float4* p) { return __ldg(p); }
__device__ __forceinline__ uint4 ld_row(const uint4* p) { return __ldg(p); }
__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Tensor memory (TMEM) access of one warp: 32 lanes x 32-bit columns.  The
// wait is part of the same asm statement, so the loaded value is never used
// before the load has completed, and a store has completed before the next
// access of the same column.
__device__ __forceinline__ unsigned tm_ld(uint32_t taddr) {
    unsigned r;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r)
        : "r"(taddr)
        : "memory");
    return r;
}
// Two columns with one wait.
__device__ __forceinline__ void tm_ld2(uint32_t a0, uint32_t a1, unsigned& r0, unsigned& r1) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%2];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%1}, [%3];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r0), "=r"(r1)
        : "r"(a0), "r"(a1)
        : "memory");
}
__device__ __forceinline__ void tm_st(uint32_t taddr, unsigned v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};\n\t"
        "tcgen05.wait::st.sync.aligned;"
        :
        : "r"(taddr), "r"(v)
        : "memory");
}
// Two columns with one wait.
__device__ __forceinline__ void tm_st2(uint32_t a0, uint32_t a1, unsigned v0, unsigned v1) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%2};\n\t"
        "tcgen05.st.sync.aligned.32x32b.x1.b32 [%1], {%3};\n\t"
        "tcgen05.wait::st.sync.aligned;"
        :
        : "r"(a0), "r"(a1), "r"(v0), "r"(v1)
        : "memory");
}

// Slot queue of capacity <= 1024 * GPL.  Distances live in shared memory;
// ids live in shared memory (TM = 0) or in the warp's 32 TMEM lanes, one
// column per group of 32 slots, slot 32g + l at lane l of column tid + g
// (TM = 1).  TD = 1 (with TM = 1): the distances too, in the columns from
// tdd on, laid out like the ids.  The summary of group g (slots 32g ..
// 32g+31) is held by lane g % 32 in entry g / 32.  Distances are
// non-negative, so their bit patterns order like the floats.  All scalar
// fields are warp-uniform.
template <int GPL, int TM = 0, int TD = 0>
struct Queue {
    float* d;      // TD = 0
    int* id;       // TM = 0
    uint32_t tid;  // TM = 1: TMEM address of group 0's id column
    uint32_t tdd;  // TD = 1: TMEM address of group 0's distance column
    int sz;
    int cap;
    unsigned xb[GPL], xi[GPL];  // group maximum bits, first slot holding it (NONE = empty)
    unsigned nb[GPL], ni[GPL];  // group minimum bits, first slot holding it
    // The queue's maximum and its first slot while cx holds (results queue
    // only: its maximum is read at every early-stop check and push): kept
    // through appends and evictions instead of recomputed from the group
    // summaries each time.
    unsigned cxb, cxi;
    bool cx;
};

// Id of slot s (warp-uniform s; every lane gets it).
template <int GPL, int TM, int TD>
__device__ __forceinline__ int q_id(const Queue<GPL, TM, TD>& q, int s) {
    if constexpr (TM) {
        const unsigned r = tm_ld(q.tid + (uint32_t)(s >> 5));
        return (int)__shfl_sync(FULL, r, s & 31);
    } else {
        return q.id[s];
    }
}

// Id of slot s := v (warp-uniform s and v; called by every lane).
template <int GPL, int TM, int TD>
__device__ __forceinline__ void q_set_id(Queue<GPL, TM, TD>& q, int s, int v, int lane) {
    if constexpr (TM) {
        const uint32_t a = q.tid + (uint32_t)(s >> 5);
        unsigned r = tm_ld(a);
        if (lane == (s & 31)) r = (unsigned)v;
        tm_st(a, r);
    } else {
        if (lane == 0) q.id[s] = v;
    }
}

// Distance bits of slot s (warp-uniform s; every lane gets them).
template <int GPL, int TM, int TD>
__device__ __forceinline__ unsigned q_dbits(const Queue<GPL, TM, TD>& q, int s) {
    if constexpr (TD) {
        const unsigned r = tm_ld(q.tdd + (uint32_t)(s >> 5));
        return __shfl_sync(FULL, r, s & 31);
    } else {
        return fbits(q.d[s]);
    }
}

// Slot s := (distance bits b, id v) (warp-uniform s, b, v; called by every
// lane).  TD: both columns read with one wait.
template <int GPL, int TM, int TD>
__device__ __forceinline__ void q_set_slot(Queue<GPL, TM, TD>& q, int s, unsigned b, int v, int lane) {
    if constexpr (TD) {
        const uint32_t ai = q.tid + (uint32_t)(s >> 5), ad = q.tdd + (uint32_t)(s >> 5);
        unsigned ri, rd;
        tm_ld2(ai, ad, ri, rd);
        if (lane == (s & 31)) {
            ri = (unsigned)v;
            rd = b;
        }
        tm_st2(ai, ad, ri, rd);
    } else {
        if (lane == 0) reinterpret_cast<unsigned*>(q.d)[s] = b;
        q_set_id(q, s, v, lane);
    }
}

// Distance bits of slot s := b (warp-uniform s and b; called by every lane).
template <int GPL, int TM, int TD>
__device__ __forceinline__ void q_set_dbits(Queue<GPL, TM, TD>& q, int s, unsigned b, int lane) {
    if constexpr (TD) {
        const uint32_t ad = q.tdd + (uint32_t)(s >> 5);
        unsigned r = tm_ld(ad);
        if (lane == (s & 31)) r = b;
        tm_st(ad, r);
    } else {
        if (lane == 0) reinterpret_cast<unsigned*>(q.d)[s] = b;
    }
}

template <int GPL, int TM, int TD>
__device__ __forceinline__ void q_init(Queue<GPL, TM, TD>& q, float* d, int* id, uint32_t tid,
                                       uint32_t tdd, int cap) {
    q.d = d;
    q.id = id;
    q.tid = tid;
    q.tdd = tdd;
    q.sz = 0;
    q.cap = cap;
    q.cx = false;
#pragma unroll
    for (int r = 0; r < GPL; ++r) {
        q.xb[r] = 0u;
        q.xi[r] = NONE;
        q.nb[r] = 0xffffffffu;
        q.ni[r] = NONE;
    }
}

// Refresh the summary of group g from the slot array.  MIN: also the minimum.
// `b`: this lane's slot's distance bits (0 if the slot is empty).
template <bool MIN, int GPL, int TM, int TD>
__device__ __forceinline__ void group_update_b(Queue<GPL, TM, TD>& q, int g, int lane, unsigned b) {
    const int s = (g << 5) + lane;
    const bool occ = s < q.sz;
    const unsigned mx = __reduce_max_sync(FULL, b);
    const unsigned mxi = __reduce_min_sync(FULL, (occ && b == mx) ? (unsigned)s : NONE);
    unsigned mn = 0xffffffffu, mni = NONE;
    if constexpr (MIN) {
        mn = __reduce_min_sync(FULL, occ ? b : 0xffffffffu);
        mni = __reduce_min_sync(FULL, (occ && b == mn) ? (unsigned)s : NONE);
    }
    if ((g & 31) == lane) {
        const int r = g >> 5;
#pragma unroll
        for (int t = 0; t < GPL; ++t) {
            if (t == r) {
                q.xb[t] = mx;
                q.xi[t] = mxi;
                if constexpr (MIN) {
                    q.nb[t] = mn;
                    q.ni[t] = mni;
                }
            }
        }
    }
}

template <bool MIN, int GPL, int TM, int TD>
__device__ __forceinline__ void group_update(Queue<GPL, TM, TD>& q, int g, int lane) {
    const bool occ = (g << 5) + lane < q.sz;
    unsigned b;
    if constexpr (TD) {
        const unsigned c = tm_ld(q.tdd + (uint32_t)g);
        b = occ ? c : 0u;
    } else {
        b = occ ? fbits(q.d[(g << 5) + lane]) : 0u;
    }
    group_update_b<MIN>(q, g, lane, b);
}

// First slot holding the maximum over [0, sz) (gpuHeap.h:29, :73, :83, :93).
template <int GPL, int TM, int TD>
__device__ __forceinline__ void root_max(const Queue<GPL, TM, TD>& q, unsigned& mb, unsigned& mi) {
    unsigned b = 0u, i = NONE;
#pragma unroll
    for (int r = 0; r < GPL; ++r)
        if (q.xi[r] != NONE && (i == NONE || q.xb[r] > b)) {
            b = q.xb[r];
            i = q.xi[r];
        }
    mb = __reduce_max_sync(FULL, i != NONE ? b : 0u);
    mi = __reduce_min_sync(FULL, (i != NONE && b == mb) ? i : NONE);
}

// First slot holding the minimum over [0, sz) (gpuHeap.h:42, :263).
template <int GPL, int TM, int TD>
__device__ __forceinline__ void root_min(const Queue<GPL, TM, TD>& q, unsigned& mb, unsigned& mi) {
    unsigned b = 0xffffffffu, i = NONE;
#pragma unroll
    for (int r = 0; r < GPL; ++r)
        if (q.ni[r] != NONE && (i == NONE || q.nb[r] < b)) {
            b = q.nb[r];
            i = q.ni[r];
        }
    mb = __reduce_min_sync(FULL, i != NONE ? b : 0xffffffffu);
    mi = __reduce_min_sync(FULL, (i != NONE && b == mb) ? i : NONE);
}

// Move the last slot into slot `hole` and shrink (the removal of
// Candidates::pop_min, Results::pop_worst and drain_best).
template <bool MIN, int GPL, int TM, int TD>
__device__ __forceinline__ void q_remove(Queue<GPL, TM, TD>& q, int hole, int lane) {
    const int last = q.sz - 1;
    __syncwarp();
    if (hole != last) {
        if constexpr (TD) {
            q_set_slot(q, hole, q_dbits(q, last), q_id(q, last), lane);
        } else if constexpr (TM) {
            if (lane == 0) q.d[hole] = q.d[last];
            q_set_id(q, hole, q_id(q, last), lane);
        } else {
            if (lane == 0) q.d[hole] = q.d[last];
            if (lane == 0) q.id[hole] = q.id[last];
        }
    }
    __syncwarp();
    q.sz = last;
    q.cx = false;
    group_update<MIN>(q, hole >> 5, lane);
    if ((last >> 5) != (hole >> 5)) group_update<MIN>(q, last >> 5, lane);
}

// Maximum and its first slot (gpuHeap.h:29, :73), from the cache when it holds.
template <int GPL, int TM, int TD>
__device__ __forceinline__ void root_max_c(Queue<GPL, TM, TD>& q, unsigned& mb, unsigned& mi) {
    if (!q.cx) {
        root_max(q, q.cxb, q.cxi);
        q.cx = true;
    }
    mb = q.cxb;
    mi = q.cxi;
}

// Id of slot `hole`, then q_remove(hole): the same queue afterwards, with the
// TMEM columns of `hole` and of the last slot read once (one wait) instead
// of once per id access.
template <bool MIN, int GPL, int TM, int TD>
__device__ __forceinline__ int q_pop(Queue<GPL, TM, TD>& q, int hole, int lane) {
    static_assert(!TD, "pops serve the candidate queue, whose distances are in shared memory");
    if constexpr (!TM) {
        const int id = q.id[hole];
        q_remove<MIN>(q, hole, lane);
        return id;
    } else {
        const int last = q.sz - 1;
        const uint32_t ch = q.tid + (uint32_t)(hole >> 5), cl = q.tid + (uint32_t)(last >> 5);
        unsigned rh, rl;
        if (ch == cl) {
            rh = tm_ld(ch);
            rl = rh;
        } else {
            tm_ld2(ch, cl, rh, rl);
        }
        const int id = (int)__shfl_sync(FULL, rh, hole & 31);
        const unsigned idl = __shfl_sync(FULL, rl, last & 31);
        __syncwarp();
        if (hole != last) {
            if (lane == 0) q.d[hole] = q.d[last];
            if (lane == (hole & 31)) rh = idl;
            tm_st(ch, rh);
        }
        __syncwarp();
        q.sz = last;
        q.cx = false;
        group_update<MIN>(q, hole >> 5, lane);
        if ((last >> 5) != (hole >> 5)) group_update<MIN>(q, last >> 5, lane);
        return id;
    }
}

// Push (d, nb) of every lane in N, in lane order, with the semantics of
// Candidates::push / Results::try_push (gpuHeap.h:23-36, :68-77).
// Returns how many pushes were accepted.  `stage` (32 ints, TM = 1 only)
// receives the ids in rank order for the column writes of an append.
// RC: keep the queue's cached maximum (cxb, cxi) current.
template <bool MIN, bool RC = false, int GPL, int TM, int TD>
__device__ __forceinline__ int q_push(Queue<GPL, TM, TD>& q, unsigned N, float d, int nb, int lane,
                                      int* stage) {
    if (N == 0u) return 0;
    const bool mine = (N >> lane) & 1u;
    const int rank = __popc(N & lanemask_lt(lane));
    const int nm = __popc(N);
    const int room = q.cap - q.sz;
    int acc = 0;
    if (room > 0) {
        const int a = nm < room ? nm : room;
        if (mine && rank < a) {
            if constexpr (TD) stage[32 + rank] = (int)fbits(d);
            else q.d[q.sz + rank] = d;
            if constexpr (TM) stage[rank] = nb;
            else q.id[q.sz + rank] = nb;
        }
        __syncwarp();
        const int g0 = q.sz >> 5, g1 = (q.sz + a - 1) >> 5;
        if constexpr (TD) {  // ids and distances, column by column; each group's summary from its column
            const int sz0 = q.sz;
            q.sz += a;
            for (int g = g0; g <= g1; ++g) {
                const uint32_t ci = q.tid + (uint32_t)g, cd = q.tdd + (uint32_t)g;
                unsigned ri, rd;
                tm_ld2(ci, cd, ri, rd);
                const int rr = (g << 5) + lane - sz0;
                if (rr >= 0 && rr < a) {
                    ri = (unsigned)stage[rr];
                    rd = (unsigned)stage[32 + rr];
                }
                tm_st2(ci, cd, ri, rd);
                group_update_b<MIN>(q, g, lane, (g << 5) + lane < q.sz ? rd : 0u);
            }
            q.sz = sz0;
            __syncwarp();
        } else if constexpr (TM) {  // slots sz .. sz+a-1 take the staged ids, column by column
            for (int g = g0; g <= g1; ++g) {
                const uint32_t col = q.tid + (uint32_t)g;
                unsigned r = tm_ld(col);
                const int rr = (g << 5) + lane - q.sz;
                if (rr >= 0 && rr < a) r = (unsigned)stage[rr];
                tm_st(col, r);
            }
            __syncwarp();
        }
        if (RC && q.cx) {  // the appended entries sit after every slot: only a larger one moves the maximum
            const bool app = mine && rank < a;
            const unsigned am = __reduce_max_sync(FULL, app ? fbits(d) : 0u);
            if (am > q.cxb) {
                const int fl = __ffs(__ballot_sync(FULL, app && fbits(d) == am)) - 1;
                q.cxb = am;
                q.cxi = (unsigned)(q.sz + __popc(N & lanemask_lt(fl)));
            }
        }
        q.sz += a;
        if constexpr (!TD)
            for (int g = g0; g <= g1; ++g) group_update<MIN>(q, g, lane);
        acc = a;
    }
    if (nm > room) {
        unsigned M, fi;
        if constexpr (RC) root_max_c(q, M, fi);
        else root_max(q, M, fi);
        unsigned rest = __ballot_sync(FULL, mine && rank >= room && fbits(d) < M);
        while (rest) {
            const int j = __ffs(rest) - 1;
            const float dj = __shfl_sync(FULL, d, j);
            const int nj = __shfl_sync(FULL, nb, j);
            if constexpr (TD) {  // the slot's two columns, then the group's summary from the distance column
                const int g = (int)(fi >> 5);
                const uint32_t ci = q.tid + (uint32_t)g, cd = q.tdd + (uint32_t)g;
                unsigned ri, rd;
                tm_ld2(ci, cd, ri, rd);
                if (lane == (int)(fi & 31)) {
                    ri = (unsigned)nj;
                    rd = fbits(dj);
                }
                tm_st2(ci, cd, ri, rd);
                group_update_b<MIN>(q, g, lane, (g << 5) + lane < q.sz ? rd : 0u);
            } else {
                if (lane == 0) q.d[fi] = dj;
                q_set_id(q, (int)fi, nj, lane);
                __syncwarp();
                group_update<MIN>(q, (int)(fi >> 5), lane);
            }
            ++acc;
            root_max(q, M, fi);
            rest &= ~(1u << j);
            rest &= __ballot_sync(FULL, fbits(d) < M);
        }
        if constexpr (RC) {
            q.cxb = M;
            q.cxi = fi;
            q.cx = true;
        }
    }
    return acc;
}

struct BloomCfg {
    uint64_t nbits;  // BF_WORDS * 64
    uint32_t words;  // BF_WORDS
    uint32_t wmask;  // BF_WORDS - 1 when a power of two
    int shift;       // log2(BF_WORDS), or -1
    int nhash;       // BF_NHASH
};

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
                const uint32_t w64 = bc.shift >= 0 ? (p & bc.wmask) : (p % bc.words);
                const uint32_t b64 = bc.shift >= 0 ? (p >> bc.shift) : (p / bc.words);
                // the same bit as a 32-bit word: the low half of 64-bit word w is word 2w
                wd[h] = 2u * w64 + (b64 >> 5);
                bt[h] = b64 & 31u;
                if (!((reinterpret_cast<const uint32_t*>(bloom)[wd[h]] >> bt[h]) & 1u)) unc |= 1u << h;
            }
        }
    }
    __syncwarp();
    bool event = false;
    if (unc) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            if ((unc >> h) & 1u) {
                const unsigned old = atomicOr(reinterpret_cast<unsigned*>(bloom) + wd[h], 1u << bt[h]);
                if ((old >> bt[h]) & 1u) event = true;
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
            x[e] = i < dim ? ld_row(row + i) : 0.0f;
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
            const float t = sq[i] - ld_row(row + i);
            s = fmaf(t, t, s);
        }
    }
    return s;
}

// Squared L2 in the reference's exact order for the rows of the lanes in N;
// lane j returns the distance of its own row.  Partial sums are combined by
// a butterfly transpose-reduce: step w (16,8,4,2,1) pairs lanes l and l^w,
// which is the reference tree's pairing of m and m+w.
template <int NE>
__device__ __forceinline__ float l2_exact(const float* __restrict__ base, int ld, int dim,
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

// Squared L2 when every partial sum is an exact integer (any order gives the
// same FP32 value): only the rows of the lanes in N are gathered, 4 rows per
// pass with 8 lanes per row and NV 16-byte loads per lane (dim = 32 * NV),
// two passes in flight.  `rows` is a 32-entry per-warp shared list.
template <int NV>
__device__ __forceinline__ float l2_int(const float* __restrict__ base, int ld,
                                        const float4 (&qv)[NV], int nb, unsigned N,
                                        int* rows, int lane) {
    const bool mine = (N >> lane) & 1u;
    const int rank = __popc(N & lanemask_lt(lane));
    const int m = __popc(N);
    if (mine) rows[rank] = nb;
    __syncwarp();
    const int grp = lane >> 3, t = lane & 7;
    float out = 0.0f;
    for (int p0 = 0; p0 < m; p0 += 8) {
        const int ra = p0 + grp, rb = p0 + 4 + grp;
        float4 xa[NV], xb[NV];
        const bool va = ra < m, vb = rb < m;
        const float4* pa = reinterpret_cast<const float4*>(base + (size_t)(va ? rows[ra] : 0) * ld);
        const float4* pb = reinterpret_cast<const float4*>(base + (size_t)(vb ? rows[rb] : 0) * ld);
#pragma unroll
        for (int e = 0; e < NV; ++e) xa[e] = va ? ld_row(pa + t + 8 * e) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int e = 0; e < NV; ++e) xb[e] = vb ? ld_row(pb + t + 8 * e) : make_float4(0.f, 0.f, 0.f, 0.f);
        float sa = 0.0f, sb = 0.0f;
#pragma unroll
        for (int e = 0; e < NV; ++e) {
            float u;
            u = qv[e].x - xa[e].x; sa = fmaf(u, u, sa);
            u = qv[e].y - xa[e].y; sa = fmaf(u, u, sa);
            u = qv[e].z - xa[e].z; sa = fmaf(u, u, sa);
            u = qv[e].w - xa[e].w; sa = fmaf(u, u, sa);
            u = qv[e].x - xb[e].x; sb = fmaf(u, u, sb);
            u = qv[e].y - xb[e].y; sb = fmaf(u, u, sb);
            u = qv[e].z - xb[e].z; sb = fmaf(u, u, sb);
            u = qv[e].w - xb[e].w; sb = fmaf(u, u, sb);
        }
#pragma unroll
        for (int w = 4; w >= 1; w >>= 1) {
            sa += __shfl_xor_sync(FULL, sa, w);
            sb += __shfl_xor_sync(FULL, sb, w);
        }
        // row of rank r sits in group r % 4 of pass r / 4
        const float ga = __shfl_sync(FULL, sa, (rank & 3) << 3);
        const float gb = __shfl_sync(FULL, sb, (rank & 3) << 3);
        if (mine && (rank >> 2) == (p0 >> 2)) out = ga;
        if (mine && (rank >> 2) == (p0 >> 2) + 1) out = gb;
    }
    __syncwarp();
    return out;
}

// Squared L2 of integer vectors in [0, 255] from their byte rows:
// sum (q - b)^2 = sum q^2 + sum b^2 - 2 sum q*b, each term an exact unsigned
// byte dot product (dp4a), so the result is the exact integer distance --
// the same FP32 value the reference's float arithmetic produces, since all
// of its partial sums are integers below 2^24 (dim <= 256).  Rows are read
// in 16-byte chunks, 8 lanes per row, NC chunks per lane, 4 rows per pass
// and two passes in flight; `qb` holds this lane's query chunks and `qq`
// the query's sum of squares.
template <int NC>
__device__ __forceinline__ float l2_u8(const uint8_t* __restrict__ base, int ld, int nch,
                                       const uint4 (&qb)[NC], int qq, int nb, unsigned N,
                                       int* rows, int lane) {
    const bool mine = (N >> lane) & 1u;
    const int rank = __popc(N & lanemask_lt(lane));
    const int m = __popc(N);
    if (mine) rows[rank] = nb;
    __syncwarp();
    const int grp = lane >> 3, t = lane & 7;
    float out = 0.0f;
    for (int p0 = 0; p0 < m; p0 += 8) {
        const int ra = p0 + grp, rb = p0 + 4 + grp;
        const bool va = ra < m, vb = rb < m;
        const uint4* pa = reinterpret_cast<const uint4*>(base + (size_t)(va ? rows[ra] : 0) * ld);
        const uint4* pb = reinterpret_cast<const uint4*>(base + (size_t)(vb ? rows[rb] : 0) * ld);
        uint4 xa[NC], xb[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int ch = t + 8 * c;
            xa[c] = (va && ch < nch) ? ld_row(pa + ch) : make_uint4(0u, 0u, 0u, 0u);
            xb[c] = (vb && ch < nch) ? ld_row(pb + ch) : make_uint4(0u, 0u, 0u, 0u);
        }
        unsigned qa = 0u, ba = 0u, qbb = 0u, bbb = 0u;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            qa = __dp4a(qb[c].x, xa[c].x, qa);
            qa = __dp4a(qb[c].y, xa[c].y, qa);
            qa = __dp4a(qb[c].z, xa[c].z, qa);
            qa = __dp4a(qb[c].w, xa[c].w, qa);
            ba = __dp4a(xa[c].x, xa[c].x, ba);
            ba = __dp4a(xa[c].y, xa[c].y, ba);
            ba = __dp4a(xa[c].z, xa[c].z, ba);
            ba = __dp4a(xa[c].w, xa[c].w, ba);
            qbb = __dp4a(qb[c].x, xb[c].x, qbb);
            qbb = __dp4a(qb[c].y, xb[c].y, qbb);
            qbb = __dp4a(qb[c].z, xb[c].z, qbb);
            qbb = __dp4a(qb[c].w, xb[c].w, qbb);
            bbb = __dp4a(xb[c].x, xb[c].x, bbb);
            bbb = __dp4a(xb[c].y, xb[c].y, bbb);
            bbb = __dp4a(xb[c].z, xb[c].z, bbb);
            bbb = __dp4a(xb[c].w, xb[c].w, bbb);
        }
        int sa = (int)ba - 2 * (int)qa, sb = (int)bbb - 2 * (int)qbb;
#pragma unroll
        for (int w = 4; w >= 1; w >>= 1) {
            sa += __shfl_xor_sync(FULL, sa, w);
            sb += __shfl_xor_sync(FULL, sb, w);
        }
        // row of rank r sits in group r % 4 of pass r / 4
        const int ga = __shfl_sync(FULL, sa, (rank & 3) << 3);
        const int gb = __shfl_sync(FULL, sb, (rank & 3) << 3);
        if (mine && (rank >> 2) == (p0 >> 2)) out = (float)(qq + ga);
        if (mine && (rank >> 2) == (p0 >> 2) + 1) out = (float)(qq + gb);
    }
    __syncwarp();
    return out;
}

// Hamming distance of this lane's own row: popcount(q ^ b) over the dim code
// words (warp_hamming, hashKernelGraph.h:215-224; integer, so order-free).
// Rows are W4 uint4 wide; words at or past dim are padding and never count,
// whatever they hold (the query's are zero, a caller's rows may not be).
template <int W4>
__device__ __forceinline__ float ham_lane(const uint32_t* __restrict__ base, int ld, int dim,
                                          const uint4 (&q)[W4], int nb, bool mine) {
    int s = 0;
    if (mine) {
        const uint4* row = reinterpret_cast<const uint4*>(base + (size_t)nb * ld);
#pragma unroll
        for (int e = 0; e < W4; ++e) {
            if (4 * e < dim) {
                uint4 x = ld_row(row + e);
                if (4 * e + 4 > dim) {  // the chunk holding the last word: drop the rest
                    const int r = dim - 4 * e;
                    if (r < 2) x.y = q[e].y;
                    if (r < 3) x.z = q[e].z;
                    x.w = q[e].w;
                }
                s += __popc(x.x ^ q[e].x) + __popc(x.y ^ q[e].y) + __popc(x.z ^ q[e].z) +
                     __popc(x.w ^ q[e].w);
            }
        }
    }
    return (float)s;
}

// Writes the k results (kernalGraph.h:292-296): `while (sz > k) pop_worst()`
// then `drain_best(out, k)`, -1 padding.  The k+1 smallest results are
// extracted first (into the free candidate arrays); if their distances are
// strictly increasing the replay's outcome is exactly those k in order.
// Otherwise the extraction is undone and the trims and drains are replayed.
// `scratch` (TM = 1: at least cap ints of shared memory) holds the slots of
// the extracted results; with TM = 0 the free candidate id array does.
template <int GPL, int TM, int TD, int TMC>
__device__ __forceinline__ int finish(Queue<GPL, TM, TD>& res, Queue<GPL, TMC>& cand, int k,
                                      int32_t* out, float* outd, int lane, int* scratch) {
    const int ng = (res.sz + 31) >> 5;
    for (int g = 0; g < ng; ++g) group_update<true>(res, g, lane);
    const int cnt = res.sz < k ? res.sz : k;
    const int take = res.sz < k + 1 ? res.sz : k + 1;
    unsigned* xv = reinterpret_cast<unsigned*>(cand.d);  // extracted distance bits
    int* xs = TMC ? scratch : cand.id;                   // their slots
    for (int i = 0; i < take; ++i) {
        unsigned mb, mi;
        root_min(res, mb, mi);
        if (lane == 0) {
            xv[i] = mb;
            xs[i] = (int)mi;
        }
        q_set_dbits(res, (int)mi, 0xffffffffu, lane);  // out of every minimum
        __syncwarp();
        group_update<true>(res, (int)(mi >> 5), lane);
    }
    bool distinct = true;
    for (int i = lane; i + 1 < take; i += 32) distinct &= xv[i] < xv[i + 1];
    distinct = __all_sync(FULL, distinct);
    if (distinct) {
        if constexpr (TM) {
            for (int i = 0; i < cnt; ++i) {
                const int id = q_id(res, xs[i]);
                if (lane == (i & 31)) out[i] = id;
            }
            for (int i = lane; i < cnt; i += 32)
                if (outd) outd[i] = __uint_as_float(xv[i]);
        } else {
            for (int i = lane; i < cnt; i += 32) {
                out[i] = res.id[xs[i]];
                if (outd) outd[i] = __uint_as_float(xv[i]);
            }
        }
    } else {
        if constexpr (TD) {
            for (int i = 0; i < take; ++i) q_set_dbits(res, xs[i], xv[i], lane);
        } else {
            for (int i = lane; i < take; i += 32) reinterpret_cast<unsigned*>(res.d)[xs[i]] = xv[i];
        }
        __syncwarp();
        for (int g = 0; g < ng; ++g) group_update<true>(res, g, lane);
        while (res.sz > k) {  // Results::pop_worst
            unsigned mb, mi;
            root_max(res, mb, mi);
            q_remove<true>(res, (int)mi, lane);
        }
        for (int i = 0; i < cnt; ++i) {  // Results::drain_best
            unsigned mb, mi;
            root_min(res, mb, mi);
            const int id = q_id(res, (int)mi);
            if (lane == 0) {
                out[i] = id;
                if (outd) outd[i] = __uint_as_float(mb);
            }
            q_remove<true>(res, (int)mi, lane);
        }
    }
    for (int i = cnt + lane; i < k; i += 32) {
        out[i] = -1;
        if (outd) outd[i] = INFINITY;
    }
    return cnt;
}

// Accumulate (q - b)^2 over one 16-byte chunk of a compressed row: 8 BF16 or
// 16 FP8 e4m3 values (times the row's scale), FP32 arithmetic.
template <int DT>
__device__ __forceinline__ void chunk_l2(const uint4 x, const float* qc, float scale, float& acc) {
    const unsigned w[4] = {x.x, x.y, x.z, x.w};
    if constexpr (DT == SONG_PREC_BF16) {
        const float4 q0 = *reinterpret_cast<const float4*>(qc);
        const float4 q1 = *reinterpret_cast<const float4*>(qc + 4);
        const float q[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float lo = __uint_as_float(w[i] << 16);
            const float hi = __uint_as_float(w[i] & 0xffff0000u);
            float t = q[2 * i] - lo;
            acc = fmaf(t, t, acc);
            t = q[2 * i + 1] - hi;
            acc = fmaf(t, t, acc);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float4 q = *reinterpret_cast<const float4*>(qc + 4 * i);
            const __half2_raw h01 = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] & 0xffffu), __NV_E4M3);
            const __half2_raw h23 = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] >> 16), __NV_E4M3);
            const float2 b01 = __half22float2(__half2(h01));
            const float2 b23 = __half22float2(__half2(h23));
            float t = fmaf(-scale, b01.x, q.x);
            acc = fmaf(t, t, acc);
            t = fmaf(-scale, b01.y, q.y);
            acc = fmaf(t, t, acc);
            t = fmaf(-scale, b23.x, q.z);
            acc = fmaf(t, t, acc);
            t = fmaf(-scale, b23.y, q.w);
            acc = fmaf(t, t, acc);
        }
    }
}

// Precision-form distances of the rows of the lanes in N (lane j gets its
// own row's): 4 rows per pass, 8 lanes per row, 16-byte loads of the
// compressed rows, query from shared memory, two passes in flight.
template <int DT>
__device__ __forceinline__ float l2_lowp(const SearchArgs& a, const float* sq, int nb, unsigned N,
                                         int* rows, int lane) {
    constexpr int EPC = DT == SONG_PREC_BF16 ? 8 : 16;  // elements per 16-byte chunk
    const bool mine = (N >> lane) & 1u;
    const int rank = __popc(N & lanemask_lt(lane));
    const int m = __popc(N);
    if (mine) rows[rank] = nb;
    __syncwarp();
    const int grp = lane >> 3, t = lane & 7;
    const int nchunk = a.lowp_ld >> 4;
    const unsigned char* lp = reinterpret_cast<const unsigned char*>(a.lowp);
    float out = 0.0f;
    for (int p0 = 0; p0 < m; p0 += 8) {
        const int ra = p0 + grp, rb = p0 + 4 + grp;
        const bool va = ra < m, vb = rb < m;
        const int ia = va ? rows[ra] : 0, ib = vb ? rows[rb] : 0;
        const uint4* pa = reinterpret_cast<const uint4*>(lp + (size_t)ia * a.lowp_ld);
        const uint4* pb = reinterpret_cast<const uint4*>(lp + (size_t)ib * a.lowp_ld);
        float sca = 1.0f, scb = 1.0f;
        if constexpr (DT == SONG_PREC_FP8) {
            sca = va ? __ldg(a.scales + ia) : 0.0f;
            scb = vb ? __ldg(a.scales + ib) : 0.0f;
        }
        float sa = 0.0f, sb = 0.0f;
        for (int c = t; c < nchunk; c += 8) {
            const uint4 xa = va ? ld_row(pa + c) : make_uint4(0u, 0u, 0u, 0u);
            const uint4 xb = vb ? ld_row(pb + c) : make_uint4(0u, 0u, 0u, 0u);
            chunk_l2<DT>(xa, sq + c * EPC, sca, sa);
            chunk_l2<DT>(xb, sq + c * EPC, scb, sb);
        }
#pragma unroll
        for (int w = 4; w >= 1; w >>= 1) {
            sa += __shfl_xor_sync(FULL, sa, w);
            sb += __shfl_xor_sync(FULL, sb, w);
        }
        const float ga = __shfl_sync(FULL, sa, (rank & 3) << 3);
        const float gb = __shfl_sync(FULL, sb, (rank & 3) << 3);
        if (mine && (rank >> 2) == (p0 >> 2)) out = ga;
        if (mine && (rank >> 2) == (p0 >> 2) + 1) out = gb;
    }
    __syncwarp();
    return out;
}

// Precision form, final step: exact FP32 distances of every entry of the
// results queue (FP32 rows, 8 lanes per row), then the k smallest by
// (distance, id) in ascending order, -1 padded.
template <int GPL, int TM, int TD, int TMC>
__device__ __forceinline__ int rerank_finish(const SearchArgs& a, Queue<GPL, TM, TD>& res,
                                             Queue<GPL, TMC>& cand, const float* sq, int32_t* out,
                                             float* outd, int lane) {
    const int m = res.sz;
    float* rd = cand.d;
    int* rid = cand.id;  // TM = 0 only; with TM = 1 the ids stay in res's TMEM columns
    const float* base = reinterpret_cast<const float*>(a.base);
    const int nch = a.ld >> 2;  // float4 per FP32 row
    const int grp = lane >> 3, t = lane & 7;
    unsigned gid = 0;  // TM = 1: ids of the current group, lane l = slot 32g + l
    for (int p0 = 0; p0 < m; p0 += 4) {
        const int r = p0 + grp;
        const bool v = r < m;
        int id;
        if constexpr (TM) {
            if ((p0 & 31) == 0) gid = tm_ld(res.tid + (uint32_t)(p0 >> 5));
            id = (int)__shfl_sync(FULL, gid, r & 31);
            if (!v) id = 0;
        } else {
            id = v ? res.id[r] : 0;
        }
        const float4* row = reinterpret_cast<const float4*>(base + (size_t)id * a.ld);
        float acc = 0.0f;
        for (int c = t; c < nch; c += 8) {
            const float4 x = v ? ld_row(row + c) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 q = *reinterpret_cast<const float4*>(sq + 4 * c);
            float u = q.x - x.x;
            acc = fmaf(u, u, acc);
            u = q.y - x.y;
            acc = fmaf(u, u, acc);
            u = q.z - x.z;
            acc = fmaf(u, u, acc);
            u = q.w - x.w;
            acc = fmaf(u, u, acc);
        }
#pragma unroll
        for (int w = 4; w >= 1; w >>= 1) acc += __shfl_xor_sync(FULL, acc, w);
        if (t == 0 && v) {
            rd[r] = acc;
            if constexpr (!TM) rid[r] = id;
        }
    }
    __syncwarp();
    const int cnt = m < a.k ? m : a.k;
    for (int i = 0; i < cnt; ++i) {
        unsigned bb = 0xffffffffu, bi = 0xffffffffu;
        for (int s0 = 0; s0 < m; s0 += 32) {  // warp-uniform trip count (TMEM loads are collective)
            const int s2 = s0 + lane;
            unsigned id;
            if constexpr (TM) id = tm_ld(res.tid + (uint32_t)(s0 >> 5));
            else id = s2 < m ? (unsigned)rid[s2] : 0u;
            if (s2 < m) {
                const unsigned b = fbits(rd[s2]);
                if (b < bb || (b == bb && id < bi)) {
                    bb = b;
                    bi = id;
                }
            }
        }
        const unsigned mb = __reduce_min_sync(FULL, bb);
        const unsigned mi = __reduce_min_sync(FULL, bb == mb ? bi : 0xffffffffu);
        if (lane == 0) {
            out[i] = (int)mi;
            if (outd) outd[i] = __uint_as_float(mb);
        }
        for (int s0 = 0; s0 < m; s0 += 32) {  // taken: out of every later minimum
            const int s2 = s0 + lane;
            unsigned id;
            if constexpr (TM) id = tm_ld(res.tid + (uint32_t)(s0 >> 5));
            else id = s2 < m ? (unsigned)rid[s2] : 0u;
            if (s2 < m && id == mi) rd[s2] = __uint_as_float(0xffffffffu);
        }
        __syncwarp();
    }
    for (int i = cnt + lane; i < a.k; i += 32) {
        out[i] = -1;
        if (outd) outd[i] = INFINITY;
    }
    return cnt;
}


// ------------------------------------------------------------ learned model

// Warp-resident MLP over warp-uniform inputs f[kFeat] with FP16 weights and
// FP32 accumulation: relu(W1 f + b1) -> relu(W2 h + b2) -> W3 h + b3.
// Lane l evaluates hidden units l and l + 32.  For n_out == 1 every lane
// returns the output; otherwise lane o < n_out (<= 32) returns output o.
__device__ __forceinline__ float mlp_warp(const __half* __restrict__ w, const float (&f)[kFeat],
                                          int n_out, int lane) {
    const __half* W1 = w;
    const __half* b1 = W1 + kHid * kFeat;
    const __half* W2 = b1 + kHid;
    const __half* b2 = W2 + kHid * kHid;
    const __half* W3 = b2 + kHid;
    const __half* b3 = W3 + n_out * kHid;
    float h0 = __half2float(b1[lane]), h1 = __half2float(b1[lane + 32]);
    const __half2* r0 = reinterpret_cast<const __half2*>(W1 + lane * kFeat);
    const __half2* r1 = reinterpret_cast<const __half2*>(W1 + (lane + 32) * kFeat);
#pragma unroll
    for (int i = 0; i < kFeat / 2; ++i) {
        const float2 a = __half22float2(r0[i]);
        const float2 b = __half22float2(r1[i]);
        h0 = fmaf(a.x, f[2 * i], h0);
        h0 = fmaf(a.y, f[2 * i + 1], h0);
        h1 = fmaf(b.x, f[2 * i], h1);
        h1 = fmaf(b.y, f[2 * i + 1], h1);
    }
    h0 = fmaxf(h0, 0.0f);
    h1 = fmaxf(h1, 0.0f);
    float g0 = __half2float(b2[lane]), g1 = __half2float(b2[lane + 32]);
    const __half2* s0 = reinterpret_cast<const __half2*>(W2 + lane * kHid);
    const __half2* s1 = reinterpret_cast<const __half2*>(W2 + (lane + 32) * kHid);
#pragma unroll 4
    for (int j = 0; j < 32; j += 2) {
        const float x0 = __shfl_sync(FULL, h0, j), x1 = __shfl_sync(FULL, h0, j + 1);
        const float y0 = __shfl_sync(FULL, h1, j), y1 = __shfl_sync(FULL, h1, j + 1);
        const float2 a = __half22float2(s0[j >> 1]), c = __half22float2(s0[(j + 32) >> 1]);
        const float2 b = __half22float2(s1[j >> 1]), e = __half22float2(s1[(j + 32) >> 1]);
        g0 = fmaf(a.x, x0, fmaf(a.y, x1, fmaf(c.x, y0, fmaf(c.y, y1, g0))));
        g1 = fmaf(b.x, x0, fmaf(b.y, x1, fmaf(e.x, y0, fmaf(e.y, y1, g1))));
    }
    g0 = fmaxf(g0, 0.0f);
    g1 = fmaxf(g1, 0.0f);
    if (n_out == 1) {
        float z = fmaf(__half2float(W3[lane]), g0, __half2float(W3[lane + 32]) * g1);
#pragma unroll
        for (int w2 = 16; w2 >= 1; w2 >>= 1) z += __shfl_xor_sync(FULL, z, w2);
        return z + __half2float(b3[0]);
    }
    const int o = lane < n_out ? lane : 0;
    const __half2* t3 = reinterpret_cast<const __half2*>(W3 + o * kHid);
    float z = __half2float(b3[o]);
#pragma unroll 4
    for (int j = 0; j < 32; j += 2) {
        const float x0 = __shfl_sync(FULL, g0, j), x1 = __shfl_sync(FULL, g0, j + 1);
        const float y0 = __shfl_sync(FULL, g1, j), y1 = __shfl_sync(FULL, g1, j + 1);
        const float2 a = __half22float2(t3[j >> 1]), c = __half22float2(t3[(j + 32) >> 1]);
        z = fmaf(a.x, x0, fmaf(a.y, x1, fmaf(c.x, y0, fmaf(c.y, y1, z))));
    }
    return z;
}

// Running statistics of a search for the learned stop.  kd: lane i < K holds
// the i-th smallest distance computed so far (+inf if fewer), which is the
// i-th entry of the results' top-K, since results only lose their maximum.
struct StopState {
    float kd, kth, best, kth_prev, entry_d;
    int K, hops_kth, hops_best, n_new, n_res, n_front, nck;
};

__device__ __forceinline__ void stop_init(StopState& s, int k) {
    s.kd = s.kth = s.best = s.kth_prev = s.entry_d = INFINITY;
    s.K = k < 1 ? 1 : (k > 32 ? 32 : k);
    s.hops_kth = s.hops_best = s.n_new = s.n_res = s.n_front = s.nck = 0;
}

// Insert the distances of the lanes in N into the sorted top-K (lane order).
__device__ __forceinline__ void topk_insert(StopState& s, unsigned N, float d, int lane) {
    const bool mine = (N >> lane) & 1u;
    unsigned ins = __ballot_sync(FULL, mine && d < s.kth);
    while (ins) {
        const int j = __ffs(ins) - 1;
        const float v = __shfl_sync(FULL, d, j);
        const int p = __popc(__ballot_sync(FULL, lane < s.K && s.kd <= v));
        const float up = __shfl_up_sync(FULL, s.kd, 1);
        if (lane < s.K && lane > p) s.kd = up;
        if (lane == p) s.kd = v;
        if (v < s.best) s.hops_best = 0;
        const float nk = __shfl_sync(FULL, s.kd, s.K - 1);
        if (nk != s.kth) s.hops_kth = 0;
        s.kth = nk;
        s.best = __shfl_sync(FULL, s.kd, 0);
        ins &= ~(1u << j);
        ins &= __ballot_sync(FULL, mine && d < s.kth);
    }
}

// The kFeat stop features (warp-uniform), all finite and roughly in [0, 1].
// cnt1/cnt11/cnt125: frontier candidates closer than 1x / 1.1x / 1.25x the
// k-th best distance (the ones that can still improve the top-k).
__device__ __forceinline__ void stop_features(float (&f)[kFeat], const StopState& s, int t,
                                              float cmin, float worst, bool res_full,
                                              float cand_fill, float res_fill, int cnt1,
                                              int cnt11, int cnt125, int window) {
    const bool kf = s.kth < INFINITY;
    const float kth = kf ? fmaxf(s.kth, 1e-30f) : 1.0f;
    const float best = s.best < INFINITY ? s.best : 0.0f;
    const float wnd = 1.0f / (float)window;
    f[0] = log1pf((float)t) * 0.125f;
    f[1] = kf ? fminf(cmin / kth, 4.0f) * 0.25f : 1.0f;
    f[2] = kf ? fminf(best / kth, 1.0f) : 0.0f;
    f[3] = (kf && s.kth_prev < INFINITY) ? fminf(s.kth / fmaxf(s.kth_prev, 1e-30f), 1.0f) : 1.0f;
    f[4] = fminf((float)s.hops_kth, 256.0f) * (1.0f / 64.0f);
    f[5] = fminf((float)s.hops_best, 256.0f) * (1.0f / 64.0f);
    f[6] = (res_full && kf) ? fminf(worst / kth, 8.0f) * 0.125f : 1.0f;
    f[7] = (float)s.n_res * wnd;
    f[8] = (float)s.n_new * wnd;
    f[9] = cand_fill;
    f[10] = res_fill;
    f[11] = kf ? fminf(logf(kth / fmaxf(best, 1e-30f)), 8.0f) * 0.125f : 1.0f;
    f[12] = log1pf((float)s.hops_kth) * (1.0f / 6.0f);
    f[13] = log1pf((float)s.hops_best) * (1.0f / 6.0f);
    f[14] = res_full ? fminf(cmin / fmaxf(worst, 1e-30f), 2.0f) * 0.5f : 0.0f;
    f[15] = fminf((float)cnt1, 16.0f) * (1.0f / 16.0f);
    f[16] = kf ? 1.0f : 0.0f;
    f[17] = log1pf(kf ? s.kth : 0.0f) * (1.0f / 16.0f);
    f[18] = fminf((float)cnt125, 64.0f) * (1.0f / 64.0f);
    f[19] = log1pf(cmin < INFINITY ? cmin : 0.0f) * (1.0f / 16.0f);
    f[20] = (float)s.n_front * wnd;
    f[21] = fminf((float)cnt11, 32.0f) * (1.0f / 32.0f);
    f[22] = (kf && s.entry_d < INFINITY) ? fminf(s.entry_d / kth, 64.0f) * (1.0f / 64.0f) : 1.0f;
    f[23] = 1.0f;
}

// Order-preserving unsigned key of a float (for redux over signed values).
__device__ __forceinline__ unsigned fkey(float x) {
    const unsigned b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// KIND 0 = L2 with NE query elements per lane (0: query in shared memory);
// KIND 1 = Hamming with NE uint4 of code per row.  GPL: queue groups per lane.
// DT: SONG_PREC_FP32 (the plain, bit-exact search) or the precision form on
// BF16 / FP8 rows (KIND 0, query in shared memory, FP32 re-rank at the end).
// LM: 0 plain; 1 learning traces; 2 learned entry and stop; 3 learned entry
// only (the instance for a stop model that cannot fire).
// TM = 1: the result ids live in this warp's TMEM lanes from column `tbase`
// (G = ceil(cap / 32) columns); TMC = 1: so do the candidate ids, in the G
// columns before them.  The per-warp shared-memory layout then has no id
// array for that queue.
// TR = 0: the per-query trace is not written (a.trace must be null), so its
// counters are dead code and free their registers.  TD = 1 (TM = TMC = 1):
// the results queue's distances in TMEM too.
template <int KIND, int NE, int GPL, int DT, int LM, int TM = 0, int TMC = TM, int TR = 1, int TD = 0>
__device__ __forceinline__ void search_query(const SearchArgs& a, int qid, unsigned char* ws,
                                             int lane, uint32_t tbase = 0) {
    static_assert(!TD || (TM && TMC), "distances in TMEM go with the ids in TMEM");
    Queue<GPL, TMC> cand;
    Queue<GPL, TM, TD> res;
    // this warp's TMEM columns: [candidate ids (TMC)] [result ids (TM)] [result distances (TD)]
    const uint32_t ngrp = (uint32_t)((a.cap + 31) >> 5);
    const uint32_t tres = tbase + (TMC ? ngrp : 0u);
    q_init(cand, reinterpret_cast<float*>(ws + a.cd_off), reinterpret_cast<int*>(ws + a.ci_off),
           tbase, 0u, a.cap);
    q_init(res, reinterpret_cast<float*>(ws + a.rd_off), reinterpret_cast<int*>(ws + a.ri_off),
           tres, tres + ngrp, a.cap);
    uint64_t* bloom = reinterpret_cast<uint64_t*>(ws + a.bl_off);
    float* sq = reinterpret_cast<float*>(ws + a.q_off);
    int* rows = reinterpret_cast<int*>(ws + a.rows_off);

    BloomCfg bc;
    bc.words = (uint32_t)a.bf_words;
    bc.nbits = (uint64_t)a.bf_words * 64ull;
    bc.shift = (a.bf_words & (a.bf_words - 1)) == 0 ? __ffs(a.bf_words) - 1 : -1;
    bc.wmask = (uint32_t)a.bf_words - 1u;
    bc.nhash = a.bf_nhash;

    // Query in registers (and shared memory for the generic L2 path).
    // NE < 0 (byte-row instances, an index with byte rows, dim <= 32 * 4 * -NE):
    // only the query's bytes stay in registers; a query that is not integral
    // in [0, 255] takes the generic exact path reading its floats from global
    // memory.  Fewer live registers let more queries reside per SM.
    constexpr bool kU8 = KIND == 0 && NE < 0;
    constexpr bool kIntPath = KIND == 0 && NE > 0 && DT == SONG_PREC_FP32;
    constexpr int kNC = kU8 ? -NE : (NE >= 8 ? 2 : 1);  // 16-byte query chunks per lane on the byte-row path
    float qreg[(KIND == 0 && NE > 0) ? NE : 1];
    float4 qv[kIntPath ? NE : 1];
    uint4 qb[(kIntPath || kU8) ? kNC : 1];
    const float* sqg = sq;  // the query for the generic path (global memory in byte-row instances)
    uint4 qcode[KIND == 1 ? NE : 1];
    bool int_exact = false, u8_mode = false;
    int qq = 0;
    if constexpr (KIND == 0) {
        const float* qg = reinterpret_cast<const float*>(a.queries) + (int64_t)qid * a.qld;
        if constexpr (NE > 0) {
            float lo = INFINITY, hi = -INFINITY;
            bool integral = true;
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                const int i = lane + 32 * e;
                qreg[e] = i < a.dim ? __ldcg(qg + i) : 0.0f;
                if (i < a.dim) {
                    lo = fminf(lo, qreg[e]);
                    hi = fmaxf(hi, qreg[e]);
                    integral &= qreg[e] == rintf(qreg[e]);
                }
            }
            if (a.int_base && (a.dim == 32 * NE || a.u8 != nullptr)) {
                // every |q_i - b_i| <= maxd; dim * maxd^2 < 2^24 keeps all sums exact
                integral = __all_sync(FULL, integral);
#pragma unroll
                for (int w = 16; w >= 1; w >>= 1) {
                    lo = fminf(lo, __shfl_xor_sync(FULL, lo, w));
                    hi = fmaxf(hi, __shfl_xor_sync(FULL, hi, w));
                }
                const double maxd = fmax((double)a.base_max - lo, (double)hi - a.base_min);
                int_exact = integral && (double)a.dim * maxd * maxd < 16777216.0;
                // byte rows (base in [0, 255]) and a query in [0, 255]: exact dp4a distances
                u8_mode = kIntPath && int_exact && a.u8 != nullptr && lo >= 0.0f && hi <= 255.0f;
                if (u8_mode) {
                    int s2 = 0;
#pragma unroll
                    for (int e = 0; e < NE; ++e) {
                        const int v = (int)qreg[e];  // zero beyond dim
                        s2 += v * v;
                    }
                    qq = (int)__reduce_add_sync(FULL, (unsigned)s2);
#pragma unroll
                    for (int c = 0; c < kNC; ++c) {  // lane t of 8: bytes 16(t + 8c) .. +15
                        const int e0 = 16 * ((lane & 7) + 8 * c);
                        unsigned w4[4];
#pragma unroll
                        for (int wd = 0; wd < 4; ++wd) {
                            unsigned wv = 0u;
#pragma unroll
                            for (int bt = 0; bt < 4; ++bt) {
                                const int e = e0 + 4 * wd + bt;
                                const unsigned bv = e < a.dim ? (unsigned)__ldcg(qg + e) : 0u;
                                wv |= bv << (8 * bt);
                            }
                            w4[wd] = wv;
                        }
                        qb[c] = make_uint4(w4[0], w4[1], w4[2], w4[3]);
                    }
                } else if (int_exact && a.dim != 32 * NE) {
                    int_exact = false;  // the float4 gather path needs dim == 32 * NE
                }
                if (int_exact && !u8_mode) {
                    const float4* q4 = reinterpret_cast<const float4*>(qg);
                    const bool aligned = ((reinterpret_cast<uintptr_t>(qg) & 15u) == 0);
#pragma unroll
                    for (int e = 0; e < NE; ++e) {
                        const int f = (lane & 7) + 8 * e;
                        qv[e] = aligned ? __ldcg(q4 + f)
                                        : make_float4(__ldcg(qg + 4 * f), __ldcg(qg + 4 * f + 1),
                                                      __ldcg(qg + 4 * f + 2), __ldcg(qg + 4 * f + 3));
                    }
                }
            }
        } else if constexpr (kU8) {
            qreg[0] = 0.0f;
            sqg = qg;
            float lo = INFINITY, hi = -INFINITY;
            bool integral = true;
            int s2 = 0;
            for (int i = lane; i < a.dim; i += 32) {
                const float v = __ldcg(qg + i);
                lo = fminf(lo, v);
                hi = fmaxf(hi, v);
                integral &= v == rintf(v);
                if (v >= 0.0f && v <= 255.0f) s2 += (int)v * (int)v;
            }
            integral = __all_sync(FULL, integral);
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(FULL, lo, w));
                hi = fmaxf(hi, __shfl_xor_sync(FULL, hi, w));
            }
            // byte rows hold a base in [0, 255]; a query there too makes every
            // partial sum an integer below 2^24 (dim <= 256): exact dp4a distances
            u8_mode = a.u8 != nullptr && integral && lo >= 0.0f && hi <= 255.0f;
            if (u8_mode) {
                qq = (int)__reduce_add_sync(FULL, (unsigned)s2);
#pragma unroll
                for (int c = 0; c < kNC; ++c) {  // lane t of 8: bytes 16(t + 8c) .. +15
                    const int e0 = 16 * ((lane & 7) + 8 * c);
                    unsigned w4[4];
#pragma unroll
                    for (int wd = 0; wd < 4; ++wd) {
                        unsigned wv = 0u;
#pragma unroll
                        for (int bt = 0; bt < 4; ++bt) {
                            const int e = e0 + 4 * wd + bt;
                            const unsigned bv = e < a.dim ? (unsigned)__ldcg(qg + e) : 0u;
                            wv |= bv << (8 * bt);
                        }
                        w4[wd] = wv;
                    }
                    qb[c] = make_uint4(w4[0], w4[1], w4[2], w4[3]);
                }
            }
        } else {
            qreg[0] = 0.0f;
            for (int i = lane; i < a.qdim; i += 32) sq[i] = i < a.dim ? __ldcg(qg + i) : 0.0f;
        }
    } else {
        const uint32_t* qg = reinterpret_cast<const uint32_t*>(a.queries) + (int64_t)qid * a.qld;
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            uint32_t w[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) w[t] = (4 * e + t) < a.dim ? __ldcg(qg + 4 * e + t) : 0u;
            qcode[e] = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    for (int w = lane; w < a.bf_words; w += 32) bloom[w] = 0ull;
    __syncwarp();

    auto distances = [&](int nb, unsigned N) -> float {
        float d;
        if constexpr (DT != SONG_PREC_FP32) {
            d = l2_lowp<DT>(a, sq, nb, N, rows, lane);
        } else if constexpr (KIND == 0) {
            const float* base = reinterpret_cast<const float*>(a.base);
            if constexpr (kIntPath) {
                if (u8_mode) d = l2_u8<kNC>(a.u8, a.u8_ld, a.u8_ld >> 4, qb, qq, nb, N, rows, lane);
                else if (int_exact) d = l2_int<NE>(base, a.ld, qv, nb, N, rows, lane);
                else d = l2_exact<NE>(base, a.ld, a.dim, qreg, sq, nb, N, lane);
            } else if constexpr (kU8) {
                if (u8_mode) d = l2_u8<kNC>(a.u8, a.u8_ld, a.u8_ld >> 4, qb, qq, nb, N, rows, lane);
                else d = l2_exact<0>(base, a.ld, a.dim, qreg, sqg, nb, N, lane);
            } else {
                d = l2_exact<NE>(base, a.ld, a.dim, qreg, sq, nb, N, lane);
            }
        } else {
            d = ham_lane<NE>(reinterpret_cast<const uint32_t*>(a.base), a.ld, a.dim, qcode, nb,
                             (N >> lane) & 1u);
        }
        return d;
    };

    // Learned entry: distances to the hub nodes are the entry features; the
    // entry model's top hubs replace the p*n/N_MULTIPROBE seeds.
    StopState ss;
    stop_init(ss, a.k);
    int seed_id = -1, n_seeds = a.n_multiprobe;
    const bool given_seeds = a.qseeds != nullptr;  // caller-chosen entry points per query
    if (given_seeds) {
        n_seeds = a.n_qseeds;
        seed_id = lane < n_seeds ? __ldg(a.qseeds + (int64_t)qid * a.n_qseeds + lane) : -1;
        if (seed_id >= a.n) {  // never read out of range
            atomicExch(a.err, 1);
            seed_id = -1;
        }
    }
    if constexpr (LM > 0) {
        if (a.ecand != nullptr && !given_seeds) {
            // entry stage: this query's kEntryK nearest hubs (nearest first) from the
            // tensor-core kernel; the entry model re-scores them, or without a model
            // the nearest N_MULTIPROBE become the entry points
            const int64_t eo = (int64_t)qid * kEntryK;
            const int hub = lane < kEntryK ? __ldg(a.ecand + eo + lane) : -1;
            const float hd = hub >= 0 ? __ldg(a.edist + eo + lane) : INFINITY;
            float dmin = hd;
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) dmin = fminf(dmin, __shfl_xor_sync(FULL, dmin, w));
            const float rel = hub >= 0 ? hd / fmaxf(dmin, 1e-30f) : 0.0f;
            const int valid = __popc(__ballot_sync(FULL, hub >= 0));
            n_seeds = a.n_multiprobe < valid ? a.n_multiprobe : valid;
            if (n_seeds > 32) n_seeds = 32;
            if (LM == 1 && a.tr_entry_feat != nullptr && lane < kFeat)
                a.tr_entry_feat[(int64_t)qid * kFeat + lane] = hub >= 0 ? fminf(rel, 64.0f) * (1.0f / 64.0f) : 1.0f;
            if (a.entry_w != nullptr) {
                float f[kFeat];
#pragma unroll
                for (int i = 0; i < kFeat; ++i) {
                    const float ri = __shfl_sync(FULL, rel, i);
                    const int hi = __shfl_sync(FULL, hub, i);
                    f[i] = hi >= 0 ? fminf(ri, 64.0f) * (1.0f / 64.0f) : 1.0f;
                }
                const float z = mlp_warp(a.entry_w, f, kEntryK, lane);
                bool used = false;
                for (int s2 = 0; s2 < n_seeds; ++s2) {  // candidates by decreasing score
                    const unsigned key = (hub >= 0 && !used) ? fkey(z) : 0u;
                    const unsigned mk = __reduce_max_sync(FULL, key);
                    const int win = __ffs(__ballot_sync(FULL, hub >= 0 && !used && key == mk)) - 1;
                    const int h = __shfl_sync(FULL, hub, win);
                    if (lane == s2) seed_id = h;
                    if (lane == win) used = true;
                }
            } else {
                seed_id = lane < n_seeds ? hub : -1;
            }
            if (n_seeds < 1) {  // no hub at all: the reference's entry points
                n_seeds = a.n_multiprobe;
                seed_id = -1;
            }
        } else if (a.n_hubs > 0 && !given_seeds) {
            const int hub = lane < a.n_hubs ? __ldg(a.hubs + lane) : -1;
            const unsigned HN = __ballot_sync(FULL, hub >= 0);
            const float hd = distances(hub, HN);
            float dmin = hub >= 0 ? hd : INFINITY;
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) dmin = fminf(dmin, __shfl_xor_sync(FULL, dmin, w));
            const float rel = hub >= 0 ? hd / fmaxf(dmin, 1e-30f) : 0.0f;
            float f[kFeat];
#pragma unroll
            for (int i = 0; i < kFeat; ++i) f[i] = fminf(__shfl_sync(FULL, rel, i), 64.0f) * (1.0f / 64.0f);
            if (LM == 1 && a.tr_entry_feat != nullptr && lane < kFeat)
                a.tr_entry_feat[(int64_t)qid * kFeat + lane] = lane < a.n_hubs ? fminf(rel, 64.0f) * (1.0f / 64.0f) : 0.0f;
            if (a.entry_w != nullptr) {
                const float z = mlp_warp(a.entry_w, f, a.n_hubs, lane);
                n_seeds = a.n_multiprobe < a.n_hubs ? a.n_multiprobe : a.n_hubs;
                if (n_seeds > 32) n_seeds = 32;
                bool used = false;
                for (int s2 = 0; s2 < n_seeds; ++s2) {  // hubs by decreasing score
                    const unsigned key = (hub >= 0 && !used) ? fkey(z) : 0u;
                    const unsigned mk = __reduce_max_sync(FULL, key);
                    const int win = __ffs(__ballot_sync(FULL, hub >= 0 && !used && key == mk)) - 1;
                    const int h = __shfl_sync(FULL, hub, win);
                    if (lane == s2) seed_id = h;
                    if (lane == win) used = true;
                }
            }
        }
    }

    song_query_trace tr = {};
    bool seeding = true;  // the first pass inserts the N_MULTIPROBE entry points
    for (;;) {
        int limit;
        const int32_t* arow = nullptr;
        // first chunk of each adjacency row; learned searches with beam > 1 expand up
        // to 3 more rows this step (BLOCK_SIZE <= 32: one chunk per row)
        int first = -1, first2 = -1, first3 = -1, first4 = -1;
        int nrows = 1;
        if (seeding) {
            limit = n_seeds;  // seeds p*n/N_MULTIPROBE (kernalGraph.h:214-231)
        } else {              // expansion (kernalGraph.h:233-289)
            if (cand.sz == 0) break;
            unsigned mb, mi;
            root_min(cand, mb, mi);
            const float cmin = __uint_as_float(mb);
            const int cn = q_pop<true>(cand, (int)mi, lane);
            limit = a.block_size;
            arow = a.adj + (int64_t)cn * a.block_size;
            if (lane < limit) first = __ldg(arow + lane);
            tr.expanded_nodes += 1;
            unsigned wb = 0xffffffffu, wi;
            if (res.sz == res.cap) {  // early stop: full and strictly worse than the worst
                if constexpr (LM == 0) root_max_c(res, wb, wi);  // cached: plain searches only
                else root_max(res, wb, wi);
                if (fbits(cmin) > wb) {
                    tr.early_stopped = 1;
                    break;
                }
            }
            if constexpr (LM > 0) {
                // Beam (learned searches only; not the reference's order): the next
                // best candidates are expanded in the same step while they would not
                // end the search, so their adjacency rows are fetched in one round trip.
                if (a.beam > 1 && a.block_size <= 32) {
                    for (int bb = 1; bb < a.beam && cand.sz > 0; ++bb) {
                        unsigned mb2, mi2;
                        root_min(cand, mb2, mi2);
                        if (res.sz == res.cap && mb2 > wb) break;
                        const int cn2 = q_pop<true>(cand, (int)mi2, lane);
                        const int f = lane < limit ? __ldg(a.adj + (int64_t)cn2 * a.block_size + lane) : -1;
                        if (bb == 1) first2 = f;
                        else if (bb == 2) first3 = f;
                        else first4 = f;
                        tr.expanded_nodes += 1;
                        nrows = bb + 1;
                    }
                }
            }
            if constexpr (LM == 1 || LM == 2) {  // learned-stop checkpoint
                ss.hops_kth += nrows;
                ss.hops_best += nrows;
                const int t = tr.expanded_nodes;
                // A checkpoint right after the k-th distance improved (hops_kth == 0 after the
                // increment below is impossible; 1 means "improved by the last expansion")
                // cannot be the converged state the model looks for: no evaluation then.
                const bool want = LM == 1 || (a.stop_w != nullptr && a.stop_thr < INFINITY &&
                                              t >= a.min_expansions && ss.kth < INFINITY &&
                                              ss.hops_kth > 1);
                if (t % a.ckpt_every < nrows) {  // a multiple of ckpt_every was reached
                    if (want) {
                        int c1 = 0, c11 = 0, c125 = 0;
                        const float k1 = ss.kth, k11 = ss.kth * 1.1f, k125 = ss.kth * 1.25f;
                        for (int s2 = lane; s2 < cand.sz; s2 += 32) {
                            const float v = cand.d[s2];
                            c1 += v < k1;
                            c11 += v < k11;
                            c125 += v < k125;
                        }
                        c1 = __reduce_add_sync(FULL, (unsigned)c1);
                        c11 = __reduce_add_sync(FULL, (unsigned)c11);
                        c125 = __reduce_add_sync(FULL, (unsigned)c125);
                        float f[kFeat];
                        stop_features(f, ss, t, cmin, __uint_as_float(wb), res.sz == res.cap,
                                      (float)cand.sz / (float)cand.cap, (float)res.sz / (float)res.cap,
                                      c1, c11, c125, a.ckpt_every * a.block_size);
                        if (LM == 1 && a.tr_feat != nullptr && ss.nck < a.max_ckpt) {
                            const int64_t row = (int64_t)qid * a.max_ckpt + ss.nck;
                            if (lane == 0) {
#pragma unroll
                                for (int i = 0; i < kFeat; ++i) a.tr_feat[row * kFeat + i] = f[i];
                                a.tr_kth[row] = ss.kth;
                            }
                            ss.nck += 1;
                        }
                        if (LM == 2) {
                            const float z = mlp_warp(a.stop_w, f, 1, lane);
                            if (z >= a.stop_thr) {
                                tr.early_stopped = 2;  // learned stop
                                break;
                            }
                        }
                    }
                    ss.kth_prev = ss.kth;
                    ss.n_new = ss.n_res = ss.n_front = 0;
                }
            }
            // The next pop is most often today's runner-up: warm its row in L2.  Learned
            // searches (short queues, rows mostly L2-resident) measured faster without it.
            if (LM == 0 && cand.sz > 0) {
                unsigned nb2, ni2;
                root_min(cand, nb2, ni2);
                const int nid = q_id(cand, (int)ni2);
                if (lane == 0) {
                    const int32_t* nrow = a.adj + (int64_t)nid * a.block_size;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(nrow));
                }
            }
        }
        for (int rr = 0; rr < nrows; ++rr)
        for (int c0 = 0; c0 < limit; c0 += 32) {
            const int j = c0 + lane;
            int nb = -1;
            if (j < limit) {
                if (seeding) {
                    nb = (given_seeds || (LM > 0 && seed_id >= 0)) ? seed_id
                                                  : (int)((unsigned long long)j * (unsigned long long)a.n /
                                                          (unsigned long long)a.n_multiprobe);
                } else if (rr == 0) {
                    nb = c0 == 0 ? first : __ldg(arow + j);
                } else {  // beam rows: one chunk each
                    nb = rr == 1 ? first2 : (rr == 2 ? first3 : first4);
                }
            }
            if (nb >= a.n) {  // impossible for a validated graph; never read out of range
                atomicExch(a.err, 1);
                nb = -1;
            }
            const unsigned N = bloom_chunk(bloom, nb, bc, lane);
            const float d = distances(nb, N);
            const int c = __popc(N);
            if (seeding) {
                tr.seed_count += c;
            } else {
                tr.neighbor_slots_scanned += min(32, limit - c0);
                tr.candidate_nodes += c;
            }
            tr.visited_nodes += c;
            tr.distance_evals += c;
            const int pf = q_push<true>(cand, N, d, nb, lane, rows);
            const int pr = q_push<false, LM == 0>(res, N, d, nb, lane, rows);
            tr.frontier_pushes += pf;
            tr.result_updates += pr;
            if constexpr (LM == 1 || LM == 2) {
                topk_insert(ss, N, d, lane);
                ss.n_new += c;
                ss.n_res += pr;
                ss.n_front += pf;
                if (seeding) {
                    float m = ((N >> lane) & 1u) ? d : INFINITY;
#pragma unroll
                    for (int w = 16; w >= 1; w >>= 1) m = fminf(m, __shfl_xor_sync(FULL, m, w));
                    ss.entry_d = fminf(ss.entry_d, m);
                }
            }
            if (N) {
                tr.peak_frontier = max(tr.peak_frontier, cand.sz);
                tr.peak_results = max(tr.peak_results, res.sz);
            }
        }
        seeding = false;
    }

    if constexpr (LM == 1) {
        if (lane == 0 && a.tr_count != nullptr) {
            a.tr_count[qid] = ss.nck;
            a.tr_final_kth[qid] = ss.kth;
        }
    }
    // a launch that may have started before the previous one on its stream
    // finished writes nothing until that launch is complete
    asm volatile("griddepcontrol.wait;" ::: "memory");
    float* outd = a.out_dist ? a.out_dist + (int64_t)qid * a.k : nullptr;
    if (DT != SONG_PREC_FP32 && a.rerank)
        tr.result_count = rerank_finish(a, res, cand, sq, a.out + (int64_t)qid * a.k, outd, lane);
    else
        tr.result_count = finish(res, cand, a.k, a.out + (int64_t)qid * a.k, outd, lane,
                                 reinterpret_cast<int*>(bloom));
    if (TR && a.trace != nullptr && lane == 0) a.trace[qid] = tr;
}

#include "song_serve_kernel.inc"

// Launch shape of a search_kernel instance.  Queues of up to 1024 slots run
// in CTAs of 4 warps with at most 96 registers per thread, so that 5 CTAs
// (20 warps) fit an SM.  The search is latency-bound and gains from every
// resident query, but not at the price of spills: capped at 80 registers (6
// CTAs) the plain and entry-only instances spilled 100-190 bytes and ran
// 16 % (plain) and 13 % (learned) slower.  The plain and precision searches
// (LM = 0, queues of hundreds of slots) keep their result ids in TMEM (TM),
// one warp per TMEM lane quarter, and their candidate ids (the hotter queue:
// every expansion pops it) in shared memory: at ef 512 with a 512-word Bloom
// filter that still fits 5 CTAs per SM, where both id arrays in shared
// memory would not (measured 4-5 % faster than both in TMEM, 11 % faster
// than both in shared memory).  Both placements are compiled; the launcher
// takes the candidate ids into TMEM too when shared memory would otherwise
// cost resident CTAs (large queues and Bloom filters).  Learned searches run short queues, whose ids fit
// shared memory without costing warps, and there an id access is one
// shared-memory load instead of a TMEM round trip (measured 11 % faster).
// The trace and learned-stop instances (LM = 1, 2: checkpoint features, a
// running top-k) still spilled at 96 registers; they get 128 (4 CTAs, 16
// warps), measured 13-16 % faster.  Larger queues keep the ids in shared
// memory, up to 8 warps per CTA.
template <int KIND, int NE, int GPL, int DT, int LM>
struct KernelShape {
    static constexpr int kTM = (GPL == 1 && LM == 0) ? 1 : 0;   // result ids in TMEM
    static constexpr int kThreads = GPL == 1 ? 128 : 256;
    // byte-row instances (NE < 0) hold fewer query registers: 80 per thread and 6 CTAs
    // (plain), 72 and 7 CTAs (learned entry without the stop model), 96 and 5 CTAs
    // (learned entry and stop)
    static constexpr int kMinBlocks =
        GPL == 1 ? (LM == 1 ? 4
                            : (LM == 2 ? (NE < 0 ? 5 : 4) : (NE < 0 ? (LM == 3 ? 7 : 6) : 5)))
                 : 1;
    // without the trace counters (TR = 0): one more CTA
    static constexpr int kMinBlocksNT = GPL == 1 && NE < 0 ? kMinBlocks + 1 : kMinBlocks;
    static constexpr bool kQuerySmem = KIND == 0 && NE == 0;  // query kept in shared memory
};

// TMC = 1 (TM instances only): the candidate ids in TMEM as well.  TR = 0:
// no per-query trace.  TD = 1 (with TMC = 1): the result distances in TMEM.
template <int KIND, int NE, int GPL, int DT, int LM = 0, int TMC = 0, int TR = 1, int TD = 0>
__global__ void __launch_bounds__((KernelShape<KIND, NE, GPL, DT, LM>::kThreads),
                                  (TR ? KernelShape<KIND, NE, GPL, DT, LM>::kMinBlocks
                                      : KernelShape<KIND, NE, GPL, DT, LM>::kMinBlocksNT))
    search_kernel(const SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int TM = KernelShape<KIND, NE, GPL, DT, LM>::kTM;
    static_assert(TM || !TMC, "candidate ids in TMEM need a TMEM allocation");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* ws = smem + (size_t)warp * a.warp_smem;
    uint32_t tbase = 0;
    __shared__ uint32_t tm_slot;
    if constexpr (TM) {  // one TMEM allocation per CTA, warp w uses lanes 32(w%4) .. +31
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                         :: "r"((uint32_t)__cvta_generic_to_shared(&tm_slot)), "r"(a.tm_cols)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tbase = tm_slot + ((uint32_t)(32 * (warp & 3)) << 16) +
                (uint32_t)((warp >> 2) * a.tm_warp_cols);
    }
    for (;;) {
        int qid = 0;
        if (lane == 0) qid = (int)atomicAdd(a.counter, 1u);
        qid = __shfl_sync(FULL, qid, 0);
        if (qid >= a.nq) break;
        search_query<KIND, NE, GPL, DT, LM, TM, TMC, TR, TD>(a, qid, ws, lane, tbase);
    }
    // Every query of this launch has been claimed: a search launched after
    // this one on the stream with programmatic serialization may start on
    // the resources this launch's tail leaves idle (it reads only the index
    // and its own queries, and waits for this launch before it writes).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if constexpr (TM) {  // every warp is done with TMEM before it is freed
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                         :: "r"(tm_slot), "r"(a.tm_cols) : "memory");
    }
    if (a.done != nullptr) {
        // The last CTA past its loop returns the work counter to zero for the
        // launch that takes this ring slot next, so no memset has to sit
        // between two launches on the stream.
        if constexpr (!TM) __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(a.done, 1u) == gridDim.x - 1) {
                atomicExch(a.counter, 0u);
                atomicExch(a.done, 0u);
            }
        }
    }
}

using KernelFn = void (*)(const SearchArgs);

// A chosen kernel instance and its launch shape.
struct KernelSel {
    KernelFn fn = nullptr;      // candidate ids in shared memory
    KernelFn fn_tmc = nullptr;  // tm only: the candidate ids in TMEM too
    KernelFn fn_nt = nullptr;   // byte-row instances: fn and fn_tmc without the trace
    KernelFn fn_tmc_nt = nullptr;
    KernelFn fn_tmd = nullptr;  // byte-row plain instances: result distances in TMEM too
    KernelFn fn_tmd_nt = nullptr;
    int tm = 0;                 // result ids in TMEM (the CTA allocates tensor memory)
    int threads = 256;
    bool query_smem = true;
};

template <int KIND, int NE, int GPL, int DT, int LM = 0>
KernelSel ksel() {
    using S = KernelShape<KIND, NE, GPL, DT, LM>;
    KernelSel k;
    k.fn = search_kernel<KIND, NE, GPL, DT, LM, 0>;
    if constexpr (S::kTM) k.fn_tmc = search_kernel<KIND, NE, GPL, DT, LM, 1>;
    if constexpr (NE < 0 && LM != 1) {  // trace-free copies of the hot instances
        k.fn_nt = search_kernel<KIND, NE, GPL, DT, LM, 0, 0>;
        if constexpr (S::kTM) {
            k.fn_tmc_nt = search_kernel<KIND, NE, GPL, DT, LM, 1, 0>;
            k.fn_tmd = search_kernel<KIND, NE, GPL, DT, LM, 1, 1, 1>;
            k.fn_tmd_nt = search_kernel<KIND, NE, GPL, DT, LM, 1, 0, 1>;
        }
    }
    k.tm = S::kTM;
    k.threads = S::kThreads;
    k.query_smem = S::kQuerySmem;
    return k;
}

template <int GPL>
KernelSel pick_gpl(int kind, const SearchArgs& a) {
    if (kind == SONG_KIND_L2) {
        if (a.prec == SONG_PREC_BF16) return ksel<0, 0, GPL, SONG_PREC_BF16>();
        if (a.prec == SONG_PREC_FP8) return ksel<0, 0, GPL, SONG_PREC_FP8>();
        if constexpr (GPL == 1) {  // an index with byte rows: the byte-row instances
            if (a.u8 != nullptr && a.dim <= 128) return ksel<0, -1, 1, 0>();
            if (a.u8 != nullptr && a.dim <= 256) return ksel<0, -2, 1, 0>();
        }
        if (a.dim <= 32) return ksel<0, 1, GPL, 0>();
        if (a.dim <= 64) return ksel<0, 2, GPL, 0>();
        if (a.dim <= 128) return ksel<0, 4, GPL, 0>();
        if (a.dim <= 256) return ksel<0, 8, GPL, 0>();
        return ksel<0, 0, GPL, 0>();
    }
    switch (a.ld) {
        case 4: return ksel<1, 1, GPL, 0>();
        case 8: return ksel<1, 2, GPL, 0>();
        case 16: return ksel<1, 4, GPL, 0>();
        case 32: return ksel<1, 8, GPL, 0>();
        default: return KernelSel();
    }
}

// FP32 rows of integers in [0, 255] -> byte rows, zero padded to out_ld bytes.
__global__ void rows_to_u8(const float* __restrict__ x, int64_t n, int dim, int ld,
                           uint8_t* __restrict__ out, int out_ld) {
    const int64_t r = blockIdx.x;
    if (r >= n) return;
    for (int i = threadIdx.x; i < out_ld; i += blockDim.x)
        out[r * out_ld + i] = i < dim ? (uint8_t)x[r * ld + i] : (uint8_t)0;
}

// FP32 -> BF16 (round to nearest even) rows, zero padded to out_ld bytes.
__global__ void quantize_bf16(const float* __restrict__ x, int64_t n, int dim, int ld,
                              unsigned short* __restrict__ out, int out_ld) {
    const int64_t r = blockIdx.x;
    if (r >= n) return;
    const int pd = out_ld / 2;
    for (int i = threadIdx.x; i < pd; i += blockDim.x) {
        const float v = i < dim ? x[r * ld + i] : 0.0f;
        out[r * pd + i] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
}

// FP32 -> FP8 e4m3 rows with scale amax/448 (448 = largest finite e4m3):
// x ~= scale * e4m3(x / scale); one warp per row.
__global__ void quantize_fp8(const float* __restrict__ x, int64_t n, int dim, int ld,
                             unsigned char* __restrict__ out, int out_ld,
                             float* __restrict__ scales) {
    const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    float amax = 0.0f;
    for (int i = lane; i < dim; i += 32) amax = fmaxf(amax, fabsf(x[r * ld + i]));
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) amax = fmaxf(amax, __shfl_xor_sync(FULL, amax, w));
    const float scale = amax > 0.0f ? amax / 448.0f : 1.0f;
    const float inv = 1.0f / scale;
    for (int i = lane; i < out_ld; i += 32) {
        const float v = i < dim ? x[r * ld + i] * inv : 0.0f;
        out[r * out_ld + i] = (unsigned char)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
    }
    if (lane == 0) scales[r] = scale;
}

template <int LM>
KernelSel pick_learned(const SearchArgs& a) {
    if (a.prec == SONG_PREC_BF16) return ksel<0, 0, 1, SONG_PREC_BF16, LM>();
    if (a.prec == SONG_PREC_FP8) return ksel<0, 0, 1, SONG_PREC_FP8, LM>();
    if (a.u8 != nullptr && a.dim <= 128) return ksel<0, -1, 1, 0, LM>();
    if (a.dim <= 128 && a.dim > 64) return ksel<0, 4, 1, 0, LM>();
    return ksel<0, 0, 1, 0, LM>();
}

KernelSel pick_kernel(int kind, const SearchArgs& a) {
    if (a.lm != 0) {  // learned entry/stop: L2, queues up to 1024 slots
        if (kind != SONG_KIND_L2 || a.cap > 1024) return KernelSel();
        if (a.lm == 1) return pick_learned<1>(a);
        // a stop model that can never fire (none, or threshold >= 1): the entry-only
        // instance, without the stop statistics -- the same results, less state
        if (a.stop_w == nullptr || !(a.stop_thr < INFINITY)) return pick_learned<3>(a);
        return pick_learned<2>(a);
    }
    if (a.cap <= 1024) return pick_gpl<1>(kind, a);
    if (a.cap <= 2048) return pick_gpl<2>(kind, a);
    if (a.cap <= 4096) return pick_gpl<4>(kind, a);
    return KernelSel();
}

// Resident CTAs per SM of a TMEM-id kernel.  The runtime's occupancy query
// reports a single CTA per SM for kernels that allocate tensor memory, yet
// several such CTAs run side by side when their registers, shared memory and
// TMEM columns fit, so the limit is computed from those resources: registers
// are allocated per warp in units of 8 per thread out of 16,384 per SM
// sub-partition (four per SM), shared memory per CTA includes the runtime's
// reservation, and each SM has 512 TMEM columns.  A CTA beyond what fits
// would only wait in tcgen05.alloc for an earlier one to finish.
cudaError_t tm_ctas_per_sm(KernelFn fn, int dev, int warps, size_t dyn_smem, int tm_cols, int* out) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    int smem_sm = 0, reserved = 0, regs_sm = 0, max_blocks = 0, max_threads = 0;
    e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_blocks, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_threads, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    if (e != cudaSuccess) return e;
    const size_t cta_smem = dyn_smem + fa.sharedSizeBytes + (size_t)reserved;
    const int by_smem = (int)((size_t)smem_sm / cta_smem);
    const int warp_regs = ((fa.numRegs + 7) / 8) * 8 * 32;
    const int warps_per_quarter = warp_regs > 0 ? (regs_sm / 4) / warp_regs : 64;
    const int by_regs = (warps_per_quarter * 4) / warps;
    const int by_threads = max_threads / (warps * 32);
    const int by_tmem = 512 / tm_cols;
    *out = std::min(std::min(std::min(by_smem, by_regs), std::min(by_threads, max_blocks)), by_tmem);
    return cudaSuccess;
}

// Per-warp shared memory of the TMEM-id kernels: [query if kept in shared
// memory][32-entry row list][candidate distances][candidate ids, unless they
// are in TMEM too][result distances][Bloom filter], the Bloom region being at
// least cap ints because finish() may keep the extracted slots there once
// the search is over.
void tm_layout(int query_floats, bool cand_in_tmem, bool res_d_in_tmem, SearchArgs* a) {
    const int capr = round_up(a->cap, 32);
    a->q_off = 0;
    a->rows_off = round_up(query_floats * 4, 16);
    // the row list doubles as the push stage: 32 ids, and 32 distances when
    // the result distances are in TMEM
    a->cd_off = a->rows_off + (res_d_in_tmem ? 256 : 128);
    int off = a->cd_off + capr * 4;
    a->ci_off = 0;
    if (!cand_in_tmem) {
        a->ci_off = off;
        off += capr * 4;
    }
    a->rd_off = 0;
    if (!res_d_in_tmem) {
        a->rd_off = off;
        off += capr * 4;
    }
    a->ri_off = 0;
    a->bl_off = round_up(off, 16);
    a->warp_smem = round_up(a->bl_off + std::max(a->bf_words * 8, capr * 4), 16);
    a->tm_warp_cols = ((cand_in_tmem ? 1 : 0) + 1 + (res_d_in_tmem ? 1 : 0)) * (capr / 32);
}

}  // namespace

int u8_row_bytes(int dim) { return round_up(dim, 16); }

cudaError_t convert_rows_u8(const float* d_rows, int64_t n, int dim, int ld, uint8_t* d_out,
                            int out_ld, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    rows_to_u8<<<(unsigned)n, 128, 0, st>>>(d_rows, n, dim, ld, d_out, out_ld);
    return cudaGetLastError();
}

int search_row_stride(int kind, int dim) {
    if (kind == SONG_KIND_L2) return round_up(dim, 4);
    if (dim <= 4) return 4;
    if (dim <= 8) return 8;
    if (dim <= 16) return 16;
    return 32;
}

int lowp_padded_dim(int prec, int dim) {
    const int unit = prec == SONG_PREC_BF16 ? 64 : 128;  // 8 lanes x 16 B per pass over a row
    return round_up(dim, unit);
}

cudaError_t quantize_rows(int prec, const float* d_rows, int64_t n, int dim, int ld, void* d_out,
                          int out_ld, float* d_scales, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (prec == SONG_PREC_BF16) {
        quantize_bf16<<<(unsigned)n, 128, 0, st>>>(d_rows, n, dim, ld,
                                                   static_cast<unsigned short*>(d_out), out_ld);
    } else if (prec == SONG_PREC_FP8) {
        quantize_fp8<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(
            d_rows, n, dim, ld, static_cast<unsigned char*>(d_out), out_ld, d_scales);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int search_warp_smem(int kind, int dim, int cap, int bf_words, SearchArgs* a) {
    (void)kind;
    const int capr = round_up(cap, 32);
    a->q_off = 0;
    a->rows_off = round_up(dim * 4, 16);
    a->cd_off = a->rows_off + 128;
    a->ci_off = a->cd_off + capr * 4;
    a->rd_off = a->ci_off + capr * 4;
    a->ri_off = a->rd_off + capr * 4;
    a->bl_off = round_up(a->ri_off + capr * 4, 16);
    a->warp_smem = round_up(a->bl_off + bf_words * 8, 16);
    return a->warp_smem;
}

cudaError_t launch_serve(const ServeArgs& s, int num_sms, int max_ctas, int reserve_sms,
                         cudaStream_t st, int* warps_out) {
    using ServeFn = void (*)(const ServeArgs);
    ServeFn fn;
    const SearchArgs& a = s.base;
    if (a.prec == SONG_PREC_BF16) fn = serve_kernel<0, SONG_PREC_BF16>;
    else if (a.prec == SONG_PREC_FP8) fn = serve_kernel<0, SONG_PREC_FP8>;
    else if (a.dim <= 128 && a.dim > 64) fn = serve_kernel<4, 0>;
    else fn = serve_kernel<0, 0>;
    int dev = 0, optin = 0, smem_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e != cudaSuccess) return e;
    int warps;
    size_t smem;
    if (reserve_sms > 0 && reserve_sms < num_sms) {
        // Leave reserve_sms SMs free for the batched entry stage: one CTA of up
        // to 16 warps per SM, its shared memory padded past half of the SM so
        // that no SM can hold two, on num_sms - reserve_sms SMs.
        warps = 16;
        while (warps > 1 && (size_t)warps * a.warp_smem > (size_t)optin) warps >>= 1;
        smem = std::max<size_t>((size_t)warps * a.warp_smem, (size_t)smem_sm / 2 + 1024);
        if (smem > (size_t)optin) return cudaErrorInvalidConfiguration;
    } else {
        warps = 8;
        while (warps > 1 && (size_t)warps * a.warp_smem > (size_t)optin / 4) warps >>= 1;
        smem = (size_t)warps * a.warp_smem;
        if (smem > (size_t)optin) return cudaErrorInvalidConfiguration;
    }
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int grid = per_sm * num_sms;
    if (reserve_sms > 0 && reserve_sms < num_sms) grid = num_sms - reserve_sms;  // per_sm is 1
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    fn<<<grid, warps * 32, smem, st>>>(s);
    if (warps_out) *warps_out = grid * warps;
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError();
}

cudaError_t launch_search(int kind, const SearchArgs& args, int num_sms, cudaStream_t stream) {
    if (args.nq <= 0) return cudaSuccess;
    KernelSel ks = pick_kernel(kind, args);
    if (ks.fn == nullptr) return cudaErrorInvalidValue;
    if (args.trace == nullptr && ks.fn_nt != nullptr) {
        ks.fn = ks.fn_nt;
        ks.fn_tmc = ks.fn_tmc_nt;
        ks.fn_tmd = ks.fn_tmd_nt;
    }
    KernelFn fn = ks.fn;
    SearchArgs a = args;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int smem_optin = 0;
    e = cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    int warps;
    int tm_per_sm = 0;
    if (ks.tm) {
        // ids in TMEM: CTAs of 4 warps, one per lane quarter; ceil(cap/32)
        // columns per warp and queue, allocated per CTA in a power of two >= 32.
        // The candidate ids go to shared memory unless that costs resident CTAs
        // (large queues and Bloom filters), then to TMEM as well.
        warps = ks.threads / 32;
        auto shape = [&](KernelFn f, bool cand_tm, bool res_d_tm, SearchArgs* s2, int* per_sm) -> cudaError_t {
            tm_layout(ks.query_smem ? s2->qdim : 0, cand_tm, res_d_tm, s2);
            int cols = 32;
            while (cols < s2->tm_warp_cols * (warps / 4)) cols <<= 1;
            s2->tm_cols = cols;
            *per_sm = 0;
            if (cols > 512 || (size_t)warps * s2->warp_smem > (size_t)smem_optin) return cudaSuccess;
            return tm_ctas_per_sm(f, dev, warps, (size_t)warps * s2->warp_smem, cols, per_sm);
        };
        // the layout with the most resident CTAs; on a tie the one with fewer
        // TMEM accesses (ids, then distances, in shared memory)
        SearchArgs a0 = a, a1 = a, a2 = a;
        int p0 = 0, p1 = 0, p2 = 0;
        e = shape(ks.fn, false, false, &a0, &p0);
        if (e == cudaSuccess) e = shape(ks.fn_tmc, true, false, &a1, &p1);
        if (e == cudaSuccess && ks.fn_tmd != nullptr) e = shape(ks.fn_tmd, true, true, &a2, &p2);
        if (e != cudaSuccess) return e;
        a = a0;
        tm_per_sm = p0;
        if (p1 > tm_per_sm) {
            a = a1;
            fn = ks.fn_tmc;
            tm_per_sm = p1;
        }
        if (p2 > tm_per_sm) {
            a = a2;
            fn = ks.fn_tmd;
            tm_per_sm = p2;
        }
        if (tm_per_sm < 1) return cudaErrorInvalidConfiguration;
    } else {
        // Up to 8 warps per CTA while the CTA's shared memory stays within a
        // quarter of the opt-in limit, so several CTAs can share an SM.
        warps = ks.threads / 32;
        while (warps > 1 && (size_t)warps * a.warp_smem > (size_t)smem_optin / 4) warps >>= 1;
    }
    const size_t smem = (size_t)warps * a.warp_smem;
    if (smem > (size_t)smem_optin) return cudaErrorInvalidConfiguration;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (ks.tm) {
        per_sm = tm_per_sm;
    } else {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, warps * 32, smem);
    }
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int64_t need = ((int64_t)a.nq + warps - 1) / warps;
    const int grid = (int)std::min<int64_t>((int64_t)per_sm * num_sms, need);
    // Plain searches (no learned stage, no caller seeds: nothing they read
    // can come from the launch before them) with a self-resetting counter
    // may overlap the previous search launch's tail on the same stream.
    const bool overlap = a.done != nullptr && a.lm == 0 && a.qseeds == nullptr;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)(warps * 32));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = overlap ? 1 : 0;
    e = cudaLaunchKernelEx(&cfg, fn, a);
    if (e != cudaSuccess) return e;
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError();
}

}  // namespace song
