// CPU restatement of the reference's GPU graph search -- the oracle.
//
// TEST INFRASTRUCTURE ONLY.  Tests, the smoke check and the CPU-baseline leg
// of bench.py call this library as a checker; the product never links it.
//
// It restates, sequentially and with the same arithmetic, what one query's
// 32-thread block computes in the reference:
//   * kg_search_kernel      kernalGraph.h:184-299  (L2, FP32)
//   * hkg_search_kernel     hashKernelGraph.h:238-352 (Hamming on u32 codes)
//   * warp_l2               kernalGraph.h:157-170  lane-strided FMA partial
//                           sums, then the shfl_down tree 16,8,4,2,1
//   * warp_hamming          hashKernelGraph.h:215-224
//   * Candidates / Results  gpuHeap.h:8-108 (unsorted slot arrays; first-index
//                           ties; swap-with-last removal)
//   * bf_hash/bf_set/bf_test bloomFilter.h:14-48
//   * the ef clamp of gpu_search kernalGraph.h:315-316
//   * QueryTrace counters   telemetry.h:5-18 updated as kernalGraph.h:222-297
// plus BitHash (bitHash.h:17-44) for the Hamming codes.
//
// Every compile-time constant of config.h is a runtime argument here.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <atomic>
#include <vector>
#include <queue>
#include <unordered_set>
#include <algorithm>
#include <utility>

namespace {

struct Trace {  // QueryTrace, telemetry.h:5-18 (same field order)
    int seed_count, visited_nodes, expanded_nodes, neighbor_slots_scanned, candidate_nodes,
        distance_evals, frontier_pushes, result_updates, peak_frontier, peak_results,
        result_count, early_stopped;
};
static_assert(sizeof(Trace) == 48, "trace layout");

// The eight 64-bit mixing constants of bloomFilter.h:14-19 (two per hash).
const uint64_t kBloomMix[8] = {
    0x4bcb391f924ed183ULL, 0xa0ab69ccd854fc0aULL, 0x91086b9cecf5e3b7ULL, 0xc68e01641bead407ULL,
    0x3a7b976128a30449ULL, 0x6d122efabfc4d99fULL, 0xe6700ef8715030e2ULL, 0x80dd0c3bffcfb45bULL,
};

// Bloom filter over bf_words 64-bit words (bloomFilter.h:23-48).
struct Bloom {
    std::vector<uint64_t> w;
    int nhash;
    Bloom(int words, int nh) : w(words, 0ULL), nhash(nh) {}
    int pos(int h, uint64_t x) const {  // bf_hash, bloomFilter.h:23-30
        x ^= x >> 33;
        x *= kBloomMix[h * 2];
        x ^= x >> 33;
        x *= kBloomMix[h * 2 + 1];
        x ^= x >> 33;
        return (int)(x % (uint64_t)(w.size() * 64));
    }
    void set(int x) {  // bf_set: word = pos % BF_WORDS, bit = pos / BF_WORDS
        const int nw = (int)w.size();
        for (int h = 0; h < nhash; ++h) {
            int p = pos(h, (uint64_t)x);
            w[p % nw] |= 1ULL << (p / nw);
        }
    }
    bool test(int x) const {  // bf_test: false as soon as one bit is clear
        const int nw = (int)w.size();
        for (int h = 0; h < nhash; ++h) {
            int p = pos(h, (uint64_t)x);
            if (!((w[p % nw] >> (p / nw)) & 1ULL)) return false;
        }
        return true;
    }
};

// Candidates<MAX> and Results<MAX> (gpuHeap.h:8-108) share one slot array
// model: capacity cap = clamp(ef, 1, MAX), append while sz < cap, otherwise
// replace the FIRST maximal slot (strict >) when the new distance is strictly
// smaller; removal moves the last slot into the hole.
struct SlotQueue {
    std::vector<float> d;
    std::vector<int> id;
    int sz = 0, cap = 1;
    void init(int cap_, int max_size) {
        sz = 0;
        cap = cap_ < 1 ? 1 : (cap_ > max_size ? max_size : cap_);
        d.assign(cap, 0.f);
        id.assign(cap, -1);
    }
    bool push(float dist, int node) {  // Candidates::push / Results::try_push
        if (sz < cap) { d[sz] = dist; id[sz] = node; ++sz; return true; }
        int fi = 0;
        for (int i = 1; i < cap; ++i) if (d[i] > d[fi]) fi = i;
        if (dist < d[fi]) { d[fi] = dist; id[fi] = node; return true; }
        return false;
    }
    int pop_min(float* out) {  // Candidates::pop_min
        int mi = 0;
        for (int i = 1; i < sz; ++i) if (d[i] < d[mi]) mi = i;
        *out = d[mi];
        int node = id[mi];
        d[mi] = d[sz - 1]; id[mi] = id[sz - 1]; --sz;
        return node;
    }
    float worst() const {  // Results::worst
        float m = d[0];
        for (int i = 1; i < sz; ++i) if (d[i] > m) m = d[i];
        return m;
    }
    void pop_worst() {  // Results::pop_worst
        int wi = 0;
        for (int i = 1; i < sz; ++i) if (d[i] > d[wi]) wi = i;
        d[wi] = d[sz - 1]; id[wi] = id[sz - 1]; --sz;
    }
    int drain_best(int32_t* out, int k) {  // Results::drain_best
        int count = sz < k ? sz : k;
        for (int i = 0; i < count; ++i) {
            int mi = 0;
            for (int j = 1; j < sz; ++j) if (d[j] < d[mi]) mi = j;
            out[i] = id[mi];
            d[mi] = d[sz - 1]; id[mi] = id[sz - 1]; --sz;
        }
        return count;
    }
};

// warp_l2 (kernalGraph.h:157-170): lane l accumulates (q[i]-b[i])^2 for
// i = l, l+32, ... with a fused multiply-add (nvcc contracts sum += d*d), then
// __shfl_down_sync with offsets 16,8,4,2,1 leaves lane 0 with the total.
float warp_l2(const float* q, const float* b, int dim) {
    float part[32];
    for (int l = 0; l < 32; ++l) {
        float s = 0.0f;
        for (int i = l; i < dim; i += 32) {
            float t = q[i] - b[i];
            s = std::fmaf(t, t, s);
        }
        part[l] = s;
    }
    for (int off = 16; off >= 1; off >>= 1)
        for (int l = 0; l < off; ++l) part[l] = part[l] + part[l + off];
    return part[0];
}

// warp_hamming (hashKernelGraph.h:215-224): integer popcount sum, as float.
float hamming(const uint32_t* q, const uint32_t* b, int words) {
    int s = 0;
    for (int i = 0; i < words; ++i) s += __builtin_popcount(q[i] ^ b[i]);
    return (float)s;
}

struct Args {
    const void* base;       // float[n*dim] or uint32[n*words]
    int64_t n;
    int dim;                // floats per row (L2) or u32 words per row (Hamming)
    bool is_hamming;
    const int32_t* adj;     // [n * block_size]
    int block_size;
    int k, ef, pq_size, bf_words, bf_nhash, n_multiprobe;
};

// One query of kg_search_kernel / hkg_search_kernel (kernalGraph.h:184-299).
void search_one(const Args& a, const void* query, int32_t* out, Trace* tr_out) {
    Trace tr{};
    SlotQueue cand, res;
    cand.init(a.ef, a.pq_size);
    res.init(a.ef, a.pq_size);
    Bloom bloom(a.bf_words, a.bf_nhash);
    auto dist = [&](int64_t node) -> float {
        if (a.is_hamming) {
            const uint32_t* b = (const uint32_t*)a.base + node * a.dim;
            return hamming((const uint32_t*)query, b, a.dim);
        }
        const float* b = (const float*)a.base + node * a.dim;
        return warp_l2((const float*)query, b, a.dim);
    };

    // Seeds: ep = p*n/N_MULTIPROBE as a 64-bit product (kernalGraph.h:214-231).
    for (int p = 0; p < a.n_multiprobe; ++p) {
        int ep = (int)((uint64_t)p * (uint64_t)a.n / (uint64_t)a.n_multiprobe);
        float dp = dist(ep);
        if (!bloom.test(ep)) {
            bloom.set(ep);
            bool fa = cand.push(dp, ep);
            bool ra = res.push(dp, ep);
            tr.seed_count++; tr.visited_nodes++; tr.distance_evals++;
            tr.frontier_pushes += fa; tr.result_updates += ra;
            if (tr.peak_frontier < cand.sz) tr.peak_frontier = cand.sz;
            if (tr.peak_results < res.sz) tr.peak_results = res.sz;
        }
    }

    for (;;) {  // expansion loop, kernalGraph.h:233-289
        if (cand.sz == 0) break;
        float c_min;
        int cn = cand.pop_min(&c_min);
        tr.expanded_nodes++;
        if (res.sz == res.cap && c_min > res.worst()) {  // early stop, strict >
            tr.early_stopped = 1;
            break;
        }
        const int32_t* row = a.adj + (int64_t)cn * a.block_size;
        for (int j = 0; j < a.block_size; ++j) {
            tr.neighbor_slots_scanned++;
            int nb = row[j];
            if (nb < 0) continue;  // empty slot: continue, not break
            if (bloom.test(nb)) continue;
            bloom.set(nb);
            tr.visited_nodes++; tr.candidate_nodes++;
            float d = dist(nb);
            tr.distance_evals++;
            bool fa = cand.push(d, nb);
            bool ra = res.push(d, nb);
            tr.frontier_pushes += fa; tr.result_updates += ra;
            if (tr.peak_frontier < cand.sz) tr.peak_frontier = cand.sz;
            if (tr.peak_results < res.sz) tr.peak_results = res.sz;
        }
    }

    // Trim to k with pop_worst, write best-first, pad with -1 (:292-296).
    while (res.sz > a.k) res.pop_worst();
    int cnt = res.drain_best(out, a.k);
    for (int i = cnt; i < a.k; ++i) out[i] = -1;
    tr.result_count = cnt;
    if (tr_out) *tr_out = tr;
}

int run(const Args& a, const void* queries, int nq, int32_t* ids, int32_t* trace, int nthreads) {
    if (a.n <= 0 || a.dim <= 0 || a.block_size <= 0 || nq < 0 || a.k < 0) return -1;
    if (a.bf_words <= 0 || a.bf_nhash < 1 || a.bf_nhash > 4 || a.n_multiprobe < 1) return -1;
    const size_t qstride = (size_t)a.dim * (a.is_hamming ? sizeof(uint32_t) : sizeof(float));
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= nq) break;
            search_one(a, (const char*)queries + (size_t)i * qstride, ids + (size_t)i * a.k,
                       trace ? (Trace*)(trace + (size_t)i * 12) : nullptr);
        }
    };
    if (nthreads <= 1) {
        work();
    } else {
        std::vector<std::thread> ts;
        for (int t = 0; t < nthreads; ++t) ts.emplace_back(work);
        for (auto& t : ts) t.join();
    }
    return 0;
}

}  // namespace

extern "C" {

// The ef clamp of gpu_search (kernalGraph.h:315-316): raise to k first,
// then cap at pq_size, so k > pq_size yields ef = pq_size.
int oracle_clamp_ef(int ef, int k, int pq_size) {
    if (ef < k) ef = k;
    if (ef > pq_size) ef = pq_size;
    return ef;
}

float oracle_warp_l2(const float* q, const float* b, int dim) { return warp_l2(q, b, dim); }

// kg_search_kernel over nq queries. `ef` is the value the kernel receives
// (already clamped by the caller, as gpu_search does).  ids[nq*k] best-first,
// -1 padded; trace[nq*12] nullable.
int oracle_search_l2(const float* data, int64_t n, int dim, const int32_t* adj, int block_size,
                     const float* queries, int nq, int k, int ef, int pq_size, int bf_words,
                     int bf_nhash, int n_multiprobe, int32_t* ids, int32_t* trace, int nthreads) {
    Args a{data, n, dim, false, adj, block_size, k, ef, pq_size, bf_words, bf_nhash, n_multiprobe};
    return run(a, queries, nq, ids, trace, nthreads);
}

// hkg_search_kernel over nq queries of `words` u32 code words each.
int oracle_search_hamming(const uint32_t* codes, int64_t n, int words, const int32_t* adj,
                          int block_size, const uint32_t* queries, int nq, int k, int ef,
                          int pq_size, int bf_words, int bf_nhash, int n_multiprobe, int32_t* ids,
                          int32_t* trace, int nthreads) {
    Args a{codes, n, words, true, adj, block_size, k, ef, pq_size, bf_words, bf_nhash, n_multiprobe};
    return run(a, queries, nq, ids, trace, nthreads);
}

// Graph::search (graph.h:33-115), restated: exact visited set, min-heap
// frontier and max-heap top-ef of (distance, id) pairs, l2 summed in
// dimension order (distance.h:5-12), seeds p*n/N_MULTIPROBE, results
// worst-first.  ids[nq*k] (-1 padded) and trace[nq*12].
void oracle_graph_search(const float* base, int64_t n, int dim, const int32_t* adj,
                         int block_size, const float* queries, int nq, int k, int ef,
                         int n_multiprobe, int32_t* ids, int32_t* trace) {
    using P = std::pair<float, int>;
    if (ef < k) ef = k;  // graph.h:36
    for (int qi = 0; qi < nq; ++qi) {
        const float* q = queries + (size_t)qi * dim;
        auto l2 = [&](int v) {  // distance.h:5-12
            const float* b = base + (size_t)v * dim;
            float s = 0.0f;
            for (int i = 0; i < dim; ++i) {
                float d = q[i] - b[i];
                float dd = d * d;
                s = s + dd;
            }
            return s;
        };
        Trace t{};
        std::priority_queue<P, std::vector<P>, std::greater<P>> fr;
        std::priority_queue<P> topk;
        std::unordered_set<int> visited;
        for (int p = 0; p < n_multiprobe; ++p) {  // graph.h:47-62
            const int ep = (int)((uint64_t)p * (uint64_t)n / (uint64_t)n_multiprobe);
            if (visited.count(ep)) continue;
            const float d = l2(ep);
            fr.push({d, ep});
            topk.push({d, ep});
            visited.insert(ep);
            t.seed_count++; t.visited_nodes++; t.distance_evals++;
            t.frontier_pushes++; t.result_updates++;
            t.peak_frontier = std::max(t.peak_frontier, (int)fr.size());
            t.peak_results = std::max(t.peak_results, (int)topk.size());
        }
        while (!fr.empty()) {  // graph.h:64-104
            const P cur = fr.top();
            fr.pop();
            t.expanded_nodes++;
            if ((int)topk.size() == ef && cur.first > topk.top().first) {
                t.early_stopped = 1;
                break;
            }
            std::vector<int> cands;
            for (int j = 0; j < block_size; ++j) {
                t.neighbor_slots_scanned++;
                const int v = adj[(size_t)cur.second * block_size + j];
                if (v < 0 || visited.count(v)) continue;
                visited.insert(v);
                cands.push_back(v);
                t.visited_nodes++; t.candidate_nodes++;
            }
            std::vector<float> dists(cands.size());
            for (size_t i = 0; i < cands.size(); ++i) { dists[i] = l2(cands[i]); t.distance_evals++; }
            for (size_t i = 0; i < cands.size(); ++i) {
                fr.push({dists[i], cands[i]});
                t.frontier_pushes++;
                t.peak_frontier = std::max(t.peak_frontier, (int)fr.size());
                if ((int)topk.size() < ef || dists[i] < topk.top().first) {
                    topk.push({dists[i], cands[i]});
                    if ((int)topk.size() > ef) topk.pop();
                    t.result_updates++;
                    t.peak_results = std::max(t.peak_results, (int)topk.size());
                }
            }
        }
        while ((int)topk.size() > k) topk.pop();  // graph.h:106-112
        int c = 0;
        while (!topk.empty()) { ids[(size_t)qi * k + c++] = topk.top().second; topk.pop(); }
        t.result_count = c;
        for (int i = c; i < k; ++i) ids[(size_t)qi * k + i] = -1;
        std::memcpy(trace + (size_t)qi * 12, &t, sizeof t);
    }
}

// BitHash(dim, seed) (bitHash.h:23-27): R[hash_bits x dim] from std::mt19937
// and std::normal_distribution<float>(0,1), filled row-major.
void oracle_bithash_matrix(int dim, int hash_bits, unsigned seed, float* R) {
    std::mt19937 rng(seed);
    std::normal_distribution<float> gauss(0.0f, 1.0f);
    for (size_t i = 0; i < (size_t)hash_bits * dim; ++i) R[i] = gauss(rng);
}

// BitHash::project (bitHash.h:32-44): bit b of word w is (R[w*32+b] . x > 0)
// with a sequential FP32 dot (separate multiply and add).
void oracle_bithash_project(const float* R, int dim, int hash_bits, const float* x, int64_t n,
                            uint32_t* out) {
    const int words = hash_bits / 32;
    for (int64_t v = 0; v < n; ++v) {
        const float* xv = x + v * dim;
        for (int w = 0; w < words; ++w) {
            uint32_t word = 0;
            for (int b = 0; b < 32; ++b) {
                const float* r = R + (size_t)(w * 32 + b) * dim;
                float dot = 0.0f;  // built with -ffp-contract=off: multiply, then add
                for (int d = 0; d < dim; ++d) {
                    float p = r[d] * xv[d];
                    dot = dot + p;
                }
                if (dot > 0) word |= 1u << b;
            }
            out[v * words + w] = word;
        }
    }
}

}  // extern "C"
