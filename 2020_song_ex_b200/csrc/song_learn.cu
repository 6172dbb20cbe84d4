// song_learn.cu -- training of the learned entry and stop models on the GPU.
//
// Two MLPs of the same shape (kFeat = 24 inputs, two ReLU layers of kHid =
// 64, FP32 master weights, FP16 copies for the warp-resident inference in
// the search kernel):
//  * entry model: inputs are the query's distances to the hub nodes
//    (relative to the nearest hub); output one logit per hub; trained with
//    softmax cross-entropy on the hub closest to the query's exact nearest
//    neighbour.  Its top-scoring hubs become the search's entry points.
//  * stop model: inputs are running statistics of one search at a
//    checkpoint (k-th and best distance, the candidate being expanded, hops
//    without improvement, update rates; see stop_features in
//    song_search.cu); output one logit; trained with binary cross-entropy
//    on "the k-th best distance at this checkpoint already equals the
//    k-th best distance of the full-budget search" -- since results only
//    improve, that means the top-k found so far is final.
// Training data are traces of the plain full-budget search (the search
// kernel in trace mode); every kernel here is the project's own.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "song_b200.h"
#include "song_kernels.cuh"

namespace song {

namespace {

constexpr int kLossBCE = 0;  // binary cross-entropy with logits, target in [0,1]
constexpr int kLossCE = 1;   // softmax cross-entropy, target = class index

// Offsets of the packed parameter layout (song_kernels.cuh).
struct Layout {
    int w1, b1, w2, b2, w3, b3, total, out;
    __host__ __device__ explicit Layout(int o) : out(o) {
        w1 = 0;
        b1 = w1 + kHid * kFeat;
        w2 = b1 + kHid;
        b2 = w2 + kHid * kHid;
        w3 = b2 + kHid;
        b3 = w3 + o * kHid;
        total = b3 + o;
    }
};

// Per-sample forward pass, loss and backward pass through the activations.
// Writes the layer inputs/outputs and deltas needed for the weight
// gradients: H1, H2 (post-ReLU), D1, D2 (pre-activation deltas), DZ (output
// deltas, already divided by the batch weight) and the per-sample loss.
// One thread per sample; parameters staged in shared memory.
__global__ void mlp_fwd_bwd(const float* __restrict__ P, int out, int loss_kind,
                            const float* __restrict__ X, const float* __restrict__ Y,
                            const float* __restrict__ SW, int B, float inv_norm,
                            float* __restrict__ H1, float* __restrict__ H2, float* __restrict__ D1,
                            float* __restrict__ D2, float* __restrict__ DZ, float* __restrict__ L) {
    extern __shared__ float sp[];
    const Layout ly(out);
    for (int i = threadIdx.x; i < ly.total; i += blockDim.x) sp[i] = P[i];
    __syncthreads();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float* x = X + (size_t)b * kFeat;
    float xi[kFeat];
#pragma unroll
    for (int i = 0; i < kFeat; ++i) xi[i] = x[i];
    float h1[kHid], h2[kHid];
    for (int u = 0; u < kHid; ++u) {
        float acc = sp[ly.b1 + u];
#pragma unroll
        for (int i = 0; i < kFeat; ++i) acc = fmaf(sp[ly.w1 + u * kFeat + i], xi[i], acc);
        h1[u] = fmaxf(acc, 0.0f);
    }
    for (int u = 0; u < kHid; ++u) {
        float acc = sp[ly.b2 + u];
        for (int j = 0; j < kHid; ++j) acc = fmaf(sp[ly.w2 + u * kHid + j], h1[j], acc);
        h2[u] = fmaxf(acc, 0.0f);
    }
    const float sw = SW ? SW[b] : 1.0f;
    float dz[64];
    float loss = 0.0f;
    if (loss_kind == kLossBCE) {
        float z = sp[ly.b3];
        for (int j = 0; j < kHid; ++j) z = fmaf(sp[ly.w3 + j], h2[j], z);
        const float y = Y[b];
        // softplus(z) - y z, stable form
        loss = fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)));
        const float p = 1.0f / (1.0f + expf(-z));
        dz[0] = (p - y) * sw * inv_norm;
    } else {
        float z[64];
        float zm = -INFINITY;
        for (int o = 0; o < out; ++o) {
            float acc = sp[ly.b3 + o];
            for (int j = 0; j < kHid; ++j) acc = fmaf(sp[ly.w3 + o * kHid + j], h2[j], acc);
            z[o] = acc;
            zm = fmaxf(zm, acc);
        }
        float se = 0.0f;
        for (int o = 0; o < out; ++o) se += expf(z[o] - zm);
        const int y = (int)Y[b];
        loss = logf(se) + zm - z[y];
        for (int o = 0; o < out; ++o) {
            const float p = expf(z[o] - zm) / se;
            dz[o] = (p - (o == y ? 1.0f : 0.0f)) * sw * inv_norm;
        }
    }
    L[b] = loss * sw;
    float d2[kHid];
    for (int j = 0; j < kHid; ++j) {
        float acc = 0.0f;
        for (int o = 0; o < out; ++o) acc = fmaf(sp[ly.w3 + o * kHid + j], dz[o], acc);
        d2[j] = h2[j] > 0.0f ? acc : 0.0f;
    }
    for (int i = 0; i < kHid; ++i) {
        float acc = 0.0f;
        for (int u = 0; u < kHid; ++u) acc = fmaf(sp[ly.w2 + u * kHid + i], d2[u], acc);
        D1[(size_t)b * kHid + i] = h1[i] > 0.0f ? acc : 0.0f;
        H1[(size_t)b * kHid + i] = h1[i];
        H2[(size_t)b * kHid + i] = h2[i];
        D2[(size_t)b * kHid + i] = d2[i];
    }
    for (int o = 0; o < out; ++o) DZ[(size_t)b * out + o] = dz[o];
}

// G[o][i] = sum_b D[b][o] * A[b][i] (i < n_in) and G[o][n_in] = sum_b D[b][o]
// (bias), written into the gradient layout at w (weights) and bias.
// One block per output unit o; threads over the inputs.
__global__ void weight_grad(const float* __restrict__ D, int n_out, const float* __restrict__ A,
                            int n_in, int B, float* __restrict__ gw, float* __restrict__ gb) {
    const int o = blockIdx.x;
    for (int i = threadIdx.x; i <= n_in; i += blockDim.x) {
        float acc = 0.0f;
        if (i < n_in) {
            for (int b = 0; b < B; ++b) acc = fmaf(D[(size_t)b * n_out + o], A[(size_t)b * n_in + i], acc);
            gw[o * n_in + i] = acc;
        } else {
            for (int b = 0; b < B; ++b) acc += D[(size_t)b * n_out + o];
            gb[o] = acc;
        }
    }
}

__global__ void adam_step(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                          float* __restrict__ V, int n, float lr, float b1, float b2, float eps,
                          float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.0f - b1) * g;
    const float v = b2 * V[i] + (1.0f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void to_half(const float* __restrict__ P, __half* __restrict__ H, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) H[i] = __float2half_rn(P[i]);
}

// Minibatch gather: row r of (Xs, Ys, Ws) = sample idx(r), idx from a hash.
__global__ void gather_batch(const float* __restrict__ X, const float* __restrict__ Y,
                             const float* __restrict__ W, int64_t M, int B, uint64_t salt,
                             float* __restrict__ Xb, float* __restrict__ Yb,
                             float* __restrict__ Wb) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    uint64_t h = salt ^ (0x9e3779b97f4a7c15ull * (uint64_t)(r + 1));
    h ^= h >> 31;
    h *= 0xbf58476d1ce4e5b9ull;
    h ^= h >> 29;
    const int64_t s = (int64_t)(h % (uint64_t)M);
#pragma unroll
    for (int i = 0; i < kFeat; ++i) Xb[(size_t)r * kFeat + i] = X[s * kFeat + i];
    Yb[r] = Y[s];
    Wb[r] = W ? W[s] : 1.0f;
}

// Stop-model samples from the trace buffers: one per written checkpoint,
// target 1 when the checkpoint's k-th distance equals the final one.
__global__ void stop_samples(const float* __restrict__ feat, const float* __restrict__ kth,
                             const int* __restrict__ count, const float* __restrict__ fin,
                             const int64_t* __restrict__ offs, int nq, int maxc,
                             float* __restrict__ X, float* __restrict__ Y) {
    const int q = blockIdx.x;
    if (q >= nq) return;
    const int c = count[q];
    const int64_t o = offs[q];
    for (int t = threadIdx.x; t < c * kFeat; t += blockDim.x) {
        const int r = t / kFeat, i = t % kFeat;
        X[(o + r) * kFeat + i] = feat[((int64_t)q * maxc + r) * kFeat + i];
    }
    for (int r = threadIdx.x; r < c; r += blockDim.x)
        Y[o + r] = kth[(int64_t)q * maxc + r] == fin[q] ? 1.0f : 0.0f;
}

// Entry labels: the hub closest to the query's exact nearest neighbour
// (first index on ties).  One warp per query.
__global__ void entry_labels(const float* __restrict__ base, int ld, int dim,
                             const int32_t* __restrict__ hubs, int n_hubs,
                             const int32_t* __restrict__ nn1, int nq, float* __restrict__ Y) {
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= nq) return;
    const float* a = base + (size_t)nn1[q] * ld;
    float best = INFINITY;
    int arg = 0;
    for (int h = 0; h < n_hubs; ++h) {
        const float* b = base + (size_t)hubs[h] * ld;
        float s = 0.0f;
        for (int i = lane; i < dim; i += 32) {
            const float t = a[i] - b[i];
            s = fmaf(t, t, s);
        }
#pragma unroll
        for (int w = 16; w >= 1; w >>= 1) s += __shfl_xor_sync(0xffffffffu, s, w);
        if (s < best) {
            best = s;
            arg = h;
        }
    }
    if (lane == 0) Y[q] = (float)arg;
}

// Entry labels when the entry stage supplies each query's kEntryK candidate
// hubs: the candidate closest to the query's exact nearest neighbour (first
// on ties; missing candidates never win).  One warp per query, lane j =
// candidate j.
__global__ void entry_labels_staged(const float* __restrict__ base, int ld, int dim,
                                    const int32_t* __restrict__ cand,
                                    const int32_t* __restrict__ nn1, int nq,
                                    float* __restrict__ Y) {
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= nq) return;
    const int c = lane < kEntryK ? cand[(size_t)q * kEntryK + lane] : -1;
    float s = INFINITY;
    if (c >= 0) {
        const float* a = base + (size_t)nn1[q] * ld;
        const float* b = base + (size_t)c * ld;
        s = 0.0f;
        for (int i = 0; i < dim; ++i) {
            const float t = a[i] - b[i];
            s = fmaf(t, t, s);
        }
    }
    float best = s;
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, w));
    const unsigned win = __ballot_sync(0xffffffffu, c >= 0 && s == best);
    if (lane == 0) Y[q] = win ? (float)(__ffs(win) - 1) : 0.0f;
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, std::max<size_t>(1, count) * sizeof(T));
}

// Adam training of one MLP on samples (X [M x kFeat], Y [M], W [M] nullable).
struct TrainResult {
    double loss_first = 0, loss_last = 0;
};

cudaError_t train_mlp(float* d_P, int out, int loss_kind, const float* X, const float* Y,
                      const float* W, int64_t M, int steps, int batch, float lr, uint64_t seed,
                      cudaStream_t st, TrainResult* res) {
    const Layout ly(out);
    const int B = (int)std::min<int64_t>(batch, M);
    float *G, *Mm, *Vv, *Xb, *Yb, *Wb, *H1, *H2, *D1, *D2, *DZ, *L;
    cudaError_t e = cudaSuccess;
    if ((e = dalloc(&G, ly.total)) || (e = dalloc(&Mm, ly.total)) || (e = dalloc(&Vv, ly.total)) ||
        (e = dalloc(&Xb, (size_t)B * kFeat)) || (e = dalloc(&Yb, B)) || (e = dalloc(&Wb, B)) ||
        (e = dalloc(&H1, (size_t)B * kHid)) || (e = dalloc(&H2, (size_t)B * kHid)) ||
        (e = dalloc(&D1, (size_t)B * kHid)) || (e = dalloc(&D2, (size_t)B * kHid)) ||
        (e = dalloc(&DZ, (size_t)B * out)) || (e = dalloc(&L, B)))
        return e;
    cudaMemsetAsync(Mm, 0, ly.total * 4, st);
    cudaMemsetAsync(Vv, 0, ly.total * 4, st);
    const size_t smem = (size_t)ly.total * 4;
    cudaFuncSetAttribute(mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    std::vector<float> hl(B);
    const float b1 = 0.9f, b2 = 0.999f;
    for (int s = 0; s < steps && e == cudaSuccess; ++s) {
        gather_batch<<<(B + 255) / 256, 256, 0, st>>>(X, Y, W, M, B, seed * 1000003ull + s, Xb, Yb, Wb);
        mlp_fwd_bwd<<<(B + 127) / 128, 128, smem, st>>>(d_P, out, loss_kind, Xb, Yb, Wb, B,
                                                        1.0f / (float)B, H1, H2, D1, D2, DZ, L);
        weight_grad<<<out, 128, 0, st>>>(DZ, out, H2, kHid, B, G + ly.w3, G + ly.b3);
        weight_grad<<<kHid, 128, 0, st>>>(D2, kHid, H1, kHid, B, G + ly.w2, G + ly.b2);
        weight_grad<<<kHid, 128, 0, st>>>(D1, kHid, Xb, kFeat, B, G + ly.w1, G + ly.b1);
        const float c1 = 1.0f - powf(b1, (float)(s + 1)), c2 = 1.0f - powf(b2, (float)(s + 1));
        const float lr_s = lr * (s < steps / 2 ? 1.0f : 0.3f);
        adam_step<<<(ly.total + 255) / 256, 256, 0, st>>>(d_P, G, Mm, Vv, ly.total, lr_s, b1, b2,
                                                          1e-8f, c1, c2);
        e = cudaGetLastError();
        if (e == cudaSuccess && (s == 0 || s == steps - 1)) {
            e = cudaMemcpyAsync(hl.data(), L, (size_t)B * 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            double sum = 0;
            for (float v : hl) sum += v;
            (s == 0 ? res->loss_first : res->loss_last) = sum / B;
        }
    }
    cudaFree(G); cudaFree(Mm); cudaFree(Vv); cudaFree(Xb); cudaFree(Yb); cudaFree(Wb);
    cudaFree(H1); cudaFree(H2); cudaFree(D1); cudaFree(D2); cudaFree(DZ); cudaFree(L);
    return e;
}

// Deterministic parameter initialisation (He-uniform from a hash).
void init_params(std::vector<float>& P, int out, uint64_t seed) {
    const Layout ly(out);
    P.assign(ly.total, 0.0f);
    auto fill = [&](int off, int rows, int fan_in) {
        const float a = std::sqrt(6.0f / (float)fan_in);
        for (int i = 0; i < rows * fan_in; ++i) {
            uint64_t h = seed ^ (0x9e3779b97f4a7c15ull * (uint64_t)(off + i + 1));
            h ^= h >> 31;
            h *= 0xbf58476d1ce4e5b9ull;
            h ^= h >> 29;
            const float u = (float)((h >> 11) * (1.0 / 9007199254740992.0));
            P[off + i] = (2.0f * u - 1.0f) * a;
        }
    };
    fill(ly.w1, kHid, kFeat);
    fill(ly.w2, kHid, kHid);
    fill(ly.w3, out, kHid);
}

}  // namespace

// Gradient of the mean sample-weighted loss for a batch (test entry point).
cudaError_t mlp_grad(const float* hP, int out, int loss_kind, const float* hX, const float* hY,
                     const float* hW, int B, float* hG, double* loss) {
    const Layout ly(out);
    float *P, *X, *Y, *W = nullptr, *G, *H1, *H2, *D1, *D2, *DZ, *L;
    cudaError_t e;
    if ((e = dalloc(&P, ly.total)) || (e = dalloc(&X, (size_t)B * kFeat)) || (e = dalloc(&Y, B)) ||
        (e = dalloc(&G, ly.total)) || (e = dalloc(&H1, (size_t)B * kHid)) ||
        (e = dalloc(&H2, (size_t)B * kHid)) || (e = dalloc(&D1, (size_t)B * kHid)) ||
        (e = dalloc(&D2, (size_t)B * kHid)) || (e = dalloc(&DZ, (size_t)B * out)) ||
        (e = dalloc(&L, B)))
        return e;
    if (hW) e = dalloc(&W, B);
    cudaMemcpy(P, hP, ly.total * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(X, hX, (size_t)B * kFeat * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(Y, hY, (size_t)B * 4, cudaMemcpyHostToDevice);
    if (hW) cudaMemcpy(W, hW, (size_t)B * 4, cudaMemcpyHostToDevice);
    const size_t smem = (size_t)ly.total * 4;
    cudaFuncSetAttribute(mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    mlp_fwd_bwd<<<(B + 127) / 128, 128, smem>>>(P, out, loss_kind, X, Y, W, B, 1.0f / (float)B,
                                                H1, H2, D1, D2, DZ, L);
    weight_grad<<<out, 128>>>(DZ, out, H2, kHid, B, G + ly.w3, G + ly.b3);
    weight_grad<<<kHid, 128>>>(D2, kHid, H1, kHid, B, G + ly.w2, G + ly.b2);
    weight_grad<<<kHid, 128>>>(D1, kHid, X, kFeat, B, G + ly.w1, G + ly.b1);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(hG, G, ly.total * 4, cudaMemcpyDeviceToHost);
    std::vector<float> hl(B);
    if (e == cudaSuccess) e = cudaMemcpy(hl.data(), L, (size_t)B * 4, cudaMemcpyDeviceToHost);
    double s = 0;
    for (float v : hl) s += v;
    *loss = s / B;
    cudaFree(P); cudaFree(X); cudaFree(Y); cudaFree(W); cudaFree(G); cudaFree(H1); cudaFree(H2);
    cudaFree(D1); cudaFree(D2); cudaFree(DZ); cudaFree(L);
    return e;
}

// Farthest-point sampling of `count` hubs over a strided sample of rows
// (FP32, host copy), starting from node 0 (the reference's build entry).
std::vector<int32_t> pick_hubs(const float* d_base, int64_t n, int dim, int ld, int count,
                               cudaError_t* err) {
    const int64_t ns = std::min<int64_t>(n, 20000);
    const int64_t stride = std::max<int64_t>(1, n / ns);
    std::vector<float> rows((size_t)ns * dim);
    std::vector<int64_t> ids(ns);
    *err = cudaSuccess;
    for (int64_t i = 0; i < ns; ++i) ids[i] = i * stride;
    *err = cudaMemcpy2D(rows.data(), (size_t)dim * 4, d_base, (size_t)ld * 4 * stride,
                        (size_t)dim * 4, (size_t)ns, cudaMemcpyDeviceToHost);
    std::vector<int32_t> hubs;
    if (*err != cudaSuccess) return hubs;
    std::vector<double> dmin(ns, INFINITY);
    int64_t cur = 0;
    for (int h = 0; h < count && h < ns; ++h) {
        hubs.push_back((int32_t)ids[cur]);
        const float* c = rows.data() + (size_t)cur * dim;
        int64_t far = 0;
        for (int64_t i = 0; i < ns; ++i) {
            const float* r = rows.data() + (size_t)i * dim;
            double s = 0;
            for (int j = 0; j < dim; ++j) {
                const double t = (double)r[j] - c[j];
                s += t * t;
            }
            dmin[i] = std::min(dmin[i], s);
            if (dmin[i] > dmin[far]) far = i;
        }
        cur = far;
    }
    return hubs;
}

cudaError_t learn_models(const LearnInputs& in, LearnOutputs* out) {
    cudaStream_t st = in.stream;
    cudaError_t e = cudaSuccess;
    const int nq = in.nq, maxc = in.max_ckpt;
    // 1) hubs: with the entry stage (args.ecand set) the entry model scores each
    // query's kEntryK candidates; otherwise kFeat farthest-point hubs are scored
    // inside the search kernel
    const bool staged = in.args.ecand != nullptr;
    if (!staged) {
        out->hubs = pick_hubs((const float*)in.base, in.n, in.dim, in.ld, kFeat, &e);
        if (e != cudaSuccess) return e;
    }
    const int H = staged ? kEntryK : (int)out->hubs.size();
    int32_t* d_hubs = nullptr;
    float *efeat = nullptr, *elab = nullptr, *tfeat = nullptr, *tkth = nullptr, *tfin = nullptr;
    int* tcnt = nullptr;
    float *P_entry = nullptr, *P_stop = nullptr;
    __half *h_entry = nullptr, *h_stop = nullptr;
    auto cleanup = [&]() {
        cudaFree(d_hubs); cudaFree(efeat); cudaFree(elab); cudaFree(tfeat); cudaFree(tkth);
        cudaFree(tfin); cudaFree(tcnt); cudaFree(P_entry); cudaFree(P_stop); cudaFree(h_entry);
        cudaFree(h_stop);
    };
    if ((e = dalloc(&d_hubs, H)) || (e = dalloc(&efeat, (size_t)nq * kFeat)) ||
        (e = dalloc(&elab, nq)) || (e = dalloc(&tfeat, (size_t)nq * maxc * kFeat)) ||
        (e = dalloc(&tkth, (size_t)nq * maxc)) || (e = dalloc(&tfin, nq)) ||
        (e = dalloc(&tcnt, nq))) {
        cleanup();
        return e;
    }
    if (!staged) cudaMemcpyAsync(d_hubs, out->hubs.data(), H * 4, cudaMemcpyHostToDevice, st);
    // 2) pass 1 (plain method from the nearest candidates when staged): entry features
    SearchArgs a = in.args;
    a.lm = 1;
    a.hubs = d_hubs;
    a.n_hubs = staged ? 0 : H;
    a.entry_w = nullptr;
    a.stop_w = nullptr;
    a.tr_entry_feat = efeat;
    a.tr_feat = tfeat;
    a.tr_kth = tkth;
    a.tr_count = tcnt;
    a.tr_final_kth = tfin;
    a.max_ckpt = maxc;
    e = cudaMemsetAsync(a.counter, 0, 4, st);
    if (e == cudaSuccess) e = launch_search(SONG_KIND_L2, a, in.num_sms, st);
    if (e == cudaSuccess) {
        if (staged)
            entry_labels_staged<<<(nq + 7) / 8, 256, 0, st>>>((const float*)in.base, in.ld, in.dim,
                                                              a.ecand, in.nn1, nq, elab);
        else
            entry_labels<<<(nq + 7) / 8, 256, 0, st>>>((const float*)in.base, in.ld, in.dim, d_hubs,
                                                       H, in.nn1, nq, elab);
        e = cudaGetLastError();
    }
    // 3) train the entry model
    std::vector<float> P;
    const Layout le(H), ls(1);
    if (e == cudaSuccess) e = dalloc(&P_entry, le.total);
    if (e == cudaSuccess) {
        init_params(P, H, in.seed);
        cudaMemcpyAsync(P_entry, P.data(), le.total * 4, cudaMemcpyHostToDevice, st);
        TrainResult r;
        e = train_mlp(P_entry, H, kLossCE, efeat, elab, nullptr, nq, in.entry_steps, in.batch,
                      in.lr, in.seed + 1, st, &r);
        out->entry_loss_first = r.loss_first;
        out->entry_loss_last = r.loss_last;
    }
    if (e == cudaSuccess) e = dalloc(&h_entry, le.total);
    if (e == cudaSuccess) {
        to_half<<<(le.total + 255) / 256, 256, 0, st>>>(P_entry, h_entry, le.total);
        e = cudaGetLastError();
    }
    // 4) pass 2 (plain method, learned entry): stop traces
    if (e == cudaSuccess) {
        a.entry_w = h_entry;
        a.tr_entry_feat = nullptr;
        e = cudaMemsetAsync(a.counter, 0, 4, st);
    }
    if (e == cudaSuccess) e = launch_search(SONG_KIND_L2, a, in.num_sms, st);
    std::vector<int> cnt(nq);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), tcnt, (size_t)nq * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    std::vector<int64_t> offs(nq + 1, 0);
    for (int q = 0; q < nq; ++q) offs[q + 1] = offs[q] + cnt[q];
    const int64_t M = offs[nq];
    out->stop_samples = M;
    float *sx = nullptr, *sy = nullptr;
    int64_t* d_offs = nullptr;
    if (e == cudaSuccess && M > 0) {
        if ((e = dalloc(&sx, (size_t)M * kFeat)) || (e = dalloc(&sy, M)) || (e = dalloc(&d_offs, nq + 1))) {
        } else {
            cudaMemcpyAsync(d_offs, offs.data(), (size_t)(nq + 1) * 8, cudaMemcpyHostToDevice, st);
            stop_samples<<<nq, 128, 0, st>>>(tfeat, tkth, tcnt, tfin, d_offs, nq, maxc, sx, sy);
            e = cudaGetLastError();
        }
    }
    // positive fraction
    if (e == cudaSuccess && M > 0) {
        std::vector<float> hy(M);
        e = cudaMemcpyAsync(hy.data(), sy, (size_t)M * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        double pos = 0;
        for (float v : hy) pos += v;
        out->stop_pos_frac = pos / (double)M;
    }
    // 5) train the stop model
    if (e == cudaSuccess) e = dalloc(&P_stop, ls.total);
    if (e == cudaSuccess && M > 0) {
        init_params(P, 1, in.seed + 7);
        cudaMemcpyAsync(P_stop, P.data(), ls.total * 4, cudaMemcpyHostToDevice, st);
        TrainResult r;
        e = train_mlp(P_stop, 1, kLossBCE, sx, sy, nullptr, M, in.stop_steps, in.batch, in.lr,
                      in.seed + 2, st, &r);
        out->stop_loss_first = r.loss_first;
        out->stop_loss_last = r.loss_last;
    }
    // 6) results: FP32 master copies to the host
    if (e == cudaSuccess) {
        out->entry.resize(le.total);
        out->stop.resize(ls.total);
        e = cudaMemcpyAsync(out->entry.data(), P_entry, le.total * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out->stop.data(), P_stop, ls.total * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaFree(sx);
    cudaFree(sy);
    cudaFree(d_offs);
    cleanup();
    return e;
}

cudaError_t upload_half(const std::vector<float>& P, __half** d) {
    std::vector<__half> h(P.size());
    for (size_t i = 0; i < P.size(); ++i) h[i] = __float2half_rn(P[i]);
    cudaFree(*d);
    *d = nullptr;
    cudaError_t e = cudaMalloc((void**)d, std::max<size_t>(1, h.size()) * sizeof(__half));
    if (e == cudaSuccess) e = cudaMemcpy(*d, h.data(), h.size() * sizeof(__half), cudaMemcpyHostToDevice);
    return e;
}

}  // namespace song
