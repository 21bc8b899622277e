// Learned quadrature selector: a small MLP (12 -> 64 -> 64 -> 4, ReLU,
// softmax, FP32) predicts, for each (source, field) pair, the cheapest outer
// Gauss-Hammer rule (3, 7, 12 or 19 nodes) whose blocks agree with the
// maximal rule within a tolerance; below a confidence threshold it falls back
// to the maximal rule.  No counterpart in the reference (which uses one rule
// for all pairs, BEMenerg_setupCore.m:13-28).
//
// Everything runs in hand-written kernels: pair features, convergence labels
// from the plain assembly at the four rules, mini-batch forward/backward with
// the weight gradients as per-block contractions over the batch, Adam, and
// inference.  The networks' GEMMs are tiny (<= 64 x 64 per sample); they run
// on the FP32 pipes, which keep a whole epoch over 2e5 samples in
// milliseconds.
#include "ebem_internal.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

namespace ebem {

constexpr int kF = 12, kH = 64, kC = 4;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kC * kH, kParams = kOffB3 + kC;
static_assert(kParams == 5252, "parameter count");
constexpr int kRules[kC] = {3, 7, 12, 19};

// ---------------------------------------------------------------------------
// features of pair (i source, j field), all O(1):
//  0 log(d/h_j)  1 log(d/h_i)  2 gap/h_j (clipped)  3 log(h_i/h_j)  4 |n_i.n_j|
//  5 |n_j.(c_i-c_j)|/d  6 |n_i.(c_i-c_j)|/d  7 log(c_P dt/h_j)  8 log(c_S dt/h_j)
//  9 c_P/c_S - 1  10 same triangle  11 area_j/h_j^2
// d = centroid distance (at least h_j/20), h = longest edge.
__device__ void pair_features(float f[kF], const TriGeom& Ti, const TriGeom& Tj, bool same, double velP, double velS,
                              double dt) {
    const double v0 = Ti.ctr[0] - Tj.ctr[0], v1 = Ti.ctr[1] - Tj.ctr[1], v2 = Ti.ctr[2] - Tj.ctr[2];
    const double hj = Tj.maxL, hi = Ti.maxL;
    const double d = fmax(sqrt(v0 * v0 + v1 * v1 + v2 * v2), 0.05 * hj);
    const double gap = (d - hi - hj) / hj;
    f[0] = (float)log(d / hj);
    f[1] = (float)log(d / hi);
    f[2] = (float)fmin(fmax(gap, -2.0), 20.0) * 0.1f;
    f[3] = (float)log(hi / hj);
    f[4] = (float)fabs(Ti.n[0] * Tj.n[0] + Ti.n[1] * Tj.n[1] + Ti.n[2] * Tj.n[2]);
    f[5] = (float)(fabs(Tj.n[0] * v0 + Tj.n[1] * v1 + Tj.n[2] * v2) / d);
    f[6] = (float)(fabs(Ti.n[0] * v0 + Ti.n[1] * v1 + Ti.n[2] * v2) / d);
    f[7] = (float)log(velP * dt / hj);
    f[8] = (float)log(velS * dt / hj);
    f[9] = (float)(velP / velS - 1.0);
    f[10] = same ? 1.0f : 0.0f;
    f[11] = (float)(Tj.area / (hj * hj));
}

__global__ void features_kernel(const TriGeom* __restrict__ geo, int N, double velP, double velS, double dt,
                                float* __restrict__ out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)N * N) return;
    const int i = (int)(p % N), j = (int)(p / N);
    float f[kF];
    pair_features(f, geo[i], geo[j], i == j, velP, velS, dt);
#pragma unroll
    for (int k = 0; k < kF; k++) out[p * kF + k] = f[k];
}

// max |E| over the whole array (non-negative doubles order like their bits)
__global__ void absmax_kernel(const double* __restrict__ E, long long n, unsigned long long* out) {
    double m = 0.0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(E[k]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// label of pair p: smallest rule whose blocks (all lags) differ from the
// maximal rule's by at most tol * max|E_max|; else the maximal rule.
__global__ void labels_kernel(const double* __restrict__ E0, const double* __restrict__ E1,
                              const double* __restrict__ E2, const double* __restrict__ E3, int N, int L,
                              const unsigned long long* __restrict__ scale_bits, double tol, int* __restrict__ labels) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)N * N) return;
    const int i = (int)(p % N), j = (int)(p / N);
    const double thr = tol * __longlong_as_double((long long)*scale_bits);
    const size_t n3 = 3 * (size_t)N;
    double err[3] = {0.0, 0.0, 0.0};
    const double* Er[3] = {E0, E1, E2};
    for (int l = 0; l < L; l++)
        for (int c = 0; c < 3; c++)
            for (int r = 0; r < 3; r++) {
                const size_t idx = (size_t)l * n3 * n3 + (3 * (size_t)j + c) * n3 + 3 * (size_t)i + r;
                const double ref = E3[idx];
#pragma unroll
                for (int q = 0; q < 3; q++) err[q] = fmax(err[q], fabs(Er[q][idx] - ref));
            }
    int lab = kC - 1;
    for (int q = 2; q >= 0; q--)
        if (err[q] <= thr) lab = q;
    labels[p] = lab;
}

// ---------------------------------------------------------------------------
// MLP: forward for one sample (weights in shared memory)

__device__ __forceinline__ void mlp_forward(const float* __restrict__ w, const float x[kF], float h1[kH], float h2[kH],
                                            float z[kC]) {
    for (int o = 0; o < kH; o++) {
        float a = w[kOffB1 + o];
#pragma unroll
        for (int k = 0; k < kF; k++) a += w[kOffW1 + o * kF + k] * x[k];
        h1[o] = fmaxf(a, 0.0f);
    }
    for (int o = 0; o < kH; o++) {
        float a = w[kOffB2 + o];
        for (int k = 0; k < kH; k++) a += w[kOffW2 + o * kH + k] * h1[k];
        h2[o] = fmaxf(a, 0.0f);
    }
#pragma unroll
    for (int o = 0; o < kC; o++) {
        float a = w[kOffB3 + o];
        for (int k = 0; k < kH; k++) a += w[kOffW3 + o * kH + k] * h2[k];
        z[o] = a;
    }
}

// Mini-batch gradient of the mean cross-entropy.  A block takes kB samples:
// activations and back-propagated errors are staged in shared memory, each
// weight gradient entry is a contraction over the block's samples, added to
// grad with one atomic per entry and block.
constexpr int kB = 64, kThreads = 256;
struct GradSmem {
    float w[kParams];
    float x[kB][kF];
    float h1[kB][kH];
    float h2[kB][kH];
    float d2[kB][kH];
    float d1[kB][kH];
    float d3[kB][kC];
};

__global__ void __launch_bounds__(kThreads) mlp_grad_kernel(const float* __restrict__ params,
                                                           const float* __restrict__ feats,
                                                           const int* __restrict__ labels,
                                                           const long long* __restrict__ index, long long n,
                                                           float inv_n, float* __restrict__ grad, float* loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem& S = *reinterpret_cast<GradSmem*>(smem_raw);
    const int t = threadIdx.x;
    for (int k = t; k < kParams; k += kThreads) S.w[k] = params[k];
    const long long s0 = (long long)blockIdx.x * kB;
    const int nb = (int)min((long long)kB, n - s0);
    for (int k = t; k < kB * kF; k += kThreads) {
        const int b = k / kF, c = k % kF;
        S.x[b][c] = (b < nb) ? feats[(index ? index[s0 + b] : s0 + b) * kF + c] : 0.0f;
    }
    __syncthreads();
    // layer 1: h1 = relu(W1 x + b1)
    for (int k = t; k < kB * kH; k += kThreads) {
        const int b = k / kH, o = k % kH;
        float a = S.w[kOffB1 + o];
#pragma unroll
        for (int c = 0; c < kF; c++) a += S.w[kOffW1 + o * kF + c] * S.x[b][c];
        S.h1[b][o] = fmaxf(a, 0.0f);
    }
    __syncthreads();
    for (int k = t; k < kB * kH; k += kThreads) {
        const int b = k / kH, o = k % kH;
        float a = S.w[kOffB2 + o];
        for (int c = 0; c < kH; c++) a += S.w[kOffW2 + o * kH + c] * S.h1[b][c];
        S.h2[b][o] = fmaxf(a, 0.0f);
    }
    __syncthreads();
    // output, softmax, loss, d3 = (p - onehot) / n
    float lsum = 0.0f;
    for (int b = t; b < kB; b += kThreads) {
        float z[kC], m = -1e30f;
        for (int o = 0; o < kC; o++) {
            float a = S.w[kOffB3 + o];
            for (int c = 0; c < kH; c++) a += S.w[kOffW3 + o * kH + c] * S.h2[b][c];
            z[o] = a;
            m = fmaxf(m, a);
        }
        float den = 0.0f;
        for (int o = 0; o < kC; o++) den += expf(z[o] - m);
        const int y = (b < nb) ? labels[index ? index[s0 + b] : s0 + b] : 0;
        for (int o = 0; o < kC; o++) {
            const float pr = expf(z[o] - m) / den;
            S.d3[b][o] = (b < nb) ? (pr - (o == y ? 1.0f : 0.0f)) * inv_n : 0.0f;
        }
        if (b < nb) lsum += (logf(den) + m - z[y]) * inv_n;
    }
    if (loss && t < kB && lsum != 0.0f) atomicAdd(loss, lsum);
    __syncthreads();
    // d2 = (W3^T d3) * (h2 > 0)
    for (int k = t; k < kB * kH; k += kThreads) {
        const int b = k / kH, c = k % kH;
        float a = 0.0f;
#pragma unroll
        for (int o = 0; o < kC; o++) a += S.w[kOffW3 + o * kH + c] * S.d3[b][o];
        S.d2[b][c] = (S.h2[b][c] > 0.0f) ? a : 0.0f;
    }
    __syncthreads();
    // d1 = (W2^T d2) * (h1 > 0)
    for (int k = t; k < kB * kH; k += kThreads) {
        const int b = k / kH, c = k % kH;
        float a = 0.0f;
        for (int o = 0; o < kH; o++) a += S.w[kOffW2 + o * kH + c] * S.d2[b][o];
        S.d1[b][c] = (S.h1[b][c] > 0.0f) ? a : 0.0f;
    }
    __syncthreads();
    // weight gradients: contractions over the block's samples
    for (int k = t; k < kParams; k += kThreads) {
        float g = 0.0f;
        if (k < kOffB1) {
            const int o = (k - kOffW1) / kF, c = (k - kOffW1) % kF;
            for (int b = 0; b < kB; b++) g += S.d1[b][o] * S.x[b][c];
        } else if (k < kOffW2) {
            const int o = k - kOffB1;
            for (int b = 0; b < kB; b++) g += S.d1[b][o];
        } else if (k < kOffB2) {
            const int o = (k - kOffW2) / kH, c = (k - kOffW2) % kH;
            for (int b = 0; b < kB; b++) g += S.d2[b][o] * S.h1[b][c];
        } else if (k < kOffW3) {
            const int o = k - kOffB2;
            for (int b = 0; b < kB; b++) g += S.d2[b][o];
        } else if (k < kOffB3) {
            const int o = (k - kOffW3) / kH, c = (k - kOffW3) % kH;
            for (int b = 0; b < kB; b++) g += S.d3[b][o] * S.h2[b][c];
        } else {
            const int o = k - kOffB3;
            for (int b = 0; b < kB; b++) g += S.d3[b][o];
        }
        if (g != 0.0f) atomicAdd(grad + k, g);
    }
}

__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                            float lr, float b1, float b2, float c1, float c2, float eps) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kParams) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1 - b1) * gk, vk = b2 * v[k] + (1 - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    g[k] = 0.0f;
}

// Inference for every pair of a mesh: class of the largest probability, or
// the maximal rule when that probability is below the threshold.
__global__ void __launch_bounds__(128) infer_kernel(const float* __restrict__ params, const TriGeom* __restrict__ geo,
                                                    int N, double velP, double velS, double dt, float threshold,
                                                    int* __restrict__ classes) {
    __shared__ float w[kParams];
    for (int k = threadIdx.x; k < kParams; k += blockDim.x) w[k] = params[k];
    __syncthreads();
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)N * N) return;
    const int i = (int)(p % N), j = (int)(p / N);
    float x[kF], h1[kH], h2[kH], z[kC];
    pair_features(x, geo[i], geo[j], i == j, velP, velS, dt);
    mlp_forward(w, x, h1, h2, z);
    float m = z[0];
    int arg = 0;
    for (int o = 1; o < kC; o++)
        if (z[o] > m) { m = z[o]; arg = o; }
    float den = 0.0f;
    for (int o = 0; o < kC; o++) den += expf(z[o] - m);
    const float pmax = 1.0f / den;
    classes[p] = (pmax >= threshold) ? arg : kC - 1;
}

// Pair lists per class that keep the pair order of each tile of kSplit pairs
// (so the assembly of a class walks the matrix in order): pass 1 counts the
// classes of each tile, the host scans the counts, pass 2 writes each pair at
// its tile's offset plus its rank among the tile's pairs of its class.
constexpr int kSplit = 1024;

__global__ void __launch_bounds__(kSplit) split_count_kernel(const int* __restrict__ classes, long long NN,
                                                            unsigned* __restrict__ tile_counts) {
    __shared__ unsigned cnt[kC];
    if (threadIdx.x < kC) cnt[threadIdx.x] = 0;
    __syncthreads();
    const long long p = (long long)blockIdx.x * kSplit + threadIdx.x;
    if (p < NN) atomicAdd(&cnt[classes[p]], 1u);
    __syncthreads();
    if (threadIdx.x < kC) tile_counts[(size_t)blockIdx.x * kC + threadIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(kSplit) split_write_kernel(const int* __restrict__ classes, int N,
                                                            const unsigned long long* __restrict__ tile_offsets,
                                                            int2* __restrict__ lists) {
    __shared__ unsigned wcnt[kSplit / 32][kC];
    const long long NN = (long long)N * N;
    const long long p = (long long)blockIdx.x * kSplit + threadIdx.x;
    const int c = (p < NN) ? classes[p] : -1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned rank = 0;
#pragma unroll
    for (int q = 0; q < kC; q++) {
        const unsigned m = __ballot_sync(0xffffffffu, c == q);
        if (c == q) rank = __popc(m & ((1u << lane) - 1u));
        if (lane == 0) wcnt[warp][q] = __popc(m);
    }
    __syncthreads();
    if (c >= 0) {
        unsigned before = 0;
        for (int w = 0; w < warp; w++) before += wcnt[w][c];
        const unsigned long long pos = tile_offsets[(size_t)blockIdx.x * kC + c] + before + rank;
        lists[(size_t)c * NN + pos] = make_int2((int)(p % N), (int)(p / N));
    }
}

// ---------------------------------------------------------------------------
// host side

int selector_features(const MeshData& m, const PhysParams& P, float* d_out, cudaStream_t s) {
    const long long NN = (long long)m.nt * m.nt;
    features_kernel<<<(unsigned)((NN + 127) / 128), 128, 0, s>>>(m.d_geo, m.nt, P.velP, P.velS, P.dt, d_out);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

int selector_labels(MeshData& m, const PhysParams& P, int L, double tol, int* d_labels, cudaStream_t s) {
    const size_t n3 = 3 * (size_t)m.nt, per = n3 * n3 * L;
    double* E[kC] = {nullptr, nullptr, nullptr, nullptr};
    unsigned long long* d_scale = nullptr;
    int rc = EBEM_OK;
    for (int q = 0; q < kC && rc == EBEM_OK; q++)
        if (cudaMalloc(&E[q], per * sizeof(double)) != cudaSuccess) { cudaGetLastError(); rc = fail(EBEM_ERR_NOMEM, "label assembly buffers"); }
    if (rc == EBEM_OK && cudaMalloc(&d_scale, sizeof(unsigned long long)) != cudaSuccess) { cudaGetLastError(); rc = fail(EBEM_ERR_NOMEM, "alloc"); }
    for (int q = 0; q < kC && rc == EBEM_OK; q++) {
        rc = map_nodes(m, kRules[q], s);
        if (!rc) rc = launch_sa_assemble(m, P, kRules[q], 0, L, 0, m.nt, E[q], n3, n3 * n3, 0, nullptr, s);
    }
    if (rc == EBEM_OK) {
        cudaMemsetAsync(d_scale, 0, sizeof(unsigned long long), s);
        absmax_kernel<<<296, 256, 0, s>>>(E[kC - 1], (long long)per, d_scale);
        const long long NN = (long long)m.nt * m.nt;
        labels_kernel<<<(unsigned)((NN + 127) / 128), 128, 0, s>>>(E[0], E[1], E[2], E[3], m.nt, L, d_scale, tol, d_labels);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, std::string("selector labels: ") + cudaGetErrorString(e));
    }
    for (int q = 0; q < kC; q++) if (E[q]) cudaFree(E[q]);
    if (d_scale) cudaFree(d_scale);
    return rc;
}

static size_t grad_smem() { return sizeof(GradSmem); }

static int grad_launch(const float* params, const float* feats, const int* labels, const long long* index, long long n,
                       float inv_n, float* grad, float* loss, cudaStream_t s) {
    EBEM_CUDA_TRY(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem()));
    const unsigned blocks = (unsigned)((n + kB - 1) / kB);
    mlp_grad_kernel<<<blocks, kThreads, grad_smem(), s>>>(params, feats, labels, index, n, inv_n, grad, loss);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

int selector_grad(const float* d_params, const float* d_feats, const int* d_labels, long long n, float* d_grad,
                  float* d_loss, cudaStream_t s) {
    EBEM_CUDA_TRY(cudaMemsetAsync(d_grad, 0, sizeof(float) * kParams, s));
    if (d_loss) EBEM_CUDA_TRY(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
    return grad_launch(d_params, d_feats, d_labels, nullptr, n, 1.0f / (float)n, d_grad, d_loss, s);
}

int selector_train(float* d_params, const float* d_feats, const int* d_labels, long long n, int epochs, int batch,
                   float lr, unsigned long long seed, float* h_losses, cudaStream_t s) {
    float *g = nullptr, *mo = nullptr, *vo = nullptr, *loss = nullptr;
    long long* d_idx = nullptr;
    int rc = EBEM_OK;
    if (cudaMalloc(&g, sizeof(float) * kParams) || cudaMalloc(&mo, sizeof(float) * kParams) ||
        cudaMalloc(&vo, sizeof(float) * kParams) || cudaMalloc(&loss, sizeof(float)) ||
        cudaMalloc(&d_idx, sizeof(long long) * n)) {
        cudaGetLastError();
        rc = fail(EBEM_ERR_NOMEM, "training workspace allocation failed");
    }
    std::vector<long long> idx(n);
    for (long long k = 0; k < n; k++) idx[k] = k;
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int step = 0;
    if (!rc) {
        cudaMemsetAsync(g, 0, sizeof(float) * kParams, s);
        cudaMemsetAsync(mo, 0, sizeof(float) * kParams, s);
        cudaMemsetAsync(vo, 0, sizeof(float) * kParams, s);
    }
    for (int ep = 0; ep < epochs && rc == EBEM_OK; ep++) {
        std::shuffle(idx.begin(), idx.end(), rng);
        if (cudaMemcpyAsync(d_idx, idx.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) {
            rc = fail(EBEM_ERR_CUDA, "training upload failed");
            break;
        }
        for (long long b0 = 0; b0 < n && rc == EBEM_OK; b0 += batch) {
            const long long nb = std::min<long long>(batch, n - b0);
            rc = grad_launch(d_params, d_feats, d_labels, d_idx + b0, nb, 1.0f / (float)nb, g, nullptr, s);
            if (rc) break;
            step++;
            const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
            adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(d_params, g, mo, vo, lr, b1, b2, c1, c2, eps);
            if (cudaGetLastError() != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "adam step failed");
        }
        if (rc) break;
        // epoch loss at the updated weights (full pass, no update)
        float* gtmp = g;
        rc = grad_launch(d_params, d_feats, d_labels, d_idx, n, 1.0f / (float)n, gtmp, loss, s);
        cudaMemsetAsync(g, 0, sizeof(float) * kParams, s);
        float hl = 0.0f;
        if (!rc && (cudaMemcpyAsync(&hl, loss, sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                    cudaStreamSynchronize(s) != cudaSuccess))
            rc = fail(EBEM_ERR_CUDA, "loss download failed");
        if (h_losses) h_losses[ep] = hl;
    }
    cudaStreamSynchronize(s);
    cudaFree(g); cudaFree(mo); cudaFree(vo); cudaFree(loss); cudaFree(d_idx);
    return rc;
}

int selector_infer(const float* d_params, const MeshData& m, const PhysParams& P, float threshold, int* d_classes,
                   cudaStream_t s) {
    const long long NN = (long long)m.nt * m.nt;
    infer_kernel<<<(unsigned)((NN + 127) / 128), 128, 0, s>>>(d_params, m.d_geo, m.nt, P.velP, P.velS, P.dt,
                                                               threshold, d_classes);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

int assemble_selected(MeshData& m, const PhysParams& P, const int* d_classes, int lag0, int nlag, double* d_E, int prec,
                      long long* h_counts, cudaStream_t s) {
    const long long NN = (long long)m.nt * m.nt;
    const long long tiles = (NN + kSplit - 1) / kSplit;
    unsigned* d_tc = nullptr;
    unsigned long long* d_off = nullptr;
    int2* lists = nullptr;
    int rc = EBEM_OK;
    if (cudaMalloc(&d_tc, sizeof(unsigned) * tiles * kC) != cudaSuccess ||
        cudaMalloc(&d_off, sizeof(unsigned long long) * tiles * kC) != cudaSuccess ||
        cudaMalloc(&lists, sizeof(int2) * (size_t)NN * kC) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_tc); cudaFree(d_off);
        return fail(EBEM_ERR_NOMEM, "pair list allocation failed");
    }
    std::vector<unsigned> tc((size_t)tiles * kC);
    std::vector<unsigned long long> off((size_t)tiles * kC);
    unsigned long long total[kC] = {0, 0, 0, 0};
    split_count_kernel<<<(unsigned)tiles, kSplit, 0, s>>>(d_classes, NN, d_tc);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(tc.data(), d_tc, sizeof(unsigned) * tc.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) {
        for (long long t = 0; t < tiles; t++)
            for (int q = 0; q < kC; q++) {
                off[(size_t)t * kC + q] = total[q];
                total[q] += tc[(size_t)t * kC + q];
            }
        e = cudaMemcpyAsync(d_off, off.data(), sizeof(unsigned long long) * off.size(), cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) {
        split_write_kernel<<<(unsigned)tiles, kSplit, 0, s>>>(d_classes, m.nt, d_off, lists);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, std::string("pair split: ") + cudaGetErrorString(e));
    const size_t n3 = 3 * (size_t)m.nt;
    for (int q = 0; q < kC && rc == EBEM_OK; q++) {
        if (h_counts) h_counts[q] = (long long)total[q];
        if (total[q] == 0) continue;
        rc = map_nodes(m, kRules[q], s);
        if (!rc)
            rc = launch_sa_assemble(m, P, kRules[q], lag0, nlag, 0, m.nt, d_E, n3, n3 * n3, 0, nullptr, s, 0, prec,
                                    lists + (size_t)q * NN, (long long)total[q]);
    }
    if (rc == EBEM_OK && (e = cudaStreamSynchronize(s)) != cudaSuccess)
        rc = fail(EBEM_ERR_CUDA, std::string("selected assembly: ") + cudaGetErrorString(e));
    cudaFree(d_tc);
    cudaFree(d_off);
    cudaFree(lists);
    return rc;
}

void selector_init(float* h_params, unsigned long long seed) {
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int n_out, int n_in) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / n_in));
        for (int k = 0; k < n_out * n_in; k++) h_params[off + k] = nd(rng);
    };
    fill(kOffW1, kH, kF);
    fill(kOffW2, kH, kH);
    fill(kOffW3, kC, kH);
    for (int k = 0; k < kH; k++) { h_params[kOffB1 + k] = 0.0f; h_params[kOffB2 + k] = 0.0f; }
    for (int k = 0; k < kC; k++) h_params[kOffB3 + k] = 0.0f;
}

}  // namespace ebem
