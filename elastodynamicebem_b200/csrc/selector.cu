// Learned quadrature selector: a small MLP (12 -> 64 -> 64 -> 4, ReLU,
// softmax, FP32) predicts, for each (source, field, lag), which of four outer
// rules -- a Gauss-Hammer order on a number of congruent sub-triangles of the
// source triangle (GaussHammerComposite.m), given by the caller -- assembles
// that block; below a confidence threshold it falls back to the last
// (maximal) rule.  No counterpart in the reference (which uses one rule for
// all pairs and lags, BEMenerg_setupCore.m:13-28).
//
// Everything runs in hand-written kernels: per-(pair, lag) features, labels
// from the plain method's convergence (the blocks of sampled pairs at the four
// rules, the smallest rule within a tolerance of the maximal one),
// mini-batch forward/backward with the weight gradients as per-block
// contractions over the batch, Adam, inference over every non-null (pair,
// lag) of a mesh, and the assembly of each class's lags with its rule.  The
// network's GEMMs are tiny (<= 64 x 64 per sample); they run on the FP32
// pipes.
#include "ebem_internal.h"
#include "sa_pair.cuh"

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

namespace ebem {

constexpr int kF = 12, kH = 64, kC = 4;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kC * kH, kParams = kOffB3 + kC;
static_assert(kParams == 5252, "parameter count");

// ---------------------------------------------------------------------------
// features of (source i, field j, lag l), all O(1):
//  0 log(d/h_j)  1 log(d/h_i)  2 gap/h_j (clipped, x 0.1)  3 log(h_i/h_j)
//  4 |n_i.n_j|  5 |n_j.(c_i-c_j)|/d  6 |n_i.(c_i-c_j)|/d
//  7 c_P l dt / r_min  8 c_S l dt / r_max  (x 0.1, clipped at 3)
//  9 (c_P l dt - d)/h_j  10 (c_S l dt - d)/h_j  (x 0.1, clipped at +-3)
// 11 log(c_S dt / h_j)
// d = centroid distance (at least h_j/20), h = longest edge, r_min / r_max =
// the null test's distance bounds d -/+ (h_i + h_j) (r_min at least h_j/20).
__device__ void lag_features(float f[kF], const TriGeom& Ti, const TriGeom& Tj, int l, double velP, double velS,
                             double dt) {
    const double v0 = Ti.ctr[0] - Tj.ctr[0], v1 = Ti.ctr[1] - Tj.ctr[1], v2 = Ti.ctr[2] - Tj.ctr[2];
    const double hj = Tj.maxL, hi = Ti.maxL;
    const double d = fmax(sqrt(v0 * v0 + v1 * v1 + v2 * v2), 0.05 * hj);
    const double gap = (d - hi - hj) / hj;
    const double rmin = fmax(d - hi - hj, 0.05 * hj), rmax = d + hi + hj;
    const double tP = velP * l * dt, tS = velS * l * dt;
    f[0] = (float)log(d / hj);
    f[1] = (float)log(d / hi);
    f[2] = (float)fmin(fmax(gap, -2.0), 20.0) * 0.1f;
    f[3] = (float)log(hi / hj);
    f[4] = (float)fabs(Ti.n[0] * Tj.n[0] + Ti.n[1] * Tj.n[1] + Ti.n[2] * Tj.n[2]);
    f[5] = (float)(fabs(Tj.n[0] * v0 + Tj.n[1] * v1 + Tj.n[2] * v2) / d);
    f[6] = (float)(fabs(Ti.n[0] * v0 + Ti.n[1] * v1 + Ti.n[2] * v2) / d);
    f[7] = (float)fmin(0.1 * tP / rmin, 3.0);
    f[8] = (float)fmin(0.1 * tS / rmax, 3.0);
    f[9] = (float)fmin(fmax(0.1 * (tP - d) / hj, -3.0), 3.0);
    f[10] = (float)fmin(fmax(0.1 * (tS - d) / hj, -3.0), 3.0);
    f[11] = (float)log(velS * dt / hj);
}

// Features of explicit samples (source, field, lag): samples[3 q + 0..2].
__global__ void sample_features_kernel(const TriGeom* __restrict__ geo, const int* __restrict__ samples, long long n,
                                       double velP, double velS, double dt, float* __restrict__ out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = samples[3 * q], j = samples[3 * q + 1], l = samples[3 * q + 2];
    float f[kF];
    lag_features(f, geo[i], geo[j], l, velP, velS, dt);
#pragma unroll
    for (int k = 0; k < kF; k++) out[q * kF + k] = f[k];
}

// Label of each sample from its blocks at the kC rules (blocks[(c n + q) 6 +
// e]): the smallest rule whose block differs from the maximal rule's by at
// most tol * scale (tol * scale * scales[q] with per-sample scales) in every
// entry; else the maximal rule.
__global__ void labels_kernel(const double* __restrict__ blocks, long long n, double thr0,
                              const double* __restrict__ scales, int* __restrict__ labels) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const double thr = scales ? thr0 * scales[q] : thr0;
    const double* ref = blocks + ((size_t)(kC - 1) * n + q) * 6;
    int lab = kC - 1;
    for (int c = kC - 2; c >= 0; c--) {
        const double* b = blocks + ((size_t)c * n + q) * 6;
        double err = 0.0;
#pragma unroll
        for (int e = 0; e < 6; e++) err = fmax(err, fabs(b[e] - ref[e]));
        if (err <= thr) lab = c;
    }
    labels[q] = lab;
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

// Whether a wavefront sweeps the pair's distance window during lag l's
// instants t_{l-1} .. t_{l+1}: c t over that interval meets [d - h_i - h_j,
// d + h_i + h_j] (the null test's bounds, d the centroid distance) for c =
// c_P or c_S.  There the kernel integral, a function of the outer node, has
// the kinks of the front crossing the field triangle and the outer rule
// converges only algebraically: those lags take the maximal rule whatever
// the network says.
EBEM_DI bool front_sweeps(const TriGeom& Ti, const TriGeom& Tj, int l, double velP, double velS, double dt) {
    const double v0 = Ti.ctr[0] - Tj.ctr[0], v1 = Ti.ctr[1] - Tj.ctr[1], v2 = Ti.ctr[2] - Tj.ctr[2];
    const double d = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    const double lo = d - Ti.maxL - Tj.maxL, hi = d + Ti.maxL + Tj.maxL;
    const double t0 = (l - 1) * dt, t1 = (l + 1) * dt;
    return (velP * t1 >= lo && velP * t0 <= hi) || (velS * t1 >= lo && velS * t0 <= hi);
}

__global__ void sweep_flags_kernel(const TriGeom* __restrict__ geo, const int* __restrict__ samples, long long n,
                                   double velP, double velS, double dt, unsigned char* __restrict__ out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    out[q] = front_sweeps(geo[samples[3 * q]], geo[samples[3 * q + 1]], samples[3 * q + 2], velP, velS, dt) ? 1 : 0;
}

// Inference for every non-null (pair, lag) of a mesh: cls[(j N + i) nlag + q]
// for lag l = lag0 + q.  A lag that a front sweeps takes the maximal rule;
// any other takes the class of the largest probability, or the maximal rule
// when that probability is below the threshold; 0 outside the pair's
// non-null lags (nothing to assemble there).  One thread per pair walks its
// lags; per-class counts of the non-null lags.
__global__ void __launch_bounds__(128) infer_kernel(const float* __restrict__ params, const TriGeom* __restrict__ geo,
                                                    int N, double velP, double velS, double dt, int lag0, int nlag,
                                                    float threshold, unsigned char* __restrict__ cls,
                                                    unsigned long long* __restrict__ counts) {
    __shared__ float w[kParams];
    __shared__ unsigned long long cnt[kC];
    for (int k = threadIdx.x; k < kParams; k += blockDim.x) w[k] = params[k];
    if (threadIdx.x < kC) cnt[threadIdx.x] = 0;
    __syncthreads();
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < (long long)N * N) {
        const int i = (int)(p % N), j = (int)(p / N);
        int llo = -1, lhi = -2;
        pair_band(geo[j], geo[i], velP, velS, dt, lag0, nlag, &llo, &lhi);
        unsigned char* out = cls + p * nlag;
        unsigned c_loc[kC] = {0, 0, 0, 0};
        for (int q = 0; q < nlag; q++) {
            const int l = lag0 + q;
            int c = 0;
            if (llo >= 0 && l >= llo && l <= lhi && front_sweeps(geo[i], geo[j], l, velP, velS, dt)) {
                c = kC - 1;
                c_loc[c]++;
            } else if (llo >= 0 && l >= llo && l <= lhi) {
                float x[kF], h1[kH], h2[kH], z[kC];
                lag_features(x, geo[i], geo[j], l, velP, velS, dt);
                mlp_forward(w, x, h1, h2, z);
                float m = z[0];
                int arg = 0;
                for (int o = 1; o < kC; o++)
                    if (z[o] > m) { m = z[o]; arg = o; }
                float den = 0.0f;
                for (int o = 0; o < kC; o++) den += expf(z[o] - m);
                c = (1.0f / den >= threshold) ? arg : kC - 1;
                c_loc[c]++;
            }
            out[q] = (unsigned char)c;
        }
        for (int o = 0; o < kC; o++)
            if (c_loc[o]) atomicAdd(&cnt[o], (unsigned long long)c_loc[o]);
    }
    __syncthreads();
    if (threadIdx.x < kC && cnt[threadIdx.x]) atomicAdd(counts + threadIdx.x, cnt[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// host side

int selector_features(const MeshData& m, const PhysParams& P, const int* d_samples, long long n, float* d_out,
                      cudaStream_t s) {
    if (n <= 0) return EBEM_OK;
    sample_features_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(m.d_geo, d_samples, n, P.velP, P.velS, P.dt,
                                                                        d_out);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

int selector_sweeps(const MeshData& m, const PhysParams& P, const int* d_samples, long long n, unsigned char* d_out,
                    cudaStream_t s) {
    if (n <= 0) return EBEM_OK;
    sweep_flags_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(m.d_geo, d_samples, n, P.velP, P.velS, P.dt, d_out);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

int selector_labels(const double* d_blocks, long long n, double tol, double scale, const double* d_scales,
                    int* d_labels, cudaStream_t s) {
    if (n <= 0) return EBEM_OK;
    labels_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d_blocks, n, tol * scale, d_scales, d_labels);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
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

int selector_infer(const float* d_params, const MeshData& m, const PhysParams& P, float threshold, int lag0, int nlag,
                   unsigned char* d_cls, long long* h_counts, cudaStream_t s) {
    unsigned long long* d_cnt = nullptr;
    if (ws_malloc(&d_cnt, sizeof(unsigned long long) * kC, s) != cudaSuccess)
        return fail(EBEM_ERR_NOMEM, "inference workspace allocation failed");
    int rc = EBEM_OK;
    cudaError_t e = cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * kC, s);
    const long long NN = (long long)m.nt * m.nt;
    if (e == cudaSuccess) {
        infer_kernel<<<(unsigned)((NN + 127) / 128), 128, 0, s>>>(d_params, m.d_geo, m.nt, P.velP, P.velS, P.dt, lag0,
                                                                   nlag, threshold, d_cls, d_cnt);
        e = cudaGetLastError();
    }
    unsigned long long hc[kC] = {0, 0, 0, 0};
    if (e == cudaSuccess && h_counts) {
        e = cudaMemcpyAsync(hc, d_cnt, sizeof(hc), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        for (int c = 0; c < kC; c++) h_counts[c] = (long long)hc[c];
    }
    if (e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, std::string("selector inference: ") + cudaGetErrorString(e));
    ws_free(d_cnt, s);
    return rc;
}

int assemble_selected(MeshData& m, const PhysParams& P, const int* h_rules, int nclass, const unsigned char* d_cls,
                      int lag0, int nlag, double* d_E, int prec, long long* h_counts, cudaStream_t s) {
    unsigned long long* d_cnt = nullptr;
    if (ws_malloc(&d_cnt, sizeof(unsigned long long) * nclass, s) != cudaSuccess)
        return fail(EBEM_ERR_NOMEM, "assembly workspace allocation failed");
    int rc = EBEM_OK;
    if (cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * nclass, s) != cudaSuccess)
        rc = fail(EBEM_ERR_CUDA, "counter reset failed");
    const size_t n3 = 3 * (size_t)m.nt;
    // class 0 also writes the zeros outside every pair's non-null lags
    for (int c = 0; c < nclass && rc == EBEM_OK; c++) {
        rc = map_nodes_composite(m, h_rules[2 * c], h_rules[2 * c + 1], s);
        if (!rc)
            rc = launch_sa_twopass(m, P, h_rules[2 * c] * h_rules[2 * c + 1], lag0, nlag, 0, m.nt, d_E, n3, n3 * n3, 0,
                                   d_cnt + c, prec, s, d_cls, c);
    }
    std::vector<unsigned long long> hc(nclass, 0ull);
    if (rc == EBEM_OK && h_counts) {
        cudaError_t e = cudaMemcpyAsync(hc.data(), d_cnt, sizeof(unsigned long long) * nclass, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, std::string("selected assembly: ") + cudaGetErrorString(e));
        for (int c = 0; c < nclass; c++) h_counts[c] = (long long)hc[c];
    }
    ws_free(d_cnt, s);
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
