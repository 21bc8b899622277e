// Banded (block-sparse) storage of the Toeplitz blocks E_0..E_{L-1} and the
// time marching on it.
//
// The reference stores every E_l densely (3N x 3N per lag,
// BEMenerg_coreGPU_timeMarching.m:139-147 keeps them in matrixSaved{l};
// BEMenerg_coreSA_timeMarching.m writes each to a .mat file), although a
// (source i, field j) block is zero outside the lags that pass the null test
// of BEMenerg_coreSA_calcMatrixBlock.m:57-61.  That test is monotone in the
// lag, so the non-null lags of a pair form one band [lo, lo + len), and every
// block of the single-layer operator is symmetric.  Here pair p = i N + j
// owns the blocks [off[p], off[p+1]) of one array, one per lag of its band,
// 6 entries (11,12,13,22,23,33) each: 48 bytes per non-null pair-lag instead
// of 72 bytes for every pair and lag (the sphere of 1280 triangles at L = 40
// keeps 26.1 M of 65.5 M pair-lags; the graded screen of 4096 triangles at
// L = 80, 582 M of 1342 M).
//
// The marching (BEMenerg_coreGPU_timeMarching.m:151-169) is unchanged in
// arithmetic content: E_0 is expanded to a dense matrix and factorised once
// (cuSOLVER getrf); step n forms b_n - sum_{l=1}^{min(n, L-1)} E_l phi_{n-l}
// with band_hist_kernel (warps over ranges of a source row's pairs, lanes
// over the (pair, lag) blocks of 32 pairs at a time, the past densities stored
// time-contiguous per field triangle) and solves with the LU factors.
#include "ebem_internal.h"
#include "sa_pair.cuh"

#include <algorithm>

namespace ebem {

// ---------------------------------------------------------------------------
// structure: band of every pair, then the exclusive prefix sum of the lengths

__global__ void band_struct_kernel(const TriGeom* __restrict__ geo, int N, double velP, double velS, double dt, int L,
                                   long long* __restrict__ len, int* __restrict__ lo) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long NN = (long long)N * N;
    if (p > NN) return;
    if (p == NN) {             // the slot that receives the total after the scan
        len[p] = 0;
        return;
    }
    const int i = (int)(p / N), j = (int)(p % N);
    int llo, lhi;
    pair_band(geo[j], geo[i], velP, velS, dt, 0, L, &llo, &lhi);
    len[p] = (llo < 0) ? 0 : (long long)(lhi - llo + 1);
    lo[p] = (llo < 0) ? 0 : llo;
}

constexpr int kScanThreads = 256, kScanPer = 4, kScanBlock = kScanThreads * kScanPer;

// exclusive scan of the per-thread values of one block (Hillis-Steele in shared memory)
__device__ long long block_exclusive_scan(long long v, long long* sh, long long* total) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int d = 1; d < blockDim.x; d <<= 1) {
        const long long add = (t >= d) ? sh[t - d] : 0;
        __syncthreads();
        sh[t] += add;
        __syncthreads();
    }
    const long long incl = sh[t];
    *total = sh[blockDim.x - 1];
    __syncthreads();
    return incl - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(const long long* __restrict__ in, long long n,
                                                                 long long* __restrict__ sums) {
    __shared__ long long sh[kScanThreads];
    const long long base = (long long)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
    long long acc = 0;
    for (int k = 0; k < kScanPer; k++)
        if (base + k < n) acc += in[base + k];
    long long total;
    block_exclusive_scan(acc, sh, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// one block: exclusive scan of the nb block sums in place
__global__ void __launch_bounds__(1024) scan_top_kernel(long long* __restrict__ sums, long long nb) {
    __shared__ long long sh[1024];
    const long long chunk = (nb + blockDim.x - 1) / blockDim.x;
    const long long a = threadIdx.x * chunk, b = (a + chunk < nb) ? a + chunk : nb;
    long long acc = 0;
    for (long long k = a; k < b; k++) acc += sums[k];
    long long total;
    long long run = block_exclusive_scan(acc, sh, &total);
    for (long long k = a; k < b; k++) {
        const long long v = sums[k];
        sums[k] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(long long* __restrict__ data, long long n,
                                                                  const long long* __restrict__ sums) {
    __shared__ long long sh[kScanThreads];
    const long long base = (long long)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
    long long v[kScanPer], acc = 0;
    for (int k = 0; k < kScanPer; k++) {
        v[k] = (base + k < n) ? data[base + k] : 0;
        acc += v[k];
    }
    long long total;
    long long run = block_exclusive_scan(acc, sh, &total) + sums[blockIdx.x];
    for (int k = 0; k < kScanPer; k++)
        if (base + k < n) {
            data[base + k] = run;
            run += v[k];
        }
}

// in-place exclusive prefix sum of n values (n <= 2^30 blocks of 1024);
// returns after the stream has finished it
int exclusive_scan(long long* d, long long n, cudaStream_t s) {
    const long long nb = (n + kScanBlock - 1) / kScanBlock;
    long long* sums = nullptr;
    EBEM_CUDA_TRY(ws_malloc(&sums, nb * sizeof(long long), s));
    scan_sums_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(d, n, sums);
    scan_top_kernel<<<1, 1024, 0, s>>>(sums, nb);
    scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(d, n, sums);
    cudaError_t e = cudaGetLastError();
    ws_free(sums, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("prefix sum: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

int band_structure(const MeshData& m, const PhysParams& P, int L, BandOp* op, cudaStream_t s) {
    const long long NN = (long long)m.nt * m.nt;
    op->N = m.nt;
    op->L = L;
    if (cudaMalloc(&op->off, (NN + 1) * sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&op->lo, NN * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return fail(EBEM_ERR_NOMEM, "band structure allocation failed");
    }
    band_struct_kernel<<<(unsigned)((NN + 1 + 255) / 256), 256, 0, s>>>(m.d_geo, m.nt, P.velP, P.velS, P.dt, L,
                                                                       op->off, op->lo);
    EBEM_CUDA_TRY(cudaGetLastError());
    if (int rc = exclusive_scan(op->off, NN + 1, s)) return rc;
    EBEM_CUDA_TRY(cudaMemcpy(&op->nblocks, op->off + NN, sizeof(long long), cudaMemcpyDeviceToHost));
    if (cudaMalloc(&op->Eb, (size_t)(op->nblocks > 0 ? op->nblocks : 1) * 6 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return fail(EBEM_ERR_NOMEM, "band storage allocation failed (" + std::to_string(op->nblocks * 48) + " bytes)");
    }
    return EBEM_OK;
}

void band_free(BandOp* op) {
    if (op->Eb) cudaFree(op->Eb);
    if (op->off) cudaFree(op->off);
    if (op->lo) cudaFree(op->lo);
    op->Eb = nullptr;
    op->off = nullptr;
    op->lo = nullptr;
}

// ---------------------------------------------------------------------------
// expansion into the dense layout of ebem_assemble_sa (column-major 3N x 3N
// per lag, row 3 source + comp, column 3 field + comp)

__global__ void band_to_dense_kernel(const double* __restrict__ Eb, const long long* __restrict__ off,
                                     const int* __restrict__ lo, int N, int lag0, int nlag, double* __restrict__ E) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)N * N) return;
    const int i = (int)(p / N), j = (int)(p % N);
    const long long b0 = off[p];
    const int len = (int)(off[p + 1] - b0), l0 = lo[p];
    const size_t n3 = 3 * (size_t)N;
    const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int k = 0; k < len; k++) {
        const int l = l0 + k;
        if (l < lag0 || l >= lag0 + nlag) continue;
        const double* B = Eb + (b0 + k) * 6;
        double* dst = E + (size_t)(l - lag0) * n3 * n3 + (3 * (size_t)j) * n3 + 3 * (size_t)i;
        for (int c = 0; c < 3; c++)
            for (int r = 0; r < 3; r++) dst[c * n3 + r] = B[sym[3 * c + r]];
    }
}

int band_to_dense(const BandOp& op, int lag0, int nlag, double* d_E, cudaStream_t s) {
    const size_t n3 = 3 * (size_t)op.N;
    EBEM_CUDA_TRY(cudaMemsetAsync(d_E, 0, n3 * n3 * nlag * sizeof(double), s));
    const long long NN = (long long)op.N * op.N;
    band_to_dense_kernel<<<(unsigned)((NN + 127) / 128), 128, 0, s>>>(op.Eb, op.off, op.lo, op.N, lag0, nlag, d_E);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// marching

// y[3i + c] -= sum_j sum_{l = max(lo,1)}^{min(hi, n)} (E_l)_{ij} phi_{n-l, j}:
// each source row i is split into `split` ranges of its pairs, one warp per
// range, added into y with one atomic per component (the order of those
// additions varies from run to run, as in the dense history product).  The
// pairs of a range are taken 32 at a time:
// each lane loads one pair's offset, first lag and active lag count, a warp
// scan of the counts numbers the chunk's (pair, lag) blocks, and the lanes
// run over those blocks (consecutive lanes read consecutive blocks of the
// band storage), each finding its pair by a binary search over the scanned
// counts.  phiT[(j nT + t) 3 + c].
__global__ void __launch_bounds__(256) band_hist_kernel(const double* __restrict__ Eb, const long long* __restrict__ off,
                                                        const int* __restrict__ lo, int N, int split, int n, int nT,
                                                        const double* __restrict__ phiT, double* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int nchunk = (N + 31) / 32;
    for (long long w = warp; w < (long long)N * split; w += nwarps) {
        const long long i = w / split;
        const int part = (int)(w - i * split);
        const int jb0 = 32 * (int)((long long)nchunk * part / split), jb1 = 32 * (int)((long long)nchunk * (part + 1) / split);
        double a0 = 0, a1 = 0, a2 = 0;
        for (int jb = jb0; jb < jb1; jb += 32) {
            const int jl = jb + lane;
            long long first = 0;          // block index of the pair's first active lag
            int ls = 0, cnt = 0;          // first active lag, active lags
            if (jl < N) {
                const long long p = i * N + jl;
                const long long b0 = off[p];
                const int len = (int)(off[p + 1] - b0), l0 = lo[p];
                ls = max(l0, 1);
                const int le = min(l0 + len - 1, n);
                cnt = max(0, le - ls + 1);
                first = b0 + (ls - l0);
            }
            int incl = cnt;               // inclusive scan of the counts over the lanes
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int t0 = 0; t0 < total; t0 += 32) {      // uniform over the warp: full-mask shuffles
                const int t = t0 + lane;
                int q = 0;                // first lane whose inclusive count exceeds t (31 when t >= total)
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int v = __shfl_sync(0xffffffffu, incl, q + step - 1);
                    if (v <= t) q += step;
                }
                const int excl = __shfl_sync(0xffffffffu, incl, q) - __shfl_sync(0xffffffffu, cnt, q);
                const long long fq = __shfl_sync(0xffffffffu, first, q);
                const int lsq = __shfl_sync(0xffffffffu, ls, q);
                if (t >= total) continue;
                const int k = t - excl, l = lsq + k;
                const double* B = Eb + (fq + k) * 6;
                const double* ph = phiT + ((size_t)(jb + q) * nT + (n - l)) * 3;
                const double p0 = ph[0], p1 = ph[1], p2 = ph[2];
                a0 += B[0] * p0 + B[1] * p1 + B[2] * p2;
                a1 += B[1] * p0 + B[3] * p1 + B[4] * p2;
                a2 += B[2] * p0 + B[4] * p1 + B[5] * p2;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (lane == 0 && (a0 != 0.0 || a1 != 0.0 || a2 != 0.0)) {
            atomicAdd(y + 3 * i, -a0);
            atomicAdd(y + 3 * i + 1, -a1);
            atomicAdd(y + 3 * i + 2, -a2);
        }
    }
}

__global__ void band_e0_kernel(const double* __restrict__ Eb, const long long* __restrict__ off,
                               const int* __restrict__ lo, int N, double* __restrict__ E0) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)N * N) return;
    if (off[p + 1] == off[p] || lo[p] != 0) return;
    const int i = (int)(p / N), j = (int)(p % N);
    const size_t n3 = 3 * (size_t)N;
    const double* B = Eb + off[p] * 6;
    const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int c = 0; c < 3; c++)
        for (int r = 0; r < 3; r++) E0[(3 * (size_t)j + c) * n3 + 3 * (size_t)i + r] = B[sym[3 * c + r]];
}

__global__ void phi_to_time_major_kernel(const double* __restrict__ y, int N, int n, int nT, double* __restrict__ phiT) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * N) return;
    const int j = e / 3, c = e - 3 * j;
    phiT[((size_t)j * nT + n) * 3 + c] = y[e];
}

// phi (device, n3 x nT column-major, i.e. one 3N vector per step) from the
// banded blocks and rhs (device, same layout).
int band_march(const BandOp& op, const double* d_rhs, int nT, double* d_phi, cudaStream_t s) {
    const int N = op.N, n3 = 3 * N;
    double* E0 = nullptr;
    double* phiT = nullptr;
    LuPlan lu;
    int rc = EBEM_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long NN = (long long)N * N;
    if (ws_malloc(&E0, (size_t)n3 * n3 * sizeof(double), s) != cudaSuccess ||
        ws_malloc(&phiT, (size_t)n3 * nT * sizeof(double), s) != cudaSuccess) {
        ws_free(E0, s);
        return fail(EBEM_ERR_NOMEM, "banded marching workspace allocation failed");
    }
    cudaMemsetAsync(E0, 0, (size_t)n3 * n3 * sizeof(double), s);
    band_e0_kernel<<<(unsigned)((NN + 127) / 128), 128, 0, s>>>(op.Eb, op.off, op.lo, N, E0);
    if (cudaGetLastError() != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "E_0 expansion failed");
    if (!rc) rc = lu_plan_create(E0, n3, s, &lu, true);
    ws_free(E0, s);
    // each source row split over enough warps to keep about 48 warps per SM
    // streaming (one warp per row leaves HBM idle when N is small)
    const int nchunk = (N + 31) / 32;
    const int split = (int)std::max<long long>(1, std::min<long long>(nchunk, ((long long)sms * 48 + N - 1) / N));
    const int hist_blocks = (int)std::min<long long>(((long long)N * split + 7) / 8, (long long)sms * 8);
    for (int n = 0; n < nT && !rc; n++) {
        double* y = d_phi + (size_t)n * n3;
        if (cudaMemcpyAsync(y, d_rhs + (size_t)n * n3, (size_t)n3 * sizeof(double), cudaMemcpyDeviceToDevice, s) !=
            cudaSuccess) {
            rc = fail(EBEM_ERR_CUDA, "right-hand side copy failed");
            break;
        }
        if (n > 0 && op.L > 1) band_hist_kernel<<<hist_blocks, 256, 0, s>>>(op.Eb, op.off, op.lo, N, split, n, nT, phiT, y);
        if (cudaGetLastError() != cudaSuccess) {
            rc = fail(EBEM_ERR_CUDA, "banded history failed");
            break;
        }
        if ((rc = lu_plan_solve(&lu, y, 1, s))) break;
        phi_to_time_major_kernel<<<(n3 + 255) / 256, 256, 0, s>>>(y, N, n, nT, phiT);
    }
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "banded marching failed");
    lu_plan_destroy(&lu);
    ws_free(phiT, s);
    return rc;
}

}  // namespace ebem
