// Right-hand side, time marching and post-processing on the device.
//
// Reference (paths relative to the reference project root;
// "CORE/" = functions/BEMenerg_indir/BEMenerg_core/):
//   right-hand side   CORE/BEMenerg_core_calcTn/BEMenerg_core_calcTnBlock.m:28-58,
//                     CORE/BEMenerg_core_calcTn/BEMenerg_core_calcNucleoTn.m:196-244
//   time marching     CORE/BEMenerg_coreGPU/BEMenerg_coreGPU_timeMarching.m:151-169
//                     (LU of E_0 once; phi_n = E_0^{-1}(b_n - sum_l E_l phi_{n-l}))
//   post-processing   functions/BEMenerg_indir/BEMenerg_postProc/BEMenerg_postProcA/
//                     BEMenerg_postProcA_singlePoint.m:21-61, _calcMatrix.m, _calcMatrixBlock.m
#include "ebem_internal.h"
#include "sa_pair.cuh"

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>

namespace ebem {

// ---------------------------------------------------------------------------
// Dirichlet data g(x, t).  Ids 2..7 are the reference's cases
// (BEMenerg_core_calcNucleoTn.m:199-237); 0 and 1 are the data of the screen
// and sphere benchmark problems.
__device__ void datum_value(int id, double velP, double Tfin, const double x[3], double t, double g[3]) {
    g[0] = g[1] = g[2] = 0.0;
    switch (id) {
    case 0: g[2] = t * t * t * t * exp(-2 * t); break;
    case 1: {
        double s = (t > 0) ? sin(2 * kPi * t) : 0.0;
        g[0] = x[0] * s; g[1] = x[1] * s; g[2] = x[2] * s;
    } break;
    case 2: g[2] = 0.5 * t; break;
    case 3: {
        double f = 1.0;
        if (t < kPi / 2) { double s = sin(t); f = s * s * s * s * s; }
        g[2] = f * (x[0] * x[0]);
    } break;
    case 4: case 5: {
        double h = (id == 4) ? 1.0 : 3.0;
        int hat_k = (int)ceil((velP * Tfin) / (2 * h)) - 1;
        double s = 0.0;
        for (int k = 0; k <= hat_k; k++) {
            double a1 = velP * t - 2 * h * k - (h - x[2]);
            double a2 = velP * t - 2 * h * (k + 1) + (h - x[2]);
            double term = a1 * (a1 > 0) - a2 * (a2 > 0);
            s += ((k & 1) ? -1.0 : 1.0) * term;
        }
        g[2] = s;
    } break;
    case 6: { double u = x[0] - 2 + velP * t - 0.475; g[0] = -exp(-20 * u * u); } break;
    case 7: { double u = x[2] + 1 - velP * t; g[2] = -exp(-20 * u * u); } break;
    default: break;
    }
}

__global__ void rhs_kernel(const NodeW* __restrict__ nodes, int N, int n_gh, int datum, double dt, int nT,
                           double velP, double Tfin, double* __restrict__ rhs) {
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * nT) return;
    int t = (int)(idx % N), n = (int)(idx / N);
    double t0 = dt * n, t1 = dt * (n + 1);
    double ris[3] = {0, 0, 0};
    for (int g = 0; g < n_gh; g++) {
        NodeW p = nodes[(size_t)t * n_gh + g];
        double x[3] = {p.x, p.y, p.z}, g1[3], g0[3];
        datum_value(datum, velP, Tfin, x, t1, g1);
        datum_value(datum, velP, Tfin, x, t0, g0);
        for (int c = 0; c < 3; c++) ris[c] = ris[c] + (g1[c] - g0[c]) * p.w;
    }
    for (int c = 0; c < 3; c++) rhs[(size_t)n * 3 * N + 3 * t + c] = (fabs(ris[c]) < 1.0e-14) ? 0.0 : ris[c];
}

// ---------------------------------------------------------------------------
// Datum 8, the reference's manufactured case 'TEST'
// (BEMenerg_core_calcNucleoTn.m:13-132): the boundary value on the screen
// [-1, 1]^2 (z = 0) whose solution is the constant density (1, 1, 1).  The
// reference integrates nucl_1..3 over the square with integral2 for each pair
// of instants (BEMenerg_core_TnTest_classic.m:11-13).  Regrouped by instant,
// nucl_c = f_c(t1) - f_c(t0) with (r = |y - x|, c, s the direction cosines)
//   f_1 = A c^2 + B (3 c^2 - 1) + S + c s (A + 3 B),
//   f_2 = A s^2 + B (3 s^2 - 1) + S + c s (A + 3 B),   f_3 = S - B,
//   A = J_P - J_S, B = I_P - I_S, S = J_S, J_v = H(t - r/v)/(v^2 r),
//   I_v = H(t - r/v)(t^2 - r^2/v^2)/(2 r^3),
// so F_c(x, t) = int f_c(t) dy / (4 pi rho) is computed per instant and the
// right-hand side takes F(t1) - F(t0).  In polar coordinates about x the
// radial integrals are closed forms (a = min(R, c_S t), b = min(R, c_P t)):
//   int_0^R r A = b/c_P^2 - a/c_S^2,   int_0^R r S = a/c_S^2,
//   int_0^R r B = (1/c_S^2 - 1/c_P^2) a/2 + t^2/2 (1/a - 1/b) - (b - a)/(2 c_P^2),
// and the angle is integrated along each side of the square: with d the
// distance of x from the side's line and u the signed position along it from
// the foot of the perpendicular, R = sqrt(d^2 + u^2) and dtheta = d du / R^2.
// The u-range is cut at the foot, at +-d 2^j (geometric grading: the
// integrand's singularities sit at u = +-i d) and where r = c_S t or r = c_P t
// crosses the side; 16-point Gauss-Legendre on each piece.
__constant__ double c_gl16[2][16];      // 16-point Gauss-Legendre on (-1, 1): nodes, weights
constexpr int kTestCuts = 64;

__device__ void test_level(double x1, double x2, double t, double cP, double cS, double F[3]) {
    F[0] = F[1] = F[2] = 0.0;
    if (t <= 0) return;
    const double iP2 = 1 / (cP * cP), iS2 = 1 / (cS * cS), rS = cS * t, rP = cP * t;
    const double cx[4] = {-1, 1, 1, -1}, cy[4] = {-1, -1, 1, 1};
    for (int k = 0; k < 4; k++) {
        const double ax = cx[k] - x1, ay = cy[k] - x2;                 // corner k - x; the side runs to corner k+1
        const double ex = 0.5 * (cx[(k + 1) & 3] - cx[k]), ey = 0.5 * (cy[(k + 1) & 3] - cy[k]);   // unit, length 2
        const double s0 = -(ax * ex + ay * ey);                         // foot at corner + s0 e
        const double fx = ax + s0 * ex, fy = ay + s0 * ey;              // foot - x, perpendicular to e
        const double d = fx * ey - fy * ex;                             // > 0: the square runs counterclockwise about x
        const double ulo = -s0, uhi = 2 - s0;
        double cut[kTestCuts];
        int nc = 0;
        auto add = [&](double u) {
            if (u > ulo && u < uhi && nc < kTestCuts - 1) cut[nc++] = u;
        };
        cut[nc++] = ulo;
        add(0.0);
        for (int q = 0; q < 2; q++) {
            const double rho = q ? rP : rS;
            if (rho > d) {
                const double w = sqrt((rho - d) * (rho + d));
                add(-w);
                add(w);
            }
        }
        const double umax = fmax(-ulo, uhi);
        for (int j = 0; j < 26 && d * (double)(1 << j) < umax; j++) {
            add(-d * (double)(1 << j));
            add(d * (double)(1 << j));
        }
        cut[nc++] = uhi;
        for (int i = 1; i < nc; i++)                                   // insertion sort
            for (int j = i; j > 0 && cut[j] < cut[j - 1]; j--) {
                const double tmp = cut[j];
                cut[j] = cut[j - 1];
                cut[j - 1] = tmp;
            }
        for (int q = 0; q + 1 < nc; q++) {
            const double h = 0.5 * (cut[q + 1] - cut[q]), mid = 0.5 * (cut[q + 1] + cut[q]);
            if (h <= 0) continue;
            for (int ia = 0; ia < 16; ia++) {
                const double u = mid + h * c_gl16[0][ia];
                const double R2 = d * d + u * u, R = sqrt(R2);
                const double w = h * c_gl16[1][ia] * d / R2;           // dtheta
                const double cs = (fx + u * ex) / R, sn = (fy + u * ey) / R;
                const double a = fmin(R, rS), b = fmin(R, rP);
                const double RS = a * iS2, RA = b * iP2 - a * iS2;
                double RB = 0.5 * (iS2 - iP2) * a;
                if (b > a) RB += 0.5 * t * t * (1 / a - 1 / b) - 0.5 * (b - a) * iP2;
                const double mixd = cs * sn * (RA + 3 * RB);
                F[0] += w * (cs * cs * RA + (3 * cs * cs - 1) * RB + RS + mixd);
                F[1] += w * (sn * sn * RA + (3 * sn * sn - 1) * RB + RS + mixd);
                F[2] += w * (RS - RB);
            }
        }
    }
}

// S_k[t] = sum_g w_g F(x_g, t_k) / (4 pi rho), k = 0..nT, one thread per (triangle, level).
__global__ void rhs_test_level_kernel(const NodeW* __restrict__ nodes, int N, int n_gh, double dt, int nT, double cP,
                                      double cS, double c4pirho, double* __restrict__ S) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * (nT + 1)) return;
    const int t = (int)(idx % N), k = (int)(idx / N);
    double acc[3] = {0, 0, 0};
    for (int g = 0; g < n_gh; g++) {
        const NodeW p = nodes[(size_t)t * n_gh + g];
        double F[3];
        test_level(p.x, p.y, dt * k, cP, cS, F);
        for (int c = 0; c < 3; c++) acc[c] += F[c] * p.w;
    }
    for (int c = 0; c < 3; c++) S[((size_t)k * N + t) * 3 + c] = acc[c] / c4pirho;
}

// b_n = S_{n+1} - S_n, entries below 1e-14 set to 0 (BEMenerg_core_calcTnBlock.m:50-51).
__global__ void rhs_test_diff_kernel(const double* __restrict__ S, int N, int nT, double* __restrict__ rhs) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 3LL * N * nT) return;
    const int n = (int)(idx / (3LL * N));
    const size_t e = (size_t)(idx % (3LL * N));
    const double v = S[(size_t)(n + 1) * 3 * N + e] - S[(size_t)n * 3 * N + e];
    rhs[idx] = (fabs(v) < 1.0e-14) ? 0.0 : v;
}

static void gauss_legendre16(double x[16], double w[16]) {
    // Newton's iteration on P_16 from cos(pi (i + 3/4) / (n + 1/2)).
    const int n = 16;
    for (int i = 0; i < n; i++) {
        double z = cos(kPi * (i + 0.75) / (n + 0.5)), dp = 1;
        for (int it = 0; it < 100; it++) {
            double p0 = 1, p1 = z;
            for (int k = 2; k <= n; k++) {
                const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1);
            const double dz = p1 / dp;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        x[i] = z;
        w[i] = 2 / ((1 - z * z) * dp * dp);
    }
}

static int launch_rhs_test(const MeshData& m, const PhysParams& P, int n_gh, double* d_rhs, cudaStream_t s) {
    double gl[2][16];
    gauss_legendre16(gl[0], gl[1]);
    EBEM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_gl16, gl, sizeof gl, 0, cudaMemcpyHostToDevice, s));
    double* d_S = nullptr;
    const size_t nS = 3 * (size_t)m.nt * (P.nT + 1);
    EBEM_CUDA_TRY(ws_malloc(&d_S, nS * sizeof(double), s));
    const int threads = 128;
    const long long lv = (long long)m.nt * (P.nT + 1), nb = 3LL * m.nt * P.nT;
    rhs_test_level_kernel<<<(unsigned)((lv + threads - 1) / threads), threads, 0, s>>>(
        m.d_nodes, m.nt, n_gh, P.dt, P.nT, P.velP, P.velS, 4 * kPi * P.rho, d_S);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        rhs_test_diff_kernel<<<(unsigned)((nb + threads - 1) / threads), threads, 0, s>>>(d_S, m.nt, P.nT, d_rhs);
        e = cudaGetLastError();
    }
    ws_free(d_S, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("TEST right-hand side: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

int launch_rhs(const MeshData& m, const PhysParams& P, int n_gh, int datum, double* d_rhs, cudaStream_t s) {
    if (datum == 8) return launch_rhs_test(m, P, n_gh, d_rhs, s);
    long long total = (long long)m.nt * P.nT;
    int threads = 128;
    rhs_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(m.d_nodes, m.nt, n_gh, datum, P.dt,
                                                                              P.nT, P.velP, P.dt * P.nT, d_rhs);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// History product y -= A x, A column-major n3 x K (the concatenated blocks
// [E_1 E_2 ... E_M]), x contiguous (phi_{n-1}, phi_{n-2}, ... thanks to the
// reversed storage of the density).  HBM-bound: each block streams a chunk
// of columns for a tile of rows, keeps per-thread partial sums of
// EBEM_GEMV_RPT rows and adds them to y with one atomic per row.
#define EBEM_GEMV_THREADS 256
#define EBEM_GEMV_RPT 8

__global__ void __launch_bounds__(EBEM_GEMV_THREADS)
hist_gemv_kernel(const double* __restrict__ A, int n3, long long K, long long cols_per_block,
                 const double* __restrict__ x, double* __restrict__ y) {
    const int tile_rows = EBEM_GEMV_THREADS * EBEM_GEMV_RPT;
    const int row0 = blockIdx.y * tile_rows + threadIdx.x;
    const long long k0 = (long long)blockIdx.x * cols_per_block;
    long long k1 = k0 + cols_per_block;
    if (k1 > K) k1 = K;
    double acc[EBEM_GEMV_RPT];
#pragma unroll
    for (int i = 0; i < EBEM_GEMV_RPT; i++) acc[i] = 0.0;
    long long k = k0;
    for (; k + 1 < k1; k += 2) {
        const double xa = x[k], xb = x[k + 1];
        const double* ca = A + k * (long long)n3;
        const double* cb = ca + n3;
#pragma unroll
        for (int i = 0; i < EBEM_GEMV_RPT; i++) {
            int r = row0 + i * EBEM_GEMV_THREADS;
            if (r < n3) acc[i] += __ldg(ca + r) * xa + __ldg(cb + r) * xb;
        }
    }
    if (k < k1) {
        const double xa = x[k];
        const double* ca = A + k * (long long)n3;
#pragma unroll
        for (int i = 0; i < EBEM_GEMV_RPT; i++) {
            int r = row0 + i * EBEM_GEMV_THREADS;
            if (r < n3) acc[i] += __ldg(ca + r) * xa;
        }
    }
#pragma unroll
    for (int i = 0; i < EBEM_GEMV_RPT; i++) {
        int r = row0 + i * EBEM_GEMV_THREADS;
        if (r < n3 && acc[i] != 0.0) atomicAdd(y + r, -acc[i]);
    }
}

int launch_hist_gemv(const double* A, int n3, long long K, const double* x, double* y, int sm_count, cudaStream_t s) {
    if (K <= 0) return EBEM_OK;
    const int tile_rows = EBEM_GEMV_THREADS * EBEM_GEMV_RPT;
    int row_tiles = (n3 + tile_rows - 1) / tile_rows;
    // about four resident blocks per SM in total, at least 64 columns each
    long long want = (long long)sm_count * 4 / row_tiles;
    if (want < 1) want = 1;
    long long cpb = (K + want - 1) / want;
    if (cpb < 64) cpb = 64;
    long long nblk = (K + cpb - 1) / cpb;
    dim3 grid((unsigned)nblk, (unsigned)row_tiles);
    hist_gemv_kernel<<<grid, EBEM_GEMV_THREADS, 0, s>>>(A, n3, K, cpb, x, y);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

__global__ void copy_reverse_kernel(const double* __restrict__ src, double* __restrict__ dst, int n3, int nT, int to_rev) {
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n3 * nT) return;
    int r = (int)(idx % n3), n = (int)(idx / n3);
    if (to_rev) dst[(size_t)(nT - 1 - n) * n3 + r] = src[idx];
    else dst[idx] = src[(size_t)(nT - 1 - n) * n3 + r];
}

#define CUSOLVER_TRY(expr)                                                                        \
    do {                                                                                          \
        cusolverStatus_t _st = (expr);                                                            \
        if (_st != CUSOLVER_STATUS_SUCCESS) {                                                     \
            rc = fail(EBEM_ERR_CUDA, std::string(#expr) + " failed with status " + std::to_string((int)_st)); \
            goto done;                                                                            \
        }                                                                                         \
    } while (0)

// ---------------------------------------------------------------------------
// Library handles per host thread and device.  A thread-local table of plain
// pointers: nothing is destroyed at thread or process exit (the driver
// reclaims the handles with the context), so no handle outlives its CUDA
// context in a destructor.
namespace {
constexpr int kHandleDevices = 64;
struct ThreadHandles {
    cusolverDnHandle_t sol[kHandleDevices];
    cublasHandle_t blas[kHandleDevices];
    unsigned sol_gen[kHandleDevices], blas_gen[kHandleDevices];   // device generation at creation
};
thread_local ThreadHandles t_handles = {};

int handle_device(int* dev) {
    if (cudaGetDevice(dev) != cudaSuccess || *dev < 0 || *dev >= kHandleDevices) {
        cudaGetLastError();
        return fail(EBEM_ERR_CUDA, "no usable current device for a library handle");
    }
    return EBEM_OK;
}
}  // namespace

int solver_handle(cudaStream_t s, cusolverDnHandle_t* h) {
    int dev = 0;
    if (int rc = handle_device(&dev)) return rc;
    cusolverDnHandle_t& c = t_handles.sol[dev];
    const unsigned gen = device_generation(dev);
    if (c && t_handles.sol_gen[dev] != gen) c = nullptr;      // released device state: abandoned
    if (!c) {
        if (cusolverDnCreate(&c) != CUSOLVER_STATUS_SUCCESS) {
            c = nullptr;
            return fail(EBEM_ERR_CUDA, "cuSOLVER handle creation failed");
        }
        t_handles.sol_gen[dev] = gen;
    }
    if (cusolverDnSetStream(c, s) != CUSOLVER_STATUS_SUCCESS) return fail(EBEM_ERR_CUDA, "cuSOLVER stream binding failed");
    *h = c;
    return EBEM_OK;
}

int blas_handle(cudaStream_t s, cublasHandle_t* h) {
    int dev = 0;
    if (int rc = handle_device(&dev)) return rc;
    cublasHandle_t& c = t_handles.blas[dev];
    const unsigned gen = device_generation(dev);
    if (c && t_handles.blas_gen[dev] != gen) c = nullptr;     // released device state: abandoned
    if (!c) {
        if (cublasCreate(&c) != CUBLAS_STATUS_SUCCESS) {
            c = nullptr;
            return fail(EBEM_ERR_CUDA, "cuBLAS handle creation failed");
        }
        t_handles.blas_gen[dev] = gen;
    }
    if (cublasSetStream(c, s) != CUBLAS_STATUS_SUCCESS) return fail(EBEM_ERR_CUDA, "cuBLAS stream binding failed");
    *h = c;
    return EBEM_OK;
}

void release_thread_handles(int dev) {
    if (dev < 0 || dev >= kHandleDevices) return;
    if (!t_handles.sol[dev] && !t_handles.blas[dev]) return;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(dev);
    if (t_handles.sol[dev]) cusolverDnDestroy(t_handles.sol[dev]);
    if (t_handles.blas[dev]) cublasDestroy(t_handles.blas[dev]);
    t_handles.sol[dev] = nullptr;
    t_handles.blas[dev] = nullptr;
    if (prev >= 0) cudaSetDevice(prev);
    cudaGetLastError();
}

// phi (device, column-major n3 x nT) from E (device, n3 x n3 x L) and rhs
// (device, n3 x nT): E_0^{-1} once, then per step the history product and
// one product with E_0^{-1}.
int march_device(const double* dE, int n3, int L, const double* drhs, int nT, double* dphi, cudaStream_t s,
                 int factor) {
    int rc = EBEM_OK, dev = 0, sms = 148;
    double* rev = nullptr;
    LuPlan lu;
    const size_t nn = (size_t)n3 * n3;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (ws_malloc(&rev, (size_t)n3 * nT * sizeof(double), s) != cudaSuccess)
        return fail(EBEM_ERR_NOMEM, "time-marching workspace allocation failed");
    rc = lu_plan_create(dE, n3, s, &lu, true, factor == EBEM_FACTOR_CHOLESKY);
    if (!rc) {
        // density in reversed time order: phi_n at column nT-1-n, so that
        // phi_{n-1}, phi_{n-2}, ... are contiguous for the history product
        const long long tot = (long long)n3 * nT;
        copy_reverse_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(drhs, rev, n3, nT, 1);
        if (cudaGetLastError() != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "rhs copy failed");
        for (int n = 0; n < nT && !rc; n++) {
            double* y = rev + (size_t)(nT - 1 - n) * n3;
            const int M = (n < L - 1) ? n : L - 1;
            if (M > 0) rc = launch_hist_gemv(dE + nn, n3, (long long)n3 * M, rev + (size_t)(nT - n) * n3, y, sms, s);
            if (!rc) rc = lu_plan_solve(&lu, y, 1, s);
        }
        if (!rc) {
            copy_reverse_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(rev, dphi, n3, nT, 0);
            if (cudaGetLastError() != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "density copy failed");
        }
        if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "time marching failed");
    }
    lu_plan_destroy(&lu);
    ws_free(rev, s);
    return rc;
}

// ---------------------------------------------------------------------------
// A^{-1} of one matrix kept on the device (the E_0 solve of the marching,
// also for callers that drive the steps themselves): LU with partial
// pivoting (getrf), then getrs on the identity, whose n right-hand sides run
// as matrix-matrix triangular solves.
__global__ void set_identity_kernel(double* __restrict__ a, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[(size_t)i * n + i] = 1.0;
}

// (A + A^T) / 2 in place (column-major n x n).
__global__ void symmetrize_kernel(double* __restrict__ a, int n) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(idx % n), j = (int)(idx / n);
    if (idx >= (long long)n * n || i >= j) return;
    const double v = 0.5 * (a[(size_t)j * n + i] + a[(size_t)i * n + j]);
    a[(size_t)j * n + i] = v;
    a[(size_t)i * n + j] = v;
}

int lu_plan_create(const double* dA, int n, cudaStream_t s, LuPlan* plan, bool pooled, bool cholesky) {
    int rc = EBEM_OK;
    int lwork = 0, hinfo = 0;
    double *lu = nullptr, *work = nullptr;
    int *ipiv = nullptr, *info = nullptr;
    const size_t nn = (size_t)n * n;
    cusolverDnHandle_t h = nullptr;
    plan->n = n;
    plan->pooled = pooled;
    plan->st = s;
    if ((rc = solver_handle(s, &h))) return rc;
    cudaError_t e = pooled ? ws_malloc(&plan->inv, nn * sizeof(double), s) : cudaMalloc(&plan->inv, nn * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        plan->inv = nullptr;
        return fail(EBEM_ERR_NOMEM, "inverse allocation failed");
    }
    if (ws_malloc(&lu, nn * sizeof(double), s) != cudaSuccess || ws_malloc(&ipiv, n * sizeof(int), s) != cudaSuccess ||
        ws_malloc(&info, sizeof(int), s) != cudaSuccess) {
        rc = fail(EBEM_ERR_NOMEM, "LU workspace allocation failed");
        goto done;
    }
    if (cudaMemcpyAsync(lu, dA, nn * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        rc = fail(EBEM_ERR_CUDA, "matrix copy failed");
        goto done;
    }
    if (cholesky) {
        symmetrize_kernel<<<(unsigned)(((long long)n * n + 255) / 256), 256, 0, s>>>(lu, n);
        CUSOLVER_TRY(cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, n, lu, n, &lwork));
    } else {
        CUSOLVER_TRY(cusolverDnDgetrf_bufferSize(h, n, n, lu, n, &lwork));
    }
    if (ws_malloc(&work, (size_t)(lwork > 0 ? lwork : 1) * sizeof(double), s) != cudaSuccess) {
        rc = fail(EBEM_ERR_NOMEM, "LU workspace allocation failed");
        goto done;
    }
    if (cholesky) CUSOLVER_TRY(cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, n, lu, n, work, lwork, info));
    else CUSOLVER_TRY(cusolverDnDgetrf(h, n, n, lu, n, work, ipiv, info));
    if (cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        rc = fail(EBEM_ERR_CUDA, "LU factorisation failed");
        goto done;
    }
    if (hinfo != 0) {
        rc = cholesky ? fail(EBEM_ERR_SINGULAR, "the symmetric part of the matrix is not positive definite (leading "
                                                "minor " + std::to_string(hinfo) + ")")
                      : fail(EBEM_ERR_SINGULAR, "matrix is singular (zero pivot " + std::to_string(hinfo) + ")");
        goto done;
    }
    if (cudaMemsetAsync(plan->inv, 0, nn * sizeof(double), s) != cudaSuccess) {
        rc = fail(EBEM_ERR_CUDA, "inverse initialisation failed");
        goto done;
    }
    set_identity_kernel<<<(n + 255) / 256, 256, 0, s>>>(plan->inv, n);
    if (cudaGetLastError() != cudaSuccess) {
        rc = fail(EBEM_ERR_CUDA, "inverse initialisation failed");
        goto done;
    }
    if (cholesky) CUSOLVER_TRY(cusolverDnDpotrs(h, CUBLAS_FILL_MODE_LOWER, n, n, lu, n, plan->inv, n, info));
    else CUSOLVER_TRY(cusolverDnDgetrs(h, CUBLAS_OP_N, n, n, lu, n, ipiv, plan->inv, n, info));
done:
    ws_free(lu, s);
    ws_free(work, s);
    ws_free(ipiv, s);
    ws_free(info, s);
    return rc;
}

// b (n x nrhs, device, overwritten) = A^{-1} b.
int lu_plan_solve(LuPlan* plan, double* db, int nrhs, cudaStream_t s) {
    cublasHandle_t hb = nullptr;
    if (int rc = blas_handle(s, &hb)) return rc;
    const int n = plan->n;
    const size_t cnt = (size_t)n * nrhs;
    double* tmp = nullptr;
    if (ws_malloc(&tmp, cnt * sizeof(double), s) != cudaSuccess) return fail(EBEM_ERR_NOMEM, "solve workspace allocation failed");
    const double one = 1.0, zero = 0.0;
    const cublasStatus_t st =
        nrhs == 1 ? cublasDgemv(hb, CUBLAS_OP_N, n, n, &one, plan->inv, n, db, 1, &zero, tmp, 1)
                  : cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, n, nrhs, n, &one, plan->inv, n, db, n, &zero, tmp, n);
    cudaError_t e = st == CUBLAS_STATUS_SUCCESS ? cudaMemcpyAsync(db, tmp, cnt * sizeof(double), cudaMemcpyDeviceToDevice, s)
                                                : cudaSuccess;
    ws_free(tmp, s);
    if (st != CUBLAS_STATUS_SUCCESS) return fail(EBEM_ERR_CUDA, "product with the inverse failed (cuBLAS status " + std::to_string((int)st) + ")");
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("solve copy: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

void lu_plan_destroy(LuPlan* plan) {
    if (plan->inv) {
        if (plan->pooled) ws_free(plan->inv, plan->st);
        else cudaFree(plan->inv);
    }
    plan->inv = nullptr;
}

// ---------------------------------------------------------------------------
// Post-processing (closed form): u(x, t) = sum_{k=1}^{nHat} (M(t - (k-1) dt)
// - M(t - k dt)) phi_k + M(t - nHat dt) phi_{nHat+1}, nHat = ceil(t/dt) - 1,
// M(tau) the single-point combined kernel integral over each triangle
// (BEMenerg_postProcA_singlePoint.m:21-61), divided by 4 pi rho and cleaned
// below 1e-14 (BEMenerg_postProcA_calcMatrix.m:103).  One thread per
// (triangle, point, time); consecutive lanes take consecutive triangles of
// one (point, time), reduce over the warp and add to u with one atomic per
// component.
__device__ __forceinline__ void pp_block(double M[6], const TriGeom& F, const NodeW& x, double tau, double velP,
                                         double velS, double c4) {
    level_value(M, 1, velP, velS, tau, F, &x, 1);
#pragma unroll
    for (int e = 0; e < 6; e++) {
        double v = M[e] / c4;
        M[e] = (fabs(v) < 1.0e-14) ? 0.0 : v;
    }
}

__device__ __forceinline__ void sym_mv_add(double acc[3], const double M[6], const double* ph, double sgn) {
    acc[0] += sgn * (M[0] * ph[0] + M[1] * ph[1] + M[2] * ph[2]);
    acc[1] += sgn * (M[1] * ph[0] + M[3] * ph[1] + M[4] * ph[2]);
    acc[2] += sgn * (M[2] * ph[0] + M[4] * ph[1] + M[5] * ph[2]);
}

// The instants at which M(tau) of triangle F seen from x is zero without
// evaluating it: the P front (radius velP tau) has not reached the triangle.
// M is zero when the closed form's case split finds no front at the node
// (T_NONE), which needs velP tau <= sqrt(zeta^2 + dMIN^2) as the
// projection computes them; that is at least the distance from x to the
// triangle less the projection's tolerances (the plane distance snapped to
// 0 below 1e-6, the inside test's 1e-6 on the barycentrics, the edge foot
// tests' 1e-6, which can take a foot up to 1e-6 / |edge| <= 1e-6 maxL / (2
// area) beyond an end), and that distance is at least the centroid distance
// less the longest edge.  pp_reach returns that bound less a margin of half
// the longest edge on top of the tolerances; an instant with velP tau below
// it is skipped.  Rounded explicitly (no contraction): the evaluation pass
// and the contraction must take the same decision for every instant.
__device__ __forceinline__ double pp_reach(const TriGeom& F, const NodeW& x) {
    const double d0 = __dsub_rn(x.x, F.ctr[0]), d1 = __dsub_rn(x.y, F.ctr[1]), d2 = __dsub_rn(x.z, F.ctr[2]);
    const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
    const double tol = __dadd_rn(__dadd_rn(__dmul_rn(0.5, F.maxL), 1.0e-5),
                                 __dadd_rn(__ddiv_rn(__dmul_rn(1.0e-6, F.maxL), F.area), __dmul_rn(1.0e-12, r)));
    return __dsub_rn(__dsub_rn(r, F.maxL), tol);     // a degenerate triangle (area 0) gives -inf: never skipped
}

__device__ __forceinline__ bool pp_before_front(double reach, double velP, double tau) {
    return __dmul_rn(velP, tau) < reach;
}

// pp_block, or zero at an instant before the P front reaches the triangle.
__device__ __forceinline__ void pp_block_or_zero(double M[6], const TriGeom& F, const NodeW& x, double reach,
                                                 double tau, double velP, double velS, double c4) {
    if (pp_before_front(reach, velP, tau)) {
#pragma unroll
        for (int e = 0; e < 6; e++) M[e] = 0.0;
    } else {
        pp_block(M, F, x, tau, velP, velS, c4);
    }
}

// At most 128 registers (4 blocks of 128 threads per SM; 254 without the
// cap): 40 scattered times at 256 points on the 1280-triangle sphere 37.1 ->
// 27.6 ms.
__global__ void __launch_bounds__(128, 4) pp_sa_kernel(const TriGeom* __restrict__ geo, int N, const double* __restrict__ pts,
                                                    int npts, const double* __restrict__ times, int ntimes,
                                                    const double* __restrict__ phi, int nT, double velP, double velS,
                                                    double dt, double c4, double* __restrict__ u) {
    // one thread per (triangle j, point p, time q), j fastest: a warp shares
    // (p, q) unless it straddles two of them
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long NP = (long long)N * npts;
    const bool valid = idx < NP * ntimes;
    const int q = valid ? (int)(idx / NP) : 0;
    const long long r = valid ? idx - (long long)q * NP : 0;
    const int j = (int)(r % N), p = (int)(r / N);
    NodeW x;
    x.x = pts[3 * p]; x.y = pts[3 * p + 1]; x.z = pts[3 * p + 2]; x.w = 1.0;
    const TriGeom& F = geo[j];
    const size_t n3 = 3 * (size_t)N;
    const double t = times[q];
    double acc[3] = {0, 0, 0};
    if (valid && t > 0) {
        int nHat = (int)ceil(t / dt) - 1;
        if (nHat > nT - 1) nHat = nT - 1;
        double Mc[6], Mn[6];
        const double reach = pp_reach(F, x);
        pp_block_or_zero(Mc, F, x, reach, t, velP, velS, c4);
        for (int k = 1; k <= nHat; k++) {
            pp_block_or_zero(Mn, F, x, reach, __dsub_rn(t, __dmul_rn((double)k, dt)), velP, velS, c4);   // no fused multiply-add
            const double* ph = phi + (size_t)(k - 1) * n3 + 3 * (size_t)j;
            double D[6];
#pragma unroll
            for (int e = 0; e < 6; e++) { D[e] = Mc[e] - Mn[e]; Mc[e] = Mn[e]; }
            sym_mv_add(acc, D, ph, 1.0);
        }
        sym_mv_add(acc, Mc, phi + (size_t)nHat * n3 + 3 * (size_t)j, 1.0);
    }
    double sum[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        sum[c] = v;
    }
    // a warp may straddle two (point, time) outputs: then every lane adds its own value
    const long long o_me = (long long)q * npts + p;
    const long long o_first = __shfl_sync(0xffffffffu, o_me, 0), o_last = __shfl_sync(0xffffffffu, o_me, 31);
    const int v_last = __shfl_sync(0xffffffffu, valid ? 1 : 0, 31);
    if (o_first == o_last && v_last) {
        if ((threadIdx.x & 31) == 0)
            for (int c = 0; c < 3; c++) atomicAdd(u + o_me * 3 + c, sum[c]);
    } else if (valid) {
        for (int c = 0; c < 3; c++) atomicAdd(u + o_me * 3 + c, acc[c]);
    }
}

// Shared instants.  By parts the sum above is
//   u(x, t_q) = M(t_q) phi_0 + sum_{k=1}^{nHat} M(t_q - k dt) (phi_k - phi_{k-1}),
// and for output times on the time grid the instants t_q - k dt of different
// (q, k) coincide.  The instants are formed on the host exactly as the
// per-time kernel forms them (k dt rounded, then subtracted from t_q, no
// fused multiply-add: the closed form's case selection is discontinuous
// where a front radius equals the point's distance from the plane, so an
// instant one unit in the last place off can change M there), deduplicated
// by value; pp_inst_count_kernel finds, per (point, triangle) row, the first
// instant that the P front reaches (the instants are sorted, so the skipped
// ones come first), a prefix sum numbers the evaluated items, and
// pp_inst_level_kernel evaluates M once per (triangle, point, distinct
// evaluated instant); pp_inst_sum_kernel contracts, one block per (time,
// point).
__global__ void __launch_bounds__(128) pp_inst_count_kernel(const TriGeom* __restrict__ geo, int N,
                                                            const double* __restrict__ pts, int p0, int np, int nu,
                                                            const double* __restrict__ taus, double velP,
                                                            long long* __restrict__ cnt, int* __restrict__ first) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long rows = (long long)N * np;
    if (r == 0) cnt[rows] = 0;            // becomes the total after the exclusive scan
    if (r >= rows) return;
    const int pl = (int)(r / N), j = (int)(r - (long long)pl * N);
    const int p = p0 + pl;
    NodeW x;
    x.x = pts[3 * p]; x.y = pts[3 * p + 1]; x.z = pts[3 * p + 2]; x.w = 1.0;
    const double reach = pp_reach(geo[j], x);
    // the skip test is monotone in the sorted instants: first instant not skipped
    int lo = 0, hi = nu;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pp_before_front(reach, velP, taus[mid])) lo = mid + 1;
        else hi = mid;
    }
    first[r] = lo;
    cnt[r] = nu - lo;
}

__global__ void __launch_bounds__(128, 6) pp_inst_level_kernel(const TriGeom* __restrict__ geo, int N,
                                                            const double* __restrict__ pts, int p0, int np, int nu,
                                                            const double* __restrict__ taus, double velP, double velS,
                                                            double c4, const long long* __restrict__ off,
                                                            const int* __restrict__ first, long long total,
                                                            double* __restrict__ Mbuf) {
    // Items numbered row by row ((point, triangle) rows, triangles fastest),
    // the evaluated instants of a row consecutive: the lanes of a warp take
    // neighbouring instants of one (triangle, point), which mostly meet the
    // fronts in the same way, and 32 evaluations whatever the skipped
    // instants (97 % of them on the 1280-triangle sphere with 256 points;
    // warps over all the instants of a row mixed skipped and evaluated lanes:
    // 4.6 ms there).  Triangles fastest over all instants took more distinct
    // branches (1.34 against 0.97 ms for 64 points x 40 grid times on 320
    // triangles before the skip); a buffer ordered (point, triangle,
    // instant), which makes the stores contiguous, made the contraction's
    // loads strided (1.8 -> 5.8 ms on 1280).  At most 80 registers (6 blocks
    // of 128 threads per SM): with 200 registers 2 blocks fitted, 1.5 warps
    // per scheduler waited on the FP64 dependencies of one evaluation, and
    // the spills this cap adds cost less than the occupancy gains (11.7 ->
    // 7.0 ms on 1280 triangles before the skip; 128 registers: 7.4 ms).
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    // the row: last r with off[r] <= idx (off: exclusive prefix sums of the
    // rows' counts, off[rows] = total; an empty row shares its offset with
    // the next one)
    const long long rows = (long long)N * np;
    long long lo = 0, hi = rows;
    while (hi - lo > 1) {
        const long long mid = (lo + hi) >> 1;
        if (off[mid] <= idx) lo = mid;
        else hi = mid;
    }
    const long long r = lo;
    const int ui = first[r] + (int)(idx - off[r]);
    const int pl = (int)(r / N), j = (int)(r - (long long)pl * N);
    const int p = p0 + pl;
    NodeW x;
    x.x = pts[3 * p]; x.y = pts[3 * p + 1]; x.z = pts[3 * p + 2]; x.w = 1.0;
    double M[6];
    pp_block(M, geo[j], x, taus[ui], velP, velS, c4);
    double* dst = Mbuf + (((size_t)pl * nu + ui) * N + j) * 6;
#pragma unroll
    for (int e = 0; e < 6; e++) dst[e] = M[e];
}

// Blocks of 128 threads, or of 1024 when there are too few (time, point)
// pairs to fill the GPU.
__global__ void __launch_bounds__(1024) pp_inst_sum_kernel(const double* __restrict__ Mbuf, const TriGeom* __restrict__ geo,
                                                          int N, const double* __restrict__ pts, int p0, int np, int nu,
                                                          const double* __restrict__ taus, double velP,
                                                          const int* __restrict__ tab, int kmax,
                                                          const int* __restrict__ nhat, int npts,
                                                          const double* __restrict__ phi, double* __restrict__ u) {
    const int q = blockIdx.x / np, pl = blockIdx.x - q * np;
    const int nh = nhat[q];
    const int* tq = tab + (size_t)q * kmax;
    const size_t n3 = 3 * (size_t)N;
    const int p = p0 + pl;
    NodeW x;
    x.x = pts[3 * p]; x.y = pts[3 * p + 1]; x.z = pts[3 * p + 2]; x.w = 1.0;
    double acc[3] = {0, 0, 0};
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const double reach = pp_reach(geo[j], x);
        for (int k = 0; k <= nh; k++) {
            if (pp_before_front(reach, velP, taus[tq[k]])) continue;    // M = 0, not stored
            const double* Mv = Mbuf + (((size_t)pl * nu + tq[k]) * N + j) * 6;
            const double* pk = phi + (size_t)k * n3 + 3 * (size_t)j;
            double d[3] = {pk[0], pk[1], pk[2]};
            if (k > 0) {
                d[0] -= pk[-(long long)n3];
                d[1] -= pk[1 - (long long)n3];
                d[2] -= pk[2 - (long long)n3];
            }
            double Ml[6];
#pragma unroll
            for (int e = 0; e < 6; e++) Ml[e] = Mv[e];
            sym_mv_add(acc, Ml, d, 1.0);
        }
    }
    __shared__ double red[3][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[c][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) v += red[threadIdx.x][i];
        u[((size_t)q * npts + p0 + pl) * 3 + threadIdx.x] = v;
    }
}

// The shared-instant path of launch_pp_sa; returns 1 (nothing done) when the
// instants barely repeat (times off the grid), where the per-time kernel
// does the same work without the buffer.
static int launch_pp_sa_shared(const MeshData& m, const PhysParams& P, const double* d_phi, const double* d_pts,
                               int npts, const double* h_times, int ntimes, double* d_u, cudaStream_t s) {
    std::vector<int> nh(ntimes);
    int kmax = 1;
    long long terms = 0;
    std::vector<double> taus;
    for (int q = 0; q < ntimes; q++) {
        const double t = h_times[q];
        int n = -1;
        if (t > 0) {
            n = (int)std::ceil(t / P.dt) - 1;
            if (n > P.nT - 1) n = P.nT - 1;
        }
        nh[q] = n;
        kmax = std::max(kmax, n + 1);
        terms += n + 1;
        for (int k = 0; k <= n; k++) {
            volatile double a = (double)k * P.dt;      // rounded product, then the difference
            taus.push_back(t - a);
        }
    }
    std::vector<double> uniq(taus);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    const int nu = (int)uniq.size();
    if (nu == 0 || 2LL * nu > terms) return 1;
    std::vector<int> tab((size_t)ntimes * kmax, 0);
    {
        size_t c = 0;
        for (int q = 0; q < ntimes; q++)
            for (int k = 0; k <= nh[q]; k++)
                tab[(size_t)q * kmax + k] = (int)(std::lower_bound(uniq.begin(), uniq.end(), taus[c++]) - uniq.begin());
    }
    const size_t per_point = (size_t)nu * m.nt * 6 * sizeof(double);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)npts, ((size_t)1 << 30) / per_point));
    // the tables in one upload: instants, index table, nHat
    HostPack pk;
    const size_t o_taus = pk.add(uniq.data(), nu * sizeof(double));
    const size_t o_tab = pk.add(tab.data(), tab.size() * sizeof(int));
    const size_t o_nh = pk.add(nh.data(), ntimes * sizeof(int));
    unsigned char* d_pack = nullptr;
    int* d_first = nullptr;
    double* Mbuf = nullptr;
    long long* d_cnt = nullptr;
    const long long rows_max = (long long)m.nt * chunk;
    if (pk.upload(&d_pack, s) != cudaSuccess ||
        ws_malloc(&d_cnt, (rows_max + 1) * sizeof(long long), s) != cudaSuccess ||
        ws_malloc(&d_first, rows_max * sizeof(int), s) != cudaSuccess || ws_malloc(&Mbuf, per_point * chunk, s) != cudaSuccess) {
        cudaGetLastError();
        ws_free(d_pack, s);
        ws_free(d_cnt, s);
        ws_free(d_first, s);
        return fail(EBEM_ERR_NOMEM, "post-processing workspace allocation failed");
    }
    const double* d_taus = reinterpret_cast<const double*>(d_pack + o_taus);
    const int* d_tab = reinterpret_cast<const int*>(d_pack + o_tab);
    const int* d_nh = reinterpret_cast<const int*>(d_pack + o_nh);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device);
    cudaError_t e = cudaSuccess;
    int rc = EBEM_OK;
    for (int p0 = 0; p0 < npts && e == cudaSuccess && rc == EBEM_OK; p0 += chunk) {
        const int np = std::min(chunk, npts - p0);
        const long long rows = (long long)m.nt * np;
        pp_inst_count_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(m.d_geo, m.nt, d_pts, p0, np, nu, d_taus,
                                                                           P.velP, d_cnt, d_first);
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        rc = exclusive_scan(d_cnt, rows + 1, s);
        if (rc) break;
        long long total = 0;
        e = cudaMemcpyAsync(&total, d_cnt + rows, sizeof(long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
        if (total > 0)
            pp_inst_level_kernel<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(
                m.d_geo, m.nt, d_pts, p0, np, nu, d_taus, P.velP, P.velS, 4 * kPi * P.rho, d_cnt, d_first, total, Mbuf);
        const int sum_threads = ((long long)ntimes * np < 2LL * sms) ? 1024 : 128;
        pp_inst_sum_kernel<<<(unsigned)((long long)ntimes * np), sum_threads, 0, s>>>(
            Mbuf, m.d_geo, m.nt, d_pts, p0, np, nu, d_taus, P.velP, d_tab, kmax, d_nh, npts, d_phi, d_u);
        e = cudaGetLastError();
    }
    ws_free(Mbuf, s);
    ws_free(d_pack, s);
    ws_free(d_cnt, s);
    ws_free(d_first, s);
    if (rc) return rc;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("post-processing kernels: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

int launch_pp_sa(const MeshData& m, const PhysParams& P, const double* d_phi, const double* d_pts, int npts,
                 const double* h_times, int ntimes, double* d_u, cudaStream_t s) {
    {
        const int rc = launch_pp_sa_shared(m, P, d_phi, d_pts, npts, h_times, ntimes, d_u, s);
        if (rc != 1) return rc;                         // done (or failed); 1: instants barely repeat
    }
    long long total = (long long)m.nt * npts * ntimes;
    int threads = 128;
    if ((total + threads - 1) / threads > 0x7fffffffLL)
        return fail(EBEM_ERR_INVALID, "too many (triangle, point, time) triples for one launch");
    double* d_times = nullptr;
    EBEM_CUDA_TRY(ws_malloc(&d_times, sizeof(double) * ntimes, s));
    cudaError_t e = cudaMemcpyAsync(d_times, h_times, sizeof(double) * ntimes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_u, 0, sizeof(double) * 3 * (size_t)npts * ntimes, s);
    if (e != cudaSuccess) {
        ws_free(d_times, s);
        return fail(EBEM_ERR_CUDA, std::string("post-processing set-up: ") + cudaGetErrorString(e));
    }
    pp_sa_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(
        m.d_geo, m.nt, d_pts, npts, d_times, ntimes, d_phi, P.nT, P.velP, P.velS, P.dt, 4 * kPi * P.rho, d_u);
    e = cudaGetLastError();
    ws_free(d_times, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("post-processing kernel: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

}  // namespace ebem
