// Numerical-inner assembly of E_l: outer Gauss-Hammer rule on the source
// triangle, composite Gauss-Hammer rule on the field triangle, the Lamé kernel
// integrated twice in time with separate P and S Heaviside fronts.
//
// Reference: functions/BEMenerg_indir/BEMenerg_core/BEMenerg_coreGPU/CUDAkernels/
// kernelGHC.cu:5-259 (identical copies: BEMenerg_coreFN/CUDAkernels/kernelGHC.cu,
// functions/BEMenerg_dir/CUDAkernels/kernelV.cu), launched by
// BEMenerg_coreGPU_launchKernel.m:11 with grid (N, N, lags) and one thread
// per inner node.  Semantics kept: off-diagonal pairs only (the diagonal
// comes from the semi-analytic path, BEMenerg_coreGPU_timeMarching.m:101-131),
// the null test (lag-1) c_S dt > max vertex distance (kernelGHC.cu:171-201),
// instants dt (lag + {-1, 0, 1}) with weights (1, -2, 1) and t >= 0
// (:88-99), entries written only when |value| > 1e-14 before the division by
// 4 pi rho (:164-165), accumulated into the output (+=).
//
// B200 design: one thread per (source, field) pair (consecutive lanes take
// consecutive sources of one field triangle).  The lag combination E_l =
// K_{l+1} - 2 K_l + K_{l-1} is taken per node pair on the kernel's scalar time
// functions (ghc_window2), so a node pair costs work only in the lags whose
// window a front crosses or lies between the fronts, where the difference
// has a closed form; windows before the P front or after the S front are
// skipped on r^2 (the reference evaluates every node pair at every instant
// of every lag and reduces through shared memory).
#include "ebem_internal.h"
#include "sa_pair.cuh"

// Dispatch between the warp-per-pair and thread-per-pair kernels (compile-time
// knobs for measuring other thresholds).  Measured with the exact lag skip in
// both kernels: the warp kernel wins up to about 16k pairs per SM at 84 node
// pairs and more (sphere of 320 triangles, rule 7/4/3: 5.5 -> 3.3 ms; sphere
// of 1280, 1.6 M pairs, rule 7/16/3: 166 -> 97 ms); on the 2800-triangle bar
// (7.8 M pairs, most of them done after the skip test) the thread kernel is
// 1.4x faster at rule 7/4/3 and even at 7/16/3.
#ifndef EBEM_GHC_WARP_MIN_NODE_PAIRS
#define EBEM_GHC_WARP_MIN_NODE_PAIRS 64
#endif
#ifndef EBEM_GHC_WARP_MAX_PAIRS_PER_SM
#define EBEM_GHC_WARP_MAX_PAIRS_PER_SM 16384
#endif

namespace ebem {

struct GHCArgs {
    const double* coords;
    const int32_t* tris;
    const TriGeom* geo;
    const double* outer;    // n_out x 3 barycentric
    const double* wout;     // n_out
    const double* inner;    // n_in x 3 barycentric (n_sub sub-triangles x n_sing nodes)
    const double* win;      // n_sing
    int n_out, n_sub, n_sing;
    int N;
    double velP, velS, dt, c4pirho;
    int lag0, nlag;
    double* E;
    size_t ld, ld_lag;
};

// Second difference over the window of lag l (levels l-1, l, l+1 of t_k =
// k dt, kernelGHC.cu:88-99) of the time functions of one front X of the
// kernel kernelGHC.cu:204-259 (nucleo): H = [t - r/c > 0] and
// Q = (c^2 t^2 - r^2) / c^2 H.  Before the front both vanish; with the whole
// window after it H is constant and Q = t^2 - r^2/c^2, so the differences
// are exactly (0, 2 dt^2).
struct Win2 {
    double H, Q;
};

__host__ __device__ __forceinline__ Win2 ghc_window2(double r, double c, int l, double dt) {
    Win2 d = {0.0, 0.0};
    if ((l + 1) * dt - r / c <= 0) return d;
    if (l >= 1 && (l - 1) * dt - r / c > 0) {
        d.Q = 2 * dt * dt;
        return d;
    }
    const double w[3] = {1.0, -2.0, 1.0};
    for (int j = 0; j < 3; j++) {
        const int k = l - 1 + j;
        if (k < 0) continue;
        const double t = k * dt;
        if (t - r / c > 0) {
            d.H += w[j];
            d.Q += w[j] * ((c * c * t * t - r * r) / (c * c));
        }
    }
    return d;
}

// One node pair's share of the lag-l second difference of nucleo, symmetric
// entries (11,12,13,22,23,33): with dQ = dQ_P - dQ_S,
//   out_ij = g1 x_i x_j + g2 delta_ij,
//   g1 = ir^3 (dH_P/c_P^2 - dH_S/c_S^2) + 3/2 ir^5 dQ,  g2 = ir dH_S/c_S^2 - 1/2 ir^3 dQ.
__host__ __device__ __forceinline__ void ghc_pair(double nu[6], const double x[3], double ir, double dHP, double dHS,
                                                  double dQ, double icP2, double icS2) {
    const double ir2 = ir * ir, ir3 = ir2 * ir, ir5 = ir3 * ir2;
    const double g1 = ir3 * (dHP * icP2 - dHS * icS2) + 1.5 * ir5 * dQ;
    const double g2 = ir * dHS * icS2 - 0.5 * ir3 * dQ;
    nu[0] = g1 * x[0] * x[0] + g2;
    nu[1] = g1 * x[0] * x[1];
    nu[2] = g1 * x[0] * x[2];
    nu[3] = g1 * x[1] * x[1] + g2;
    nu[4] = g1 * x[1] * x[2];
    nu[5] = g1 * x[2] * x[2] + g2;
}

__global__ void __launch_bounds__(128, 6) ghc_assemble_kernel(GHCArgs A) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)A.N * A.N) return;
    const int i = (int)(p % A.N);          // source (outer rule)
    const int j = (int)(p / A.N);          // field (inner rule)
    if (i == j) return;
    double VS[3][3], VF[3][3];
    for (int v = 0; v < 3; v++)
        for (int c = 0; c < 3; c++) {
            VS[v][c] = A.coords[3 * A.tris[3 * i + v] + c];
            VF[v][c] = A.coords[3 * A.tris[3 * j + v] + c];
        }
    double distMax = 0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double d0 = VS[a][0] - VF[b][0], d1 = VS[a][1] - VF[b][1], d2 = VS[a][2] - VF[b][2];
            distMax = fmax(distMax, sqrt(d0 * d0 + d1 * d1 + d2 * d2));
        }
    // lags computed: not null, i.e. (l-1) c_S dt <= distMax
    int lhi = A.lag0 + A.nlag - 1;
    while (lhi >= A.lag0 && (lhi - 1) * A.velS * A.dt > distMax) lhi--;
    if (lhi < A.lag0) return;
    const double aS = A.geo[i].area, aF = A.geo[j].area;
    const double cP = A.velP, cS = A.velS, dt = A.dt;
    const double icP2 = 1 / (cP * cP), icS2 = 1 / (cS * cS);
    const size_t n3 = A.ld;
    const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    // the node pairs' exact distance range (one pass): a lag whose window lies
    // before the P front or after the S front for all of them adds nothing
    // (the null test above bounds the lags by vertex distances only)
    double r2min = 1e300, r2max = 0.0;
    for (int q = 0; q < A.n_sub * A.n_sing; q++) {
        const double* bq = A.inner + 3 * q;
        double y[3];
        for (int c = 0; c < 3; c++) y[c] = bq[0] * VF[0][c] + bq[1] * VF[1][c] + bq[2] * VF[2][c];
        for (int o = 0; o < A.n_out; o++) {
            const double* bl = A.outer + 3 * o;
            double x[3];
            for (int c = 0; c < 3; c++) x[c] = y[c] - (bl[0] * VS[0][c] + bl[1] * VS[1][c] + bl[2] * VS[2][c]);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            r2min = fmin(r2min, r2);
            r2max = fmax(r2max, r2);
        }
    }
    for (int l = A.lag0; l <= lhi; l++) {
        const double thi = (l + 1) * dt, tlo = (l - 1) * dt;
        const double skipP2 = (cP * thi) * (cP * thi) * (1 + 1e-12);
        const double skipS2 = (l >= 1) ? (cS * tlo) * (cS * tlo) * (1 - 1e-12) : -1.0;
        if (r2min > skipP2 || r2max < skipS2) continue;
        double K[6] = {0, 0, 0, 0, 0, 0};
        for (int q = 0; q < A.n_sub * A.n_sing; q++) {
            const double* bq = A.inner + 3 * q;
            double y[3];
            for (int c = 0; c < 3; c++) y[c] = bq[0] * VF[0][c] + bq[1] * VF[1][c] + bq[2] * VF[2][c];
            const double wq = A.win[q % A.n_sing] * aF;
            for (int o = 0; o < A.n_out; o++) {
                const double* bl = A.outer + 3 * o;
                double x[3];
                for (int c = 0; c < 3; c++) x[c] = y[c] - (bl[0] * VS[0][c] + bl[1] * VS[1][c] + bl[2] * VS[2][c]);
                const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                if (r2 > skipP2 || r2 < skipS2) continue;
                const double r = sqrt(r2);
                const Win2 P = ghc_window2(r, cP, l, dt), S = ghc_window2(r, cS, l, dt);
                const double w = (A.wout[o] * aS) * wq;
                double nu[6];
                ghc_pair(nu, x, 1 / r, P.H, S.H, P.Q - S.Q, icP2, icS2);
#pragma unroll
                for (int e = 0; e < 6; e++) K[e] += w * nu[e];
            }
        }
        double* base = A.E + (size_t)(l - A.lag0) * A.ld_lag + (3 * (size_t)j) * n3 + 3 * (size_t)i;
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const double v = K[map[3 * c + r]];
                if (fabs(v) > 1.0e-14) base[c * n3 + r] += v / A.c4pirho;
            }
    }
}

// Warp-per-pair variant for small meshes and rules with at least 160 node
// pairs (see the dispatch in launch_ghc_assemble): the lanes
// take the node pairs (inner node q, outer node o) of the pair, the same
// per-node-pair arithmetic as ghc_assemble_kernel, and a warp reduction per
// lag gives the 6 entries (the thread kernel leaves half of each warp's
// lanes idle on the skip test).  Both kernels are capped at 80 registers (6
// blocks of 128 threads per SM); with the compiler's 157 and 170 registers
// 3 blocks fitted and the FP64 dependency chains were not hidden: sphere of
// 320 triangles, rule 7/16/3 13.7 -> 6.6 ms (warp kernel); bar of 2800
// triangles, rule 7/4/3 188 -> 137 ms (thread kernel); 128 registers gave
// 7.3 and 152 ms.
__global__ void __launch_bounds__(128, 6) ghc_assemble_warp_kernel(GHCArgs A) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int n_in = A.n_sub * A.n_sing, NP = n_in * A.n_out;
    const double cP = A.velP, cS = A.velS, dt = A.dt;
    const double icP2 = 1 / (cP * cP), icS2 = 1 / (cS * cS);
    const size_t n3 = A.ld;
    for (long long p = warp; p < (long long)A.N * A.N; p += nwarps) {
        const int i = (int)(p % A.N);      // source (outer rule)
        const int j = (int)(p / A.N);      // field (inner rule)
        if (i == j) continue;
        double VS[3][3], VF[3][3];
        for (int v = 0; v < 3; v++)
            for (int c = 0; c < 3; c++) {
                VS[v][c] = A.coords[3 * A.tris[3 * i + v] + c];
                VF[v][c] = A.coords[3 * A.tris[3 * j + v] + c];
            }
        double distMax = 0;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                double d0 = VS[a][0] - VF[b][0], d1 = VS[a][1] - VF[b][1], d2 = VS[a][2] - VF[b][2];
                distMax = fmax(distMax, sqrt(d0 * d0 + d1 * d1 + d2 * d2));
            }
        int lhi = A.lag0 + A.nlag - 1;
        while (lhi >= A.lag0 && (lhi - 1) * A.velS * A.dt > distMax) lhi--;
        if (lhi < A.lag0) continue;
        const double aS = A.geo[i].area, aF = A.geo[j].area;
        // the node pairs' exact distance range (warp min/max): lags whose
        // window lies before the P front or after the S front for every node
        // pair add nothing and are skipped by the whole warp
        double r2min = 1e300, r2max = 0.0;
        for (int np = lane; np < NP; np += 32) {
            const int q = np / A.n_out, o = np - q * A.n_out;
            const double* bq = A.inner + 3 * q;
            const double* bl = A.outer + 3 * o;
            double r2 = 0.0;
            for (int c = 0; c < 3; c++) {
                const double xc = (bq[0] * VF[0][c] + bq[1] * VF[1][c] + bq[2] * VF[2][c]) -
                                  (bl[0] * VS[0][c] + bl[1] * VS[1][c] + bl[2] * VS[2][c]);
                r2 += xc * xc;
            }
            r2min = fmin(r2min, r2);
            r2max = fmax(r2max, r2);
        }
        for (int off = 16; off > 0; off >>= 1) {
            r2min = fmin(r2min, __shfl_xor_sync(0xffffffffu, r2min, off));
            r2max = fmax(r2max, __shfl_xor_sync(0xffffffffu, r2max, off));
        }
        for (int l = A.lag0; l <= lhi; l++) {
            const double thi = (l + 1) * dt, tlo = (l - 1) * dt;
            const double skipP2 = (cP * thi) * (cP * thi) * (1 + 1e-12);
            const double skipS2 = (l >= 1) ? (cS * tlo) * (cS * tlo) * (1 - 1e-12) : -1.0;
            if (r2min > skipP2 || r2max < skipS2) continue;
            double K[6] = {0, 0, 0, 0, 0, 0};
            for (int np = lane; np < NP; np += 32) {
                const int q = np / A.n_out, o = np - q * A.n_out;
                const double* bq = A.inner + 3 * q;
                const double* bl = A.outer + 3 * o;
                double x[3];
                for (int c = 0; c < 3; c++)
                    x[c] = (bq[0] * VF[0][c] + bq[1] * VF[1][c] + bq[2] * VF[2][c]) -
                           (bl[0] * VS[0][c] + bl[1] * VS[1][c] + bl[2] * VS[2][c]);
                const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                if (r2 > skipP2 || r2 < skipS2) continue;
                const double r = sqrt(r2);
                const Win2 P = ghc_window2(r, cP, l, dt), S = ghc_window2(r, cS, l, dt);
                const double w = (A.wout[o] * aS) * (A.win[q % A.n_sing] * aF);
                double nu[6];
                ghc_pair(nu, x, 1 / r, P.H, S.H, P.Q - S.Q, icP2, icS2);
#pragma unroll
                for (int e = 0; e < 6; e++) K[e] += w * nu[e];
            }
#pragma unroll
            for (int e = 0; e < 6; e++)
                for (int off = 16; off > 0; off >>= 1) K[e] += __shfl_xor_sync(0xffffffffu, K[e], off);
            if (lane < 9) {
                const int c = lane / 3, r = lane - 3 * c;
                const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
                double v = 0;
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if (e == map[lane]) v = K[e];
                double* base = A.E + (size_t)(l - A.lag0) * A.ld_lag + (3 * (size_t)j) * n3 + 3 * (size_t)i;
                if (fabs(v) > 1.0e-14) base[c * n3 + r] += v / A.c4pirho;
            }
        }
    }
}

int launch_ghc_assemble(const MeshData& m, const PhysParams& P, int n_gh, int n_sub, int n_sing, int lag0, int nlag,
                        double* d_E, size_t ld, size_t ld_lag, cudaStream_t s) {
    double ob[28 * 3], ow[28];
    if (gh_composite(n_gh, 1, ob, ow)) return fail(EBEM_ERR_INVALID, "unsupported outer rule");
    std::vector<double> ib((size_t)3 * n_sub * n_sing), iw(n_sing);
    if (gh_composite(n_sing, n_sub, ib.data(), iw.data())) return fail(EBEM_ERR_INVALID, "unsupported inner rule");
    size_t nb = 3 * n_gh + n_gh + ib.size() + iw.size();
    std::vector<double> tab(nb);
    size_t o = 0;
    for (int k = 0; k < 3 * n_gh; k++) tab[o++] = ob[k];
    for (int k = 0; k < n_gh; k++) tab[o++] = ow[k];
    for (double v : ib) tab[o++] = v;
    for (double v : iw) tab[o++] = v;
    double* d_tab = nullptr;
    EBEM_CUDA_TRY(ws_malloc(&d_tab, nb * sizeof(double), s));
    if (cudaError_t e = cudaMemcpyAsync(d_tab, tab.data(), nb * sizeof(double), cudaMemcpyHostToDevice, s)) {
        ws_free(d_tab, s);
        return fail(EBEM_ERR_CUDA, std::string("rule table upload: ") + cudaGetErrorString(e));
    }
    GHCArgs A;
    A.coords = m.d_coords;
    A.tris = m.d_tris;
    A.geo = m.d_geo;
    A.outer = d_tab;
    A.wout = d_tab + 3 * n_gh;
    A.inner = d_tab + 4 * n_gh;
    A.win = d_tab + 4 * n_gh + ib.size();
    A.n_out = n_gh;
    A.n_sub = n_sub;
    A.n_sing = n_sing;
    A.N = m.nt;
    A.velP = P.velP;
    A.velS = P.velS;
    A.dt = P.dt;
    A.c4pirho = 4 * kPi * P.rho;
    A.lag0 = lag0;
    A.nlag = nlag;
    A.E = d_E;
    A.ld = ld;
    A.ld_lag = ld_lag;
    long long NN = (long long)m.nt * m.nt;
    int threads = 128;
    // warp per pair below the thresholds at the top of this file
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device);
    if ((long long)n_gh * n_sub * n_sing >= EBEM_GHC_WARP_MIN_NODE_PAIRS &&
        NN < (long long)sms * EBEM_GHC_WARP_MAX_PAIRS_PER_SM) {
        const long long want = (NN + 3) / 4, cap = (long long)sms * 64;
        ghc_assemble_warp_kernel<<<(unsigned)(want < cap ? want : cap), threads, 0, s>>>(A);
    } else {
        ghc_assemble_kernel<<<(unsigned)((NN + threads - 1) / threads), threads, 0, s>>>(A);
    }
    cudaError_t e = cudaGetLastError();
    ws_free(d_tab, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("numerical-inner assembly: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

}  // namespace ebem
