// Direct (displacement / traction) formulation on the device: the
// double-layer operator K_l with its P1 basis, its same-triangle parts and the
// diagonal blocks of V_l on the Duffy-type DIAG rule, the direct
// post-processing operators, and the direct time marching.
//
// Reference (paths relative to the reference project root; "DIR/" =
// functions/BEMenerg_dir/, "PP/" = functions/BEMenerg_dirPP/):
//   P1 basis         DIR/BEMenerg_dir_calcCostantData.m:17-21
//   K_l              DIR/CUDAkernels/kernelK.cu:14-460, launched by
//                    DIR/BEMenerg_dir_timeMarchingN.m:172-266
//   singular K_l     DIR/BEMenerg_dir_calcSubBlockSingK.m:1-41, DIR/BEMenerg_dir_calcKIntgSing.m
//   diagonal V_l     DIR/BEMenerg_dir_calcSubBlockDiagV.m:1-118
//   DIAG rule        functions/utility/quadRules/doppioGauss1D.m:1-43
//   post-processing  PP/CUDAkernels/kernelG.cu, PP/CUDAkernels/kernelP.cu,
//                    PP/BEMenerg_ppN_calc.m:115-124, PP/BEMenerg_ppD_calc.m:91-99
//   time marching    DIR/BEMenerg_dir_timeMarchingN.m:268-299 (least squares),
//                    DIR/BEMenerg_dir_timeMarchingD.m:272-296, DIR/BEMenerg_dir_calcBetaVgpu.m,
//                    DIR/BEMenerg_dir_calcBetaKgpu.m
//
// B200 design (not the reference's): one thread per (row triangle, vertex)
// pair walks the time levels once (level reuse, a 4-level window for the
// third difference of K, 3 levels for V and P) and visits only the
// triangles that contain the vertex (an adjacency list; the reference scans
// all N triangles per block).  Post-processing is contracted with the data
// in the kernel (each instant evaluated once, no nHat x N matrices), with
// the reference's matrices available for verification.  The DN system is
// factorised once (QR), the reference re-solves densely every step.
#include "ebem_internal.h"

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <vector>

// Dispatch between the warp-per-pair and thread-per-pair K kernels
// (compile-time knobs for measuring other thresholds).
#ifndef EBEM_K_WARP_MIN_NODE_PAIRS
#define EBEM_K_WARP_MIN_NODE_PAIRS 32
#endif
#ifndef EBEM_K_WARP_MAX_PAIRS_PER_SM
#define EBEM_K_WARP_MAX_PAIRS_PER_SM 4096
#endif

namespace ebem {

// ---------------------------------------------------------------------------
// DIAG rule (doppioGauss1D): n = n1^2 nodes on the triangle (A, B, C) with the
// singular vertex C: node (i, j) = ((1-x_j)(1-x_i), x_j (1-x_i), x_i) with
// weight 2 w_i w_j (1 - x_i), x, w the n1-point Gauss-Legendre rule on (0,1)
// (Newton's iteration on the Legendre polynomial).
int diag_rule(int n, std::vector<double>& nodes, std::vector<double>& w) {
    int n1 = (int)std::lround(std::sqrt((double)n));
    if (n1 < 1 || n1 * n1 != n) return EBEM_ERR_INVALID;
    std::vector<double> x(n1), wt(n1);
    for (int i = 0; i < n1; i++) {
        double z = std::cos(kPi * (i + 0.75) / (n1 + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n1; k++) {
                double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n1 * (z * p1 - p0) / (z * z - 1);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n1; k++) {
            double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n1 * (z * p1 - p0) / (z * z - 1);
        x[n1 - 1 - i] = z;
        wt[n1 - 1 - i] = 2 / ((1 - z * z) * dp * dp);
    }
    if (n1 == 1) { x[0] = 0.0; wt[0] = 2.0; }
    nodes.resize(3 * (size_t)n);
    w.resize(n);
    for (int j = 0; j < n1; j++)
        for (int i = 0; i < n1; i++) {
            const double xi = 0.5 + x[i] / 2, xj = 0.5 + x[j] / 2, wi = wt[i] / 2, wj = wt[j] / 2;
            const int k = i + n1 * j;
            nodes[3 * k] = (1 - xj) * (1 - xi);
            nodes[3 * k + 1] = xj * (1 - xi);
            nodes[3 * k + 2] = xi;
            w[k] = 2 * wj * (wi * (1 - xi));
        }
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// mesh data

__global__ void dir_prep_kernel(const double* __restrict__ coords, const int32_t* __restrict__ tris, int nt,
                                DirTri* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    DirTri d;
    for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++) d.V[a][c] = coords[3 * tris[3 * t + a] + c];
    double g1[3], g2[3], g3[3];
    for (int c = 0; c < 3; c++) {
        g1[c] = d.V[0][c] - d.V[2][c];
        g2[c] = d.V[1][c] - d.V[2][c];
        g3[c] = d.V[0][c] - d.V[1][c];
    }
    double nn[3] = {g1[1] * g2[2] - g2[1] * g1[2], -g1[0] * g2[2] + g2[0] * g1[2], g1[0] * g2[1] - g2[0] * g1[1]};
    d.area = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]) / 2;
    for (int c = 0; c < 3; c++) d.n[c] = nn[c] / (2 * d.area);
    d.maxL = fmax(fmax(sqrt(g3[0] * g3[0] + g3[1] * g3[1] + g3[2] * g3[2]), sqrt(g2[0] * g2[0] + g2[1] * g2[1] + g2[2] * g2[2])),
                  sqrt(g1[0] * g1[0] + g1[1] * g1[1] + g1[2] * g1[2]));
    // P1 basis: M = A B^-1, B = [l21, l31, l21 x l31]; rows of B^-1 are
    // (l31 x n, n x l21, l21 x l31) / det
    double l21[3], l31[3];
    for (int c = 0; c < 3; c++) { l21[c] = d.V[1][c] - d.V[0][c]; l31[c] = d.V[2][c] - d.V[0][c]; }
    double cn[3] = {l21[1] * l31[2] - l21[2] * l31[1], l21[2] * l31[0] - l21[0] * l31[2], l21[0] * l31[1] - l21[1] * l31[0]};
    double r0[3] = {l31[1] * cn[2] - l31[2] * cn[1], l31[2] * cn[0] - l31[0] * cn[2], l31[0] * cn[1] - l31[1] * cn[0]};
    double r1[3] = {cn[1] * l21[2] - cn[2] * l21[1], cn[2] * l21[0] - cn[0] * l21[2], cn[0] * l21[1] - cn[1] * l21[0]};
    double det = l21[0] * r0[0] + l21[1] * r0[1] + l21[2] * r0[2];
    for (int c = 0; c < 3; c++) {
        r0[c] /= det;
        r1[c] /= det;
        d.M[c] = -r0[c] - r1[c];
        d.M[3 + c] = r0[c];
        d.M[6 + c] = r1[c];
    }
    for (int k = 0; k < 3; k++)
        d.v[k] = (k == 0 ? 1.0 : 0.0) - (d.M[3 * k] * d.V[0][0] + d.M[3 * k + 1] * d.V[0][1] + d.M[3 * k + 2] * d.V[0][2]);
    out[t] = d;
}

int prep_direct(MeshData& m, cudaStream_t s) {
    if (m.d_dir) return EBEM_OK;
    std::vector<int32_t> tris(3 * (size_t)m.nt);
    EBEM_CUDA_TRY(cudaMemcpy(tris.data(), m.d_tris, sizeof(int32_t) * tris.size(), cudaMemcpyDeviceToHost));
    std::vector<int32_t> off(m.nv + 1, 0), lst(3 * (size_t)m.nt);
    for (int32_t v : tris) off[v + 1]++;
    for (int v = 0; v < m.nv; v++) off[v + 1] += off[v];
    std::vector<int32_t> pos(off.begin(), off.end() - 1);
    for (int t = 0; t < m.nt; t++)
        for (int k = 0; k < 3; k++) lst[pos[tris[3 * t + k]]++] = t;      // ascending triangle order per vertex
    if (cudaMalloc(&m.d_dir, sizeof(DirTri) * (size_t)m.nt) != cudaSuccess ||
        cudaMalloc(&m.d_vt_off, sizeof(int32_t) * off.size()) != cudaSuccess ||
        cudaMalloc(&m.d_vt_tri, sizeof(int32_t) * lst.size()) != cudaSuccess) {
        cudaGetLastError();
        free_direct(m);
        return fail(EBEM_ERR_NOMEM, "direct-formulation mesh data allocation failed");
    }
    // d_dir marks the data as built: on a failure below it is released, so
    // the next call starts over instead of using a half-built table
    std::vector<DirTri> h(m.nt);
    cudaError_t e = cudaMemcpyAsync(m.d_vt_off, off.data(), sizeof(int32_t) * off.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m.d_vt_tri, lst.data(), sizeof(int32_t) * lst.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        dir_prep_kernel<<<(m.nt + 127) / 128, 128, 0, s>>>(m.d_coords, m.d_tris, m.nt, m.d_dir);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), m.d_dir, sizeof(DirTri) * h.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_direct(m);
        return fail(EBEM_ERR_CUDA, std::string("direct-formulation mesh data: ") + cudaGetErrorString(e));
    }
    m.max_len = 0.0;
    for (const DirTri& d : h) m.max_len = std::max(m.max_len, d.maxL);
    return EBEM_OK;
}

void free_direct(MeshData& m) {
    if (m.d_dir) cudaFree(m.d_dir);
    if (m.d_vt_off) cudaFree(m.d_vt_off);
    if (m.d_vt_tri) cudaFree(m.d_vt_tri);
    m.d_dir = nullptr;
    m.d_vt_off = m.d_vt_tri = nullptr;
}

// ---------------------------------------------------------------------------
// kernels of the direct formulation

struct Mat {
    double lam, mu, rho, cP, cS;
};

struct TimeF {
    double HP, HS, RP, RS, SP, SS;   // fronts, (t - r/c) H, (t - r/c)^2 (t + 2r/c) / 6 H
};

__device__ __forceinline__ TimeF time_f(double r, double t, const Mat& p) {
    TimeF f;
    const double aP = t - r / p.cP, aS = t - r / p.cS;
    f.HP = aP > 0 ? 1.0 : 0.0;
    f.HS = aS > 0 ? 1.0 : 0.0;
    f.RP = aP * f.HP;
    f.RS = aS * f.HS;
    f.SP = aP * aP * (t + 2 * r / p.cP) / 6 * f.HP;
    f.SS = aS * aS * (t + 2 * r / p.cS) / 6 * f.HS;
    return f;
}

__device__ __forceinline__ int levi(int a, int b, int c) {
    return (a == b || b == c || a == c) ? 0 : (((a + 1) % 3 == b) ? 1 : -1);
}

// Double-layer kernel (kernelK.cu: nucleoKL + nucleoKT - sum_j vms_j nucleoKRj)
// for basis value phik and vms = n x grad phi, x = outer - inner node.
// with_xn: the (x . n) terms (dropped on the same triangle); bad_front: the
// H(r - r/c_P) of kernelK.cu:414-449.
__device__ void kern_k(double out[9], const double x[3], double r, const double n[3], double t, const double vms[3],
                       double phik, const Mat& p, bool with_xn, bool bad_front) {
    const TimeF f = time_f(r, t, p);
    const double a1 = p.lam / (p.lam + p.mu), a2 = p.mu / (p.lam + p.mu);
    const double c1 = p.lam * p.mu / (p.rho * (p.lam + p.mu)), c2 = 2 * p.mu / p.rho;
    const double ir = 1.0 / r, ir2 = ir * ir, ir3 = ir2 * ir, ir5 = ir3 * ir2;
    const double xn = x[0] * n[0] + x[1] * n[1] + x[2] * n[2];
    const double D = f.RP - f.RS, DT = f.HP / p.cP - f.HS / p.cS;
    const double RPl = bad_front ? (t - r / p.cP) * ((r - r / p.cP) > 0 ? 1.0 : 0.0) : f.RP;
    const double Dl = f.RS / (p.cS * p.cS) - RPl / (p.cP * p.cP);
    const double Dd = f.RS / (p.cS * p.cS) - f.RP / (p.cP * p.cP);
    const double Hh = f.SS - f.SP;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double mix = a1 * x[i] * n[k] + a2 * x[k] * n[i];
            double kl = mix * ir3 * D, kt = mix * ir2 * DT;
            if (with_xn && i == k) {
                kl += xn * ir3 * f.RS;
                kt += xn * ir2 * f.HS / p.cS;
            }
            double kr = 0.0;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                double h = 0.0, d = 0.0;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const int e = levi(j, i, q);
                    if (e == 0) continue;
                    h += e * (3 * x[q] * x[k] * ir5 - ((q == k) ? ir3 : 0.0));
                    d += e * (x[q] * x[k] * ir3);
                }
                kr += vms[j] * (c1 * levi(j, k, i) * ir * Dl + c2 * h * Hh + c2 * d * Dd);
            }
            out[3 * i + k] = -kr + phik * (kl + kt);
        }
}

// Lame kernel twice integrated in time (kernelGHC.cu nucleo).
__device__ __forceinline__ void kern_v(double nu[9], const double x[3], double r, double t, double cP, double cS) {
    const double HP = (t - r / cP) > 0 ? 1.0 : 0.0, HS = (t - r / cS) > 0 ? 1.0 : 0.0;
    const double r3 = r * r * r, r5 = r3 * r * r;
    const double tail = (cP * cP * t * t - r * r) / (cP * cP) * HP - (cS * cS * t * t - r * r) / (cS * cS) * HS;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double xx = x[i] * x[j], d = (i == j) ? 1.0 : 0.0;
            nu[3 * i + j] = (xx / r3) * (1 / (cP * cP)) * HP + (d / r - xx / r3) * (1 / (cS * cS)) * HS -
                            0.5 * (d / r3 - 3 * (xx / r5)) * tail;
        }
}

// Traction kernel of kernelP.cu times phik, x = source - node.
__device__ void kern_p(double nu[9], const double x[3], const double n[3], double r, double t, double phik,
                       const Mat& p) {
    const TimeF f = time_f(r, t, p);
    const double xn = x[0] * n[0] + x[1] * n[1] + x[2] * n[2];
    const double ir = 1.0 / r, ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2, ir5 = ir4 * ir, ir7 = ir5 * ir2;
    const double lam = p.lam, mu = p.mu;
    const double fP3 = f.HP / (p.cP * p.cP * p.cP), fS3 = f.HS / (p.cS * p.cS * p.cS);
    const double fP2 = f.RP / (p.cP * p.cP), fS2 = f.RS / (p.cS * p.cS), fH = f.SP - f.SS;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double d = (i == j) ? 1.0 : 0.0;
            const double a = x[i] * n[j], b = x[j] * n[i], xx = x[j] * x[i];
            const double v = (lam * a * ir2 + 2 * mu * xx * ir4 * xn) * fP3 +
                             mu * (b * ir2 + (d * ir2 - 2 * xx * ir4) * xn) * fS3 +
                             ((lam - 2 * mu) * a * ir3 - 2 * mu * b * ir3 - 2 * mu * (d * ir3 - 6 * xx * ir5) * xn) * fP2 +
                             mu * (2 * a * ir3 + 3 * b * ir3 + 3 * (d * ir3 - 4 * xx * ir5) * xn) * fS2 -
                             6 * mu * (a * ir5 + b * ir5 + (d * ir5 - 5 * xx * ir7) * xn) * fH;
            nu[3 * i + j] = v * phik;
        }
}

__device__ __forceinline__ void bary_point(double y[3], const double* b, const double V[3][3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) y[c] = b[0] * V[0][c] + b[1] * V[1][c] + b[2] * V[2][c];
}

__device__ __forceinline__ int local_index(const int32_t* tris, int t, int s) {
    return (tris[3 * t] == s) ? 1 : (tris[3 * t + 1] == s) ? 2 : (tris[3 * t + 2] == s) ? 3 : 0;
}

// ---------------------------------------------------------------------------
// K_l, off-singular part: one thread per (row triangle x, vertex s)

struct KArgs {
    const DirTri* tri;
    const double* coords;
    const int32_t* tris;
    const int32_t* vt_off;
    const int32_t* vt_tri;
    const double* outer;     // n_gh x 3
    const double* wout;      // n_gh
    const double* inner;     // n_in x 3 (n_sub x n_sing)
    const double* win;       // n_sing
    int n_gh, n_in, n_sing;
    int N, Nv;
    Mat p;
    double dt, max_len;
    int lag0, nlag, nblocks, fix;
    double* K;
    size_t ld, ld_lag;
};

__device__ __forceinline__ void k_emit(const KArgs& A, int l, int x, int s, const double Tm3[9], const double Tm2[9],
                                       const double Tm1[9], const double T[9], bool clamp) {
    double* base = A.K + (size_t)(l - A.lag0) * A.ld_lag + (3 * (size_t)s) * A.ld + 3 * (size_t)x;
    const double c = 4 * kPi * A.dt;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int e = 3 * i + j;
            const double v = ((-Tm3[e] + 3 * Tm2[e]) + (-3 * Tm1[e])) + T[e];
            if (!clamp || fabs(v) > 1.0e-14) base[(size_t)j * A.ld + i] += v / c;
        }
}

// Third difference over the window of lag l, E_l = T_{l+1} - 3 T_l + 3 T_{l-1}
// - T_{l-2} on the levels t_k = k dt with levels k < 1 read as 0 (the lag
// combination of kernelK.cu), taken per node pair on the scalar time
// functions of one front X (arrival tX = r / c_X):
//   R = (t - tX) H,  H = [t - tX > 0],  S = (t - tX)^2 (t + 2 tX) / 6 H.
// Before the front all three vanish; with the whole window after it R is
// linear, H constant and S a cubic of leading coefficient 1/6, so the
// differences are exactly (0, 0, dt^3).  Only windows that a front crosses,
// or that reach below level 1, are summed level by level.
struct Win3 {
    double R, H, S;
};

__host__ __device__ __forceinline__ Win3 front_window3(double tX, int l, double dt) {
    Win3 d = {0.0, 0.0, 0.0};
    if ((l + 1) * dt - tX <= 0) return d;
    if (l >= 3 && (l - 2) * dt - tX > 0) {
        d.S = dt * dt * dt;
        return d;
    }
    const double c[4] = {-1.0, 3.0, -3.0, 1.0};
    for (int w = 0; w < 4; w++) {
        const int k = l - 2 + w;
        if (k < 1) continue;
        const double t = k * dt, a = t - tX;
        if (a > 0) {
            d.R += c[w] * a;
            d.H += c[w];
            d.S += c[w] * (a * a * (t + 2 * tX) / 6);
        }
    }
    return d;
}

// Third difference of the linear (t - tP) of the reference's H(r - r/c_P)
// term (kernelK.cu:414-449): zero unless the window reaches below level 1.
__host__ __device__ __forceinline__ double lin_window3(double tP, int l, double dt) {
    if (l >= 3) return 0.0;
    const double c[4] = {-1.0, 3.0, -3.0, 1.0};
    double d = 0.0;
    for (int w = 0; w < 4; w++) {
        const int k = l - 2 + w;
        if (k >= 1) d += c[w] * (k * dt - tP);
    }
    return d;
}

struct KCoef {
    double a1, a2, c1, c2, icP, icS, icP2, icS2;
};

__host__ __device__ inline KCoef k_coef(const Mat& p) {
    KCoef c;
    c.a1 = p.lam / (p.lam + p.mu);
    c.a2 = p.mu / (p.lam + p.mu);
    c.c1 = p.lam * p.mu / (p.rho * (p.lam + p.mu));
    c.c2 = 2 * p.mu / p.rho;
    c.icP = 1 / p.cP;
    c.icS = 1 / p.cS;
    c.icP2 = 1 / (p.cP * p.cP);
    c.icS2 = 1 / (p.cS * p.cS);
    return c;
}

// One node pair's share of the lag-l third difference of the double-layer
// kernel (nucleoKL + nucleoKT - sum_j vms_j nucleoKRj of kernelK.cu), x =
// outer - inner node, n the field triangle's normal, v = vms.  With the
// window differences dRP, dRS, dHP, dHS, dRPl (the lambda-mu term's R_P) and
// dHh = dS_S - dS_P the kernel collapses to
//   out_ik = b1 (a1 x_i n_k + a2 x_k n_i) + b2 delta_ik - b3 w_i x_k - b4 u_ik,
//   w = v x x,  u_ik = sum_j eps_jik v_j,
//   b1 = phik (ir^3 (dRP - dRS) + ir^2 (dHP/c_P - dHS/c_S)),
//   b2 = phik (x.n) (ir^3 dRS + ir^2 dHS/c_S),
//   b3 = c2 ir^3 (dRP/c_P^2 - dRS/c_S^2) - 3 c2 ir^5 dHh,
//   b4 = c1 ir (dRPl/c_P^2 - dRS/c_S^2) - c2 ir^3 dHh,
// a1 = lambda/(lambda+mu), a2 = mu/(lambda+mu), c1 = lambda mu/(rho(lambda+mu)),
// c2 = 2 mu/rho.
__host__ __device__ __forceinline__ void k_pair(double out[9], const double x[3], double ir, const double n[3],
                                                const double v[3], double phik, double dRP, double dRS, double dHP,
                                                double dHS, double dRPl, double dHh, const KCoef& c) {
    const double ir2 = ir * ir, ir3 = ir2 * ir, ir5 = ir3 * ir2;
    const double xn = x[0] * n[0] + x[1] * n[1] + x[2] * n[2];
    const double b1 = phik * (ir3 * (dRP - dRS) + ir2 * (dHP * c.icP - dHS * c.icS));
    const double b2 = phik * xn * (ir3 * dRS + ir2 * dHS * c.icS);
    const double b3 = c.c2 * ir3 * (dRP * c.icP2 - dRS * c.icS2) - 3 * c.c2 * ir5 * dHh;
    const double b4 = c.c1 * ir * (dRPl * c.icP2 - dRS * c.icS2) - c.c2 * ir3 * dHh;
    const double w[3] = {v[1] * x[2] - v[2] * x[1], v[2] * x[0] - v[0] * x[2], v[0] * x[1] - v[1] * x[0]};
    const double u[9] = {0, v[2], -v[1], -v[2], 0, v[0], v[1], -v[0], 0};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++)
            out[3 * i + k] = b1 * (c.a1 * x[i] * n[k] + c.a2 * x[k] * n[i]) + ((i == k) ? b2 : 0.0) -
                             b3 * w[i] * x[k] - b4 * u[3 * i + k];
}

// Register caps of the double-layer kernels, from an A/B of builds on the
// 448- and 2800-triangle bars (rule 7/4/3): the thread kernel at 128
// registers (4 blocks per SM: 725 -> 633 ms; 80 registers 721 ms), the warp
// kernel at 80 (6 blocks per SM: 28.8 -> 23.4 ms; 128 registers 24.3 ms).
__global__ void __launch_bounds__(128, 4) k_assemble_kernel(KArgs A) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)A.N * A.Nv) return;
    const int x = (int)(p % A.N), s = (int)(p / A.N);
    const DirTri& X = A.tri[x];
    // isBlockNull (kernelK.cu:234-262), distMin starting at 100 unless fixed
    double distMax = 0.0, distMin = A.fix ? 1e300 : 100.0;
    for (int a = 0; a < 3; a++) {
        const double d0 = X.V[a][0] - A.coords[3 * s], d1 = X.V[a][1] - A.coords[3 * s + 1],
                     d2 = X.V[a][2] - A.coords[3 * s + 2];
        const double d = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        distMax = fmax(distMax, d);
        distMin = fmin(distMin, d);
    }
    int llo = -1, lhi = -2;
    for (int q = 0; q < A.nlag; q++) {
        const int l = A.lag0 + q;
        if (l >= A.nblocks) break;
        const bool null = ((l - 2) * A.p.cS * A.dt > distMax + A.max_len) || ((l + 1) * A.p.cP * A.dt < distMin - 2 * A.max_len);
        if (!null) {
            if (llo < 0) llo = l;
            lhi = l;
        }
    }
    if (llo < 0) return;
    const int e0 = A.vt_off[s], e1 = A.vt_off[s + 1];
    const double cP = A.p.cP, cS = A.p.cS, dt = A.dt;
    const KCoef cd = k_coef(A.p);
    for (int l = llo; l <= lhi; l++) {
        // node pairs provably outside the window's fronts are skipped on r^2:
        // all four levels before the P front, or all after the S front
        const bool lin = !A.fix && l < 3;
        const double thi = (l + 1) * dt, tlo = (l - 2) * dt;
        const double skipP2 = lin ? 1e300 : (cP * thi) * (cP * thi) * (1 + 1e-12);
        const double skipS2 = (l >= 3) ? (cS * tlo) * (cS * tlo) * (1 - 1e-12) : -1.0;
        double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int ee = e0; ee < e1; ee++) {
            const int m = A.vt_tri[ee];
            if (m == x) continue;
            const int kv = local_index(A.tris, m, s);
            const DirTri& F = A.tri[m];
            const double g[3] = {F.M[3 * (kv - 1)], F.M[3 * (kv - 1) + 1], F.M[3 * (kv - 1) + 2]};
            const double vms[3] = {F.n[1] * g[2] - F.n[2] * g[1], F.n[2] * g[0] - F.n[0] * g[2], F.n[0] * g[1] - F.n[1] * g[0]};
            for (int q = 0; q < A.n_in; q++) {
                double y[3];
                bary_point(y, A.inner + 3 * q, F.V);
                const double phik = F.v[kv - 1] + g[0] * y[0] + g[1] * y[1] + g[2] * y[2];
                const double wi = A.win[q % A.n_sing] * F.area;
                for (int o = 0; o < A.n_gh; o++) {
                    double xo[3];
                    bary_point(xo, A.outer + 3 * o, X.V);
                    const double pt[3] = {xo[0] - y[0], xo[1] - y[1], xo[2] - y[2]};
                    const double r2 = pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2];
                    if (r2 > skipP2 || r2 < skipS2) continue;
                    const double r = sqrt(r2);
                    const double tP = r / cP, tS = r / cS;
                    const Win3 P = front_window3(tP, l, dt), S = front_window3(tS, l, dt);
                    const double dRPl = A.fix ? P.R : ((r - tP > 0) ? lin_window3(tP, l, dt) : 0.0);
                    const double dHh = S.S - P.S;
                    const double w = (A.wout[o] * X.area) * wi;
                    double v[9];
                    k_pair(v, pt, 1.0 / r, F.n, vms, phik, P.R, S.R, P.H, S.H, dRPl, dHh, cd);
#pragma unroll
                    for (int e = 0; e < 9; e++) T[e] += w * v[e];
                }
            }
        }
        double* base = A.K + (size_t)(l - A.lag0) * A.ld_lag + (3 * (size_t)s) * A.ld + 3 * (size_t)x;
        const double c = 4 * kPi * dt;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                if (fabs(T[3 * i + j]) > 1.0e-14) base[(size_t)j * A.ld + i] += T[3 * i + j] / c;
    }
}

// Warp-per-pair variant of k_assemble_kernel: one warp per (triangle x,
// vertex s), the lanes over the node pairs (star triangle of s, inner node,
// outer node), the same per-node-pair arithmetic, a warp reduction per lag.
__global__ void __launch_bounds__(128, 6) k_assemble_warp_kernel(KArgs A) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const double cP = A.p.cP, cS = A.p.cS, dt = A.dt;
    const KCoef cd = k_coef(A.p);
    const int per_tri = A.n_in * A.n_gh;
    for (long long p = warp; p < (long long)A.N * A.Nv; p += nwarps) {
        const int x = (int)(p % A.N), s = (int)(p / A.N);
        const DirTri& X = A.tri[x];
        double distMax = 0.0, distMin = A.fix ? 1e300 : 100.0;
        for (int a = 0; a < 3; a++) {
            const double d0 = X.V[a][0] - A.coords[3 * s], d1 = X.V[a][1] - A.coords[3 * s + 1],
                         d2 = X.V[a][2] - A.coords[3 * s + 2];
            const double d = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            distMax = fmax(distMax, d);
            distMin = fmin(distMin, d);
        }
        int llo = -1, lhi = -2;
        for (int q = 0; q < A.nlag; q++) {
            const int l = A.lag0 + q;
            if (l >= A.nblocks) break;
            const bool null = ((l - 2) * A.p.cS * A.dt > distMax + A.max_len) ||
                              ((l + 1) * A.p.cP * A.dt < distMin - 2 * A.max_len);
            if (!null) {
                if (llo < 0) llo = l;
                lhi = l;
            }
        }
        if (llo < 0) continue;
        const int e0 = A.vt_off[s], e1 = A.vt_off[s + 1];
        const int NP = (e1 - e0) * per_tri;
        // the node pairs' exact distance range (warp min/max): lags in which
        // every node pair would be skipped below add nothing and are skipped
        // by the whole warp (the null test above bounds them by vertex
        // distances and triangle sizes only)
        double r2min = 1e300, r2max = 0.0;
        for (int np = lane; np < NP; np += 32) {
            const int ee = e0 + np / per_tri, rem = np - (np / per_tri) * per_tri;
            const int m = A.vt_tri[ee];
            if (m == x) continue;
            const int qi = rem / A.n_gh, o = rem - qi * A.n_gh;
            double y[3], xo[3];
            bary_point(y, A.inner + 3 * qi, A.tri[m].V);
            bary_point(xo, A.outer + 3 * o, X.V);
            const double pt[3] = {xo[0] - y[0], xo[1] - y[1], xo[2] - y[2]};
            const double r2 = pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2];
            r2min = fmin(r2min, r2);
            r2max = fmax(r2max, r2);
        }
        for (int off = 16; off > 0; off >>= 1) {
            r2min = fmin(r2min, __shfl_xor_sync(0xffffffffu, r2min, off));
            r2max = fmax(r2max, __shfl_xor_sync(0xffffffffu, r2max, off));
        }
        for (int l = llo; l <= lhi; l++) {
            const bool lin = !A.fix && l < 3;
            const double thi = (l + 1) * dt, tlo = (l - 2) * dt;
            const double skipP2 = lin ? 1e300 : (cP * thi) * (cP * thi) * (1 + 1e-12);
            const double skipS2 = (l >= 3) ? (cS * tlo) * (cS * tlo) * (1 - 1e-12) : -1.0;
            if (r2min > skipP2 || r2max < skipS2) continue;
            double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int np = lane; np < NP; np += 32) {
                const int ee = e0 + np / per_tri, rem = np - (np / per_tri) * per_tri;
                const int m = A.vt_tri[ee];
                if (m == x) continue;
                const int qi = rem / A.n_gh, o = rem - qi * A.n_gh;
                const int kv = local_index(A.tris, m, s);
                const DirTri& F = A.tri[m];
                const double g[3] = {F.M[3 * (kv - 1)], F.M[3 * (kv - 1) + 1], F.M[3 * (kv - 1) + 2]};
                double y[3], xo[3];
                bary_point(y, A.inner + 3 * qi, F.V);
                bary_point(xo, A.outer + 3 * o, X.V);
                const double pt[3] = {xo[0] - y[0], xo[1] - y[1], xo[2] - y[2]};
                const double r2 = pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2];
                if (r2 > skipP2 || r2 < skipS2) continue;
                const double vms[3] = {F.n[1] * g[2] - F.n[2] * g[1], F.n[2] * g[0] - F.n[0] * g[2],
                                       F.n[0] * g[1] - F.n[1] * g[0]};
                const double phik = F.v[kv - 1] + g[0] * y[0] + g[1] * y[1] + g[2] * y[2];
                const double wi = A.win[qi % A.n_sing] * F.area;
                const double r = sqrt(r2);
                const double tP = r / cP, tS = r / cS;
                const Win3 P = front_window3(tP, l, dt), S = front_window3(tS, l, dt);
                const double dRPl = A.fix ? P.R : ((r - tP > 0) ? lin_window3(tP, l, dt) : 0.0);
                const double w = (A.wout[o] * X.area) * wi;
                double v[9];
                k_pair(v, pt, 1.0 / r, F.n, vms, phik, P.R, S.R, P.H, S.H, dRPl, S.S - P.S, cd);
#pragma unroll
                for (int e = 0; e < 9; e++) T[e] += w * v[e];
            }
#pragma unroll
            for (int e = 0; e < 9; e++)
                for (int off = 16; off > 0; off >>= 1) T[e] += __shfl_xor_sync(0xffffffffu, T[e], off);
            if (lane < 9) {
                const int ii = lane / 3, jj = lane - 3 * ii;
                double v = 0;
#pragma unroll
                for (int e = 0; e < 9; e++)
                    if (e == lane) v = T[e];
                double* base = A.K + (size_t)(l - A.lag0) * A.ld_lag + (3 * (size_t)s) * A.ld + 3 * (size_t)x;
                if (fabs(v) > 1.0e-14) base[(size_t)jj * A.ld + ii] += v / (4 * kPi * dt);
            }
        }
    }
}

// Same-triangle parts of K_l, in two passes.  Levels: one warp per (triangle
// x, local vertex kv, level k) over the call's levels kmin..kmin+nk-1, the
// lanes over the (outer node, child, DIAG node) evaluations, reduced over the
// warp into Tb[3x + kv - 1][k - kmin]; a level outside the triangle's own
// range klo..khi (its parts vanish from lag lmax on) is left unwritten and
// never read.  Emission: one thread per (x, kv, lag) adds the third
// difference (k_emit), levels below klo read as zero.  (One thread per
// (x, kv) walking all levels left most SMs idle on small meshes.)
struct KSingRange {
    int llo, lhi, klo, khi;
};
__device__ __forceinline__ KSingRange k_sing_range(const KArgs& A, const DirTri& X) {
    KSingRange r;
    const int lmax = (int)ceil(X.maxL / (A.p.cS * A.dt)) + 2;      // lags >= lmax are zero
    r.llo = A.lag0;
    r.lhi = min(A.lag0 + A.nlag - 1, lmax - 1);
    r.klo = max(1, r.llo - 2);
    r.khi = r.lhi + 1;
    return r;
}

__global__ void __launch_bounds__(128) k_sing_level_kernel(KArgs A, const double* __restrict__ dn,
                                                           const double* __restrict__ dw, int n_diag, int kmin, int nk,
                                                           double* __restrict__ Tb) {
    const int lane = threadIdx.x & 31;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= 3LL * A.N * nk) return;                    // uniform across the warp
    const int p = (int)(w / nk), kk = (int)(w - (long long)p * nk);
    const int x = p / 3, kv = p % 3 + 1;
    const DirTri& X = A.tri[x];
    const KSingRange rg = k_sing_range(A, X);
    const int k = kmin + kk;
    if (rg.lhi < rg.llo || k < rg.klo || k > rg.khi) return;
    const double t = k * A.dt;
    const double g[3] = {X.M[3 * (kv - 1)], X.M[3 * (kv - 1) + 1], X.M[3 * (kv - 1) + 2]};
    const double vms[3] = {X.n[1] * g[2] - X.n[2] * g[1], X.n[2] * g[0] - X.n[0] * g[2], X.n[0] * g[1] - X.n[1] * g[0]};
    const int per_o = 3 * n_diag, total = A.n_gh * per_o;
    double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = lane; c < total; c += 32) {
        const int o = c / per_o, rem = c - o * per_o, ch = rem / n_diag, d = rem - ch * n_diag;
        double xo[3];
        bary_point(xo, A.outer + 3 * o, X.V);
        const int a = ch, b = (ch + 2) % 3;               // children (V1,V3,x), (V2,V1,x), (V3,V2,x)
        const double ea[3] = {X.V[a][0] - xo[0], X.V[a][1] - xo[1], X.V[a][2] - xo[2]};
        const double eb[3] = {X.V[b][0] - xo[0], X.V[b][1] - xo[1], X.V[b][2] - xo[2]};
        const double cr[3] = {ea[1] * eb[2] - ea[2] * eb[1], ea[2] * eb[0] - ea[0] * eb[2], ea[0] * eb[1] - ea[1] * eb[0]};
        const double ac = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) / 2;
        const double* bd = dn + 3 * d;
        double y[3];
#pragma unroll
        for (int q = 0; q < 3; q++) y[q] = bd[0] * X.V[a][q] + bd[1] * X.V[b][q] + bd[2] * xo[q];
        const double R[3] = {xo[0] - y[0], xo[1] - y[1], xo[2] - y[2]};
        const double r = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
        const double phik = X.v[kv - 1] + g[0] * y[0] + g[1] * y[1] + g[2] * y[2];
        double v[9];
        kern_k(v, R, r, X.n, t, vms, phik, A.p, false, false);
        const double wgt = (X.area * A.wout[o]) * (dw[d] * ac);
#pragma unroll
        for (int e = 0; e < 9; e++) T[e] += wgt * v[e];
    }
#pragma unroll
    for (int e = 0; e < 9; e++)
        for (int off = 16; off > 0; off >>= 1) T[e] += __shfl_xor_sync(0xffffffffu, T[e], off);
    if (lane < 9) {
        double v = 0.0;
#pragma unroll
        for (int e = 0; e < 9; e++)
            if (e == lane) v = T[e];
        Tb[((size_t)p * nk + kk) * 9 + lane] = v;
    }
}

__global__ void __launch_bounds__(128) k_sing_emit_kernel(KArgs A, int kmin, int nk, const double* __restrict__ Tb) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 3LL * A.N * A.nlag) return;
    const int p = (int)(idx / A.nlag), q = (int)(idx - (long long)p * A.nlag);
    const int x = p / 3, kv = p % 3 + 1;
    const KSingRange rg = k_sing_range(A, A.tri[x]);
    const int l = A.lag0 + q;
    if (l > rg.lhi) return;
    double Tl[4][9];                                    // levels l-2, l-1, l, l+1
#pragma unroll
    for (int h = 0; h < 4; h++) {
        const int k = l - 2 + h;
#pragma unroll
        for (int e = 0; e < 9; e++) Tl[h][e] = (k >= rg.klo) ? Tb[((size_t)p * nk + (k - kmin)) * 9 + e] : 0.0;
    }
    k_emit(A, l, x, A.tris[3 * x + kv - 1], Tl[0], Tl[1], Tl[2], Tl[3], false);
}

// Diagonal blocks of V_l on the DIAG rule, in two passes.  Levels: one warp
// per (triangle x, time level k), the lanes over the (outer node, child, DIAG
// node) evaluations of the level integral T_k (9 entries), reduced over the
// warp into Tb[x][k - kmin].  Combine: one thread per (triangle, lag, entry),
// V_l = (T_{l+1} - 2 T_l + T_{l-1}) / (4 pi rho) with T_0 taken as zero.
// (One thread per triangle walking every level left all but a few SMs idle
// on meshes of a few hundred triangles.)
__global__ void __launch_bounds__(128) v_diag_level_kernel(const DirTri* __restrict__ tri, int N,
                                                           const double* __restrict__ outer,
                                                           const double* __restrict__ wout, int n_gh,
                                                           const double* __restrict__ dn, const double* __restrict__ dw,
                                                           int n_diag, double cP, double cS, double dt, int kmin, int nk,
                                                           double* __restrict__ Tb) {
    const int lane = threadIdx.x & 31;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= (long long)N * nk) return;                 // uniform across the warp
    const int x = (int)(w / nk), kk = (int)(w - (long long)x * nk);
    const double t = (kmin + kk) * dt;
    const DirTri& X = tri[x];
    const int per_o = 3 * n_diag, total = n_gh * per_o;
    double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = lane; c < total; c += 32) {
        const int o = c / per_o, rem = c - o * per_o, ch = rem / n_diag, d = rem - ch * n_diag;
        double xo[3];
        bary_point(xo, outer + 3 * o, X.V);
        const int a = ch, b = (ch + 2) % 3;
        const double ea[3] = {X.V[a][0] - xo[0], X.V[a][1] - xo[1], X.V[a][2] - xo[2]};
        const double eb[3] = {X.V[b][0] - xo[0], X.V[b][1] - xo[1], X.V[b][2] - xo[2]};
        const double cr[3] = {ea[1] * eb[2] - ea[2] * eb[1], ea[2] * eb[0] - ea[0] * eb[2], ea[0] * eb[1] - ea[1] * eb[0]};
        const double ac = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) / 2;
        const double* bd = dn + 3 * d;
        double X3[3];
#pragma unroll
        for (int q = 0; q < 3; q++) X3[q] = (bd[0] * X.V[a][q] + bd[1] * X.V[b][q] + bd[2] * xo[q]) - xo[q];
        double nu[9];
        kern_v(nu, X3, sqrt(X3[0] * X3[0] + X3[1] * X3[1] + X3[2] * X3[2]), t, cP, cS);
        const double wgt = (X.area * wout[o]) * (dw[d] * ac);
#pragma unroll
        for (int e = 0; e < 9; e++) T[e] += wgt * nu[e];
    }
#pragma unroll
    for (int e = 0; e < 9; e++)
        for (int off = 16; off > 0; off >>= 1) T[e] += __shfl_xor_sync(0xffffffffu, T[e], off);
    if (lane < 9) {
        double v = 0.0;
#pragma unroll
        for (int e = 0; e < 9; e++)
            if (e == lane) v = T[e];
        Tb[((size_t)x * nk + kk) * 9 + lane] = v;
    }
}

__global__ void __launch_bounds__(128) v_diag_combine_kernel(const double* __restrict__ Tb, int N, int kmin, int nk,
                                                             int lag0, int nlag, double c4pirho, double* __restrict__ V,
                                                             size_t ld, size_t ld_lag) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * nlag * 9) return;
    const int e = (int)(idx % 9);
    const long long r = idx / 9;
    const int q = (int)(r % nlag), x = (int)(r / nlag);
    const int l = lag0 + q, k = l + 1;
    auto level = [&](int kk) {
        return (kk >= kmin && kk < kmin + nk) ? Tb[((size_t)x * nk + (kk - kmin)) * 9 + e] : 0.0;
    };
    const double prev = (l - 1 >= 1) ? level(k - 2) : 0.0;
    const int i = e / 3, j = e - 3 * i;
    V[(size_t)q * ld_lag + (3 * (size_t)x + j) * ld + 3 * (size_t)x + i] = ((level(k) - 2 * level(k - 1)) + prev) / c4pirho;
}

// Rule tables in one device buffer.
struct Tables {
    double* d = nullptr;
    size_t outer = 0, wout = 0, inner = 0, win = 0, dn = 0, dw = 0;
    cudaStream_t st = nullptr;
    ~Tables() { ws_free(d, st); }
};

static int upload_tables(Tables& T, int n_gh, int n_sub, int n_sing, int n_diag, cudaStream_t s) {
    std::vector<double> buf;
    double ob[28 * 3], ow[28];
    if (n_gh > 0) {
        if (gh_composite(n_gh, 1, ob, ow)) return fail(EBEM_ERR_INVALID, "unsupported outer rule");
        T.outer = buf.size(); buf.insert(buf.end(), ob, ob + 3 * n_gh);
        T.wout = buf.size(); buf.insert(buf.end(), ow, ow + n_gh);
    }
    if (n_sing > 0) {
        std::vector<double> ib((size_t)3 * n_sub * n_sing), iw(n_sing);
        if (gh_composite(n_sing, n_sub, ib.data(), iw.data())) return fail(EBEM_ERR_INVALID, "unsupported inner rule");
        T.inner = buf.size(); buf.insert(buf.end(), ib.begin(), ib.end());
        T.win = buf.size(); buf.insert(buf.end(), iw.begin(), iw.end());
    }
    if (n_diag > 0) {
        std::vector<double> dn, dw;
        if (diag_rule(n_diag, dn, dw)) return fail(EBEM_ERR_INVALID, "DIAG rule size must be a square");
        T.dn = buf.size(); buf.insert(buf.end(), dn.begin(), dn.end());
        T.dw = buf.size(); buf.insert(buf.end(), dw.begin(), dw.end());
    }
    if (buf.empty()) buf.push_back(0.0);
    T.st = s;
    EBEM_CUDA_TRY(ws_malloc(&T.d, buf.size() * sizeof(double), s));
    EBEM_CUDA_TRY(cudaMemcpyAsync(T.d, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    return EBEM_OK;
}

static Mat mat_of(const PhysParams& P) {
    Mat p;
    p.lam = P.lam;
    p.mu = P.mu;
    p.rho = P.rho;
    p.cP = P.velP;
    p.cS = P.velS;
    return p;
}

int launch_k_assemble(const MeshData& m, const PhysParams& P, int n_gh, int n_sub, int n_sing, int n_diag, int lag0,
                      int nlag, int nblocks, int fix, double* d_K, cudaStream_t s) {
    Tables T;
    if (int rc = upload_tables(T, n_gh, n_sub, n_sing, n_diag, s)) return rc;
    KArgs A;
    A.tri = m.d_dir;
    A.coords = m.d_coords;
    A.tris = m.d_tris;
    A.vt_off = m.d_vt_off;
    A.vt_tri = m.d_vt_tri;
    A.outer = T.d + T.outer;
    A.wout = T.d + T.wout;
    A.inner = T.d + T.inner;
    A.win = T.d + T.win;
    A.n_gh = n_gh;
    A.n_in = n_sub * n_sing;
    A.n_sing = n_sing;
    A.N = m.nt;
    A.Nv = m.nv;
    A.p = mat_of(P);
    A.dt = P.dt;
    A.max_len = m.max_len;
    A.lag0 = lag0;
    A.nlag = nlag;
    A.nblocks = nblocks;
    A.fix = fix;
    A.K = d_K;
    A.ld = 3 * (size_t)m.nt;
    A.ld_lag = A.ld * 3 * (size_t)m.nv;
    const long long pairs = (long long)m.nt * m.nv;
    // warp per pair only when the thread kernel would not fill the GPU
    // (fewer pairs than two waves of threads; measured: bar of 448 triangles
    // 1.08x faster, bar of 2800 triangles 1.37x slower)
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device);
    if (n_sub * n_sing * n_gh >= EBEM_K_WARP_MIN_NODE_PAIRS && pairs < (long long)sms * EBEM_K_WARP_MAX_PAIRS_PER_SM) {
        const long long want = (pairs + 3) / 4, cap = (long long)sms * 64;
        k_assemble_warp_kernel<<<(unsigned)(want < cap ? want : cap), 128, 0, s>>>(A);
    } else {
        k_assemble_kernel<<<(unsigned)((pairs + 127) / 128), 128, 0, s>>>(A);
    }
    EBEM_CUDA_TRY(cudaGetLastError());
    if (n_diag > 0) {
        const int kmin = std::max(1, lag0 - 2), nk = lag0 + nlag - kmin + 1;
        double* Tb = nullptr;
        EBEM_CUDA_TRY(ws_malloc(&Tb, sizeof(double) * 27 * (size_t)m.nt * nk, s));
        const long long lv_threads = 32LL * 3 * m.nt * nk, em_threads = 3LL * m.nt * nlag;
        k_sing_level_kernel<<<(unsigned)((lv_threads + 127) / 128), 128, 0, s>>>(A, T.d + T.dn, T.d + T.dw, n_diag, kmin,
                                                                                  nk, Tb);
        k_sing_emit_kernel<<<(unsigned)((em_threads + 127) / 128), 128, 0, s>>>(A, kmin, nk, Tb);
        cudaError_t e = cudaGetLastError();
        ws_free(Tb, s);
        if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("K same-triangle parts: ") + cudaGetErrorString(e));
    }
    EBEM_CUDA_TRY(cudaStreamSynchronize(s));
    return EBEM_OK;
}

int launch_v_diag(const MeshData& m, const PhysParams& P, int n_gh, int n_diag, int lag0, int nlag, double* d_V,
                  cudaStream_t s) {
    Tables T;
    if (int rc = upload_tables(T, n_gh, 0, 0, n_diag, s)) return rc;
    const size_t ld = 3 * (size_t)m.nt;
    // levels k = kmin .. lag0 + nlag (t = k dt; t = 0 contributes nothing)
    const int kmin = std::max(1, lag0 - 1), nk = lag0 + nlag - kmin + 1;
    double* Tb = nullptr;
    EBEM_CUDA_TRY(ws_malloc(&Tb, sizeof(double) * 9 * (size_t)m.nt * nk, s));
    const long long lv_threads = 32LL * m.nt * nk, cb_threads = 9LL * m.nt * nlag;
    v_diag_level_kernel<<<(unsigned)((lv_threads + 127) / 128), 128, 0, s>>>(
        m.d_dir, m.nt, T.d + T.outer, T.d + T.wout, n_gh, T.d + T.dn, T.d + T.dw, n_diag, P.velP, P.velS, P.dt, kmin,
        nk, Tb);
    v_diag_combine_kernel<<<(unsigned)((cb_threads + 127) / 128), 128, 0, s>>>(Tb, m.nt, kmin, nk, lag0, nlag,
                                                                               4 * kPi * P.rho, d_V, ld, ld * ld);
    cudaError_t e = cudaGetLastError();
    ws_free(Tb, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("V diagonal blocks: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// post-processing: one thread per (triangle or vertex, evaluation (t, x))

struct PPArgs {
    const DirTri* tri;
    const int32_t* tris;
    const int32_t* vt_off;
    const int32_t* vt_tri;
    const double* pn;        // n_sub * n_sing x 3
    const double* pw;        // n_sing
    int n_sub, n_sing, gstride;
    int N, Nv;
    Mat p;
    double dt;
    const double* pts;       // npts x 3
    const double* times;     // ntimes (device copy)
    int npts, ntimes, nT;
    const double* a;         // 3N x nT  (multiplies G)
    const double* b;         // 3Nv x nT (multiplies P)
    double* u;               // ntimes x npts x 3
    double* G;               // matrix mode
    double* Pm;
    int mode;
};

__device__ __forceinline__ void warp_add3(double* dst, double v0, double v1, double v2) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
        v2 += __shfl_xor_sync(0xffffffffu, v2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (v0 != 0.0) atomicAdd(dst, v0);
        if (v1 != 0.0) atomicAdd(dst + 1, v1);
        if (v2 != 0.0) atomicAdd(dst + 2, v2);
    }
}

// G part: sum over slices n of clamp(G(t - (n-1) dt) - G(t - n dt)) / (4 pi rho) a_n.
// Block (x-tile, evaluation, chunk c) takes the slices n in
// [c kchunk + 1, (c + 1) kchunk] and evaluates G at the levels n_lo - 1 .. n_hi
// (one level more than its slices), so that short meshes still fill the GPU.
// kernelG / kernelP evaluations capped at 128 registers (4 blocks per SM):
// 16 points x 4 times on the 448-triangle bar 3.51 -> 3.23 ms (80 registers:
// 3.63 ms, the spills then cost more than the occupancy gains).
__global__ void __launch_bounds__(128, 4) pp_g_kernel(PPArgs A, int kchunk) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int ev = blockIdx.y;                          // evaluation index q * npts + ip
    const int q = ev / A.npts, ip = ev % A.npts;
    const double t = A.times[q];
    const double* src = A.pts + 3 * ip;
    const int nhat = (t > 0) ? (int)ceil(t / A.dt) : 0;
    const int n_lo = blockIdx.z * kchunk + 1, n_hi = min((int)(blockIdx.z + 1) * kchunk, nhat);
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    if (x < A.N && n_lo <= n_hi) {
        const DirTri& X = A.tri[x];
        double Gp[9] = {0}, Gk[9];
        const double c4 = 4 * kPi * A.p.rho;
        for (int k = n_lo - 1; k <= n_hi; k++) {
            const double tk = t - k * A.dt;
#pragma unroll
            for (int e = 0; e < 9; e++) Gk[e] = 0.0;
            if (tk > 0) {
                for (int tx = 0; tx < A.n_sub; tx++)
                    for (int l = 0; l < A.n_sing; l++) {
                        double y[3];
                        bary_point(y, A.pn + 3 * (A.gstride * tx + l), X.V);
                        const double pt[3] = {y[0] - src[0], y[1] - src[1], y[2] - src[2]};
                        double nu[9];
                        kern_v(nu, pt, sqrt(pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2]), tk, A.p.cP, A.p.cS);
                        const double w = A.pw[l] * X.area;
#pragma unroll
                        for (int e = 0; e < 9; e++) Gk[e] += w * nu[e];
                    }
            }
            if (k >= n_lo) {
                const int n = k;                        // slice n uses instants t - (n-1) dt and t - n dt
                double S[9];
#pragma unroll
                for (int e = 0; e < 9; e++) {
                    const double v = Gp[e] - Gk[e];
                    S[e] = (fabs(v) > 1.0e-14) ? v / c4 : 0.0;
                }
                if (A.mode == 1) {
                    const size_t R = 3 * (size_t)nhat;
#pragma unroll
                    for (int i = 0; i < 3; i++)
#pragma unroll
                        for (int j = 0; j < 3; j++) A.G[(3 * (size_t)x + j) * R + 3 * (size_t)(n - 1) + i] = S[3 * i + j];
                } else if (n <= A.nT) {
                    const double* an = A.a + (size_t)(n - 1) * 3 * A.N + 3 * (size_t)x;
                    u0 += S[0] * an[0] + S[1] * an[1] + S[2] * an[2];
                    u1 += S[3] * an[0] + S[4] * an[1] + S[5] * an[2];
                    u2 += S[6] * an[0] + S[7] * an[1] + S[8] * an[2];
                }
            }
#pragma unroll
            for (int e = 0; e < 9; e++) Gp[e] = Gk[e];
        }
    }
    if (A.mode == 0) warp_add3(A.u + 3 * (size_t)ev, u0, u1, u2);
}

// P part: minus the sum over slices n of clamp(P_{n-1} - 2 P_n + P_{n+1}) / (4 pi rho dt) b_n.
// Chunked over the slices as pp_g_kernel; a chunk evaluates P at the levels
// n_lo - 1 .. n_hi + 1.
__global__ void __launch_bounds__(128, 4) pp_p_kernel(PPArgs A, int kchunk) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int ev = blockIdx.y;
    const int q = ev / A.npts, ip = ev % A.npts;
    const double t = A.times[q];
    const double* src = A.pts + 3 * ip;
    const int nhat = (t > 0) ? (int)ceil(t / A.dt) : 0;
    const int n_lo = blockIdx.z * kchunk + 1, n_hi = min((int)(blockIdx.z + 1) * kchunk, nhat);
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    if (s < A.Nv && n_lo <= n_hi) {
        double Pm2[9] = {0}, Pm1[9] = {0}, Pk[9];
        const double c4 = 4 * kPi * A.p.rho * A.dt;
        const int e0 = A.vt_off[s], e1 = A.vt_off[s + 1];
        for (int k = n_lo - 1; k <= n_hi + 1; k++) {
            const double tk = t - k * A.dt;
#pragma unroll
            for (int e = 0; e < 9; e++) Pk[e] = 0.0;
            if (tk > 0) {
                for (int ee = e0; ee < e1; ee++) {
                    const int m = A.vt_tri[ee];
                    const int kv = local_index(A.tris, m, s);
                    const DirTri& F = A.tri[m];
                    const double* g = F.M + 3 * (kv - 1);
                    for (int tx = 0; tx < A.n_sub; tx++)
                        for (int l = 0; l < A.n_sing; l++) {
                            double y[3];
                            bary_point(y, A.pn + 3 * (A.n_sing * tx + l), F.V);
                            const double pt[3] = {src[0] - y[0], src[1] - y[1], src[2] - y[2]};
                            const double phik = F.v[kv - 1] + g[0] * y[0] + g[1] * y[1] + g[2] * y[2];
                            double nu[9];
                            kern_p(nu, pt, F.n, sqrt(pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2]), tk, phik, A.p);
                            const double w = A.pw[l] * F.area;
#pragma unroll
                            for (int e = 0; e < 9; e++) Pk[e] += w * nu[e];
                        }
                }
            }
            if (k >= n_lo + 1) {
                const int n = k - 1;                    // slice n: P_{n-1} - 2 P_n + P_{n+1}
                double S[9];
#pragma unroll
                for (int e = 0; e < 9; e++) {
                    const double v = (Pm2[e] - 2 * Pm1[e]) + Pk[e];
                    S[e] = (fabs(v) > 1.0e-14) ? v / c4 : 0.0;
                }
                if (n <= nhat) {
                    if (A.mode == 1) {
                        const size_t R = 3 * (size_t)nhat;
#pragma unroll
                        for (int i = 0; i < 3; i++)
#pragma unroll
                            for (int j = 0; j < 3; j++) A.Pm[(3 * (size_t)s + j) * R + 3 * (size_t)(n - 1) + i] = S[3 * i + j];
                    } else if (n <= A.nT) {
                        const double* bn = A.b + (size_t)(n - 1) * 3 * A.Nv + 3 * (size_t)s;
                        u0 -= S[0] * bn[0] + S[1] * bn[1] + S[2] * bn[2];
                        u1 -= S[3] * bn[0] + S[4] * bn[1] + S[5] * bn[2];
                        u2 -= S[6] * bn[0] + S[7] * bn[1] + S[8] * bn[2];
                    }
                }
            }
#pragma unroll
            for (int e = 0; e < 9; e++) { Pm2[e] = Pm1[e]; Pm1[e] = Pk[e]; }
        }
    }
    if (A.mode == 0) warp_add3(A.u + 3 * (size_t)ev, u0, u1, u2);
}

int launch_pp_dir(const MeshData& m, const PhysParams& P, int n_sub, int n_sing, int fix, const double* d_pts, int npts,
                  const double* h_times, int ntimes, const double* d_a, const double* d_b, double* d_u, double* d_G,
                  double* d_P, int mode, cudaStream_t s) {
    const int gstride = fix ? n_sing : 3;
    if (3 * (n_sub - 1) + n_sing > n_sub * n_sing && !fix)
        return fail(EBEM_ERR_INVALID, "the reference's node stride 3 needs n_sing >= 3 (or the fixed stride)");
    if ((long long)npts * ntimes > 65535)
        return fail(EBEM_ERR_INVALID, "at most 65535 (point, time) evaluations per call");
    Tables T;
    if (int rc = upload_tables(T, 0, n_sub, n_sing, 0, s)) return rc;
    double* d_times = nullptr;
    EBEM_CUDA_TRY(ws_malloc(&d_times, sizeof(double) * ntimes, s));
    cudaError_t e = cudaMemcpyAsync(d_times, h_times, sizeof(double) * ntimes, cudaMemcpyHostToDevice, s);
    PPArgs A;
    A.tri = m.d_dir;
    A.tris = m.d_tris;
    A.vt_off = m.d_vt_off;
    A.vt_tri = m.d_vt_tri;
    A.pn = T.d + T.inner;
    A.pw = T.d + T.win;
    A.n_sub = n_sub;
    A.n_sing = n_sing;
    A.gstride = gstride;
    A.N = m.nt;
    A.Nv = m.nv;
    A.p = mat_of(P);
    A.dt = P.dt;
    A.pts = d_pts;
    A.times = d_times;
    A.npts = npts;
    A.ntimes = ntimes;
    A.nT = P.nT;
    A.a = d_a;
    A.b = d_b;
    A.u = d_u;
    A.G = d_G;
    A.Pm = d_P;
    A.mode = mode;
    if (e == cudaSuccess) {
        // slices split into chunks over grid z so that about 8 blocks per SM
        // run (a chunk re-evaluates 1 (G) or 2 (P) boundary levels: at least
        // 4 and 8 slices per chunk keep that under a quarter)
        int nhat_max = 0;
        for (int q = 0; q < ntimes; q++)
            if (h_times[q] > 0) nhat_max = std::max(nhat_max, (int)std::ceil(h_times[q] / P.dt));
        nhat_max = std::max(nhat_max, 1);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device);
        const long long evs = (long long)npts * ntimes, target = 8LL * sms;
        auto chunk_of = [&](long long bxy, int kmin) {
            const long long want = (nhat_max * bxy + target - 1) / target;
            return (int)std::min<long long>(nhat_max, std::max<long long>(kmin, want));
        };
        const long long bg = (m.nt + 127) / 128, bp = (m.nv + 127) / 128;
        const int kg = chunk_of(bg * evs, 4), kp = chunk_of(bp * evs, 8);
        dim3 gg((unsigned)bg, (unsigned)evs, (unsigned)((nhat_max + kg - 1) / kg));
        dim3 gp((unsigned)bp, (unsigned)evs, (unsigned)((nhat_max + kp - 1) / kp));
        if (mode == 0) e = cudaMemsetAsync(d_u, 0, sizeof(double) * 3 * (size_t)npts * ntimes, s);
        if (e == cudaSuccess) {
            pp_g_kernel<<<gg, 128, 0, s>>>(A, kg);
            pp_p_kernel<<<gp, 128, 0, s>>>(A, kp);
            e = cudaGetLastError();
        }
    }
    ws_free(d_times, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("direct post-processing: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// time marching

// y += I_Gamma u: (3x+i) += area_x / 6 u(3s+i) for each vertex s of x
// (BEMenerg_dir_timeMarchingN.m:275, kron((indSM > 0) .* area / 6, eye(3))).
__global__ void mass_apply_kernel(const DirTri* __restrict__ tri, const int32_t* __restrict__ tris, int N,
                                  const double* __restrict__ u, double* __restrict__ y) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= N) return;
    const double c = tri[x].area / 6;
    for (int i = 0; i < 3; i++) {
        double acc = 0.0;
        for (int k = 0; k < 3; k++) acc += u[3 * tris[3 * x + k] + i];
        y[3 * x + i] += c * acc;
    }
}

// A += I_Gamma (A: 3N x 3Nv column-major).
__global__ void mass_add_kernel(const DirTri* __restrict__ tri, const int32_t* __restrict__ tris, int N,
                                double* __restrict__ A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= N) return;
    const double c = tri[x].area / 6;
    const size_t ld = 3 * (size_t)N;
    for (int k = 0; k < 3; k++) {
        const int s = tris[3 * x + k];
        for (int i = 0; i < 3; i++) A[(3 * (size_t)s + i) * ld + 3 * (size_t)x + i] += c;
    }
}

__global__ void copy_cols_rev_kernel(const double* __restrict__ src, double* __restrict__ dst, int n, int nT, int to_rev) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * nT) return;
    const int r = (int)(idx % n), c = (int)(idx / n);
    if (to_rev) dst[(size_t)(nT - 1 - c) * n + r] = src[idx];
    else dst[idx] = src[(size_t)(nT - 1 - c) * n + r];
}

// beta (rows x nT) += sum_l B_l * shift(g, l), B_l rows x cols per lag.
static int beta_gemm(cublasHandle_t hb, const double* dB, int L, int rows, int cols, const double* dg, int nT,
                     double* dbeta) {
    const double one = 1.0;
    for (int l = 0; l < L && l < nT; l++) {
        const double* Bl = dB + (size_t)l * rows * cols;
        cublasStatus_t st = cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, rows, nT - l, cols, &one, Bl, rows, dg, cols, &one,
                                        dbeta + (size_t)l * rows, rows);
        if (st != CUBLAS_STATUS_SUCCESS) return fail(EBEM_ERR_CUDA, "cublasDgemm failed in the data convolution");
    }
    return EBEM_OK;
}

int march_dn_device(const MeshData& m, const double* dV, int LV, const double* dK, int LK, const double* d_gV, int nT,
                    double* d_u, cudaStream_t s) {
    const int R = 3 * m.nt, Cn = 3 * m.nv;
    if (R < Cn) return fail(EBEM_ERR_INVALID, "least-squares system needs 3N >= 3Nv");
    int rc = EBEM_OK, dev = 0, sms = 148, lwork = 0, lw2 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cusolverDnHandle_t hs = nullptr;
    cublasHandle_t hb = nullptr;
    double *A = nullptr, *Q = nullptr, *X = nullptr, *tau = nullptr, *work = nullptr, *beta = nullptr, *rev = nullptr,
           *y = nullptr;
    int* info = nullptr;
    const double one = 1.0, zero = 0.0;
    auto cu = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && rc == EBEM_OK) rc = fail(EBEM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        return rc == EBEM_OK;
    };
    auto blas_ok = [&](cublasStatus_t st, const char* what) {
        if (st != CUBLAS_STATUS_SUCCESS && rc == EBEM_OK)
            rc = fail(EBEM_ERR_CUDA, std::string(what) + " failed (cuBLAS status " + std::to_string((int)st) + ")");
        return rc == EBEM_OK;
    };
    auto sol_ok = [&](cusolverStatus_t st, const char* what) {
        if (st != CUSOLVER_STATUS_SUCCESS && rc == EBEM_OK)
            rc = fail(EBEM_ERR_CUDA, std::string(what) + " failed (cuSOLVER status " + std::to_string((int)st) + ")");
        return rc == EBEM_OK;
    };
    const size_t RC = (size_t)R * Cn;
    if (!cu(ws_malloc(&A, sizeof(double) * RC, s), "alloc") || !cu(ws_malloc(&Q, sizeof(double) * RC, s), "alloc") ||
        !cu(ws_malloc(&X, sizeof(double) * RC, s), "alloc") || !cu(ws_malloc(&tau, sizeof(double) * Cn, s), "alloc") ||
        !cu(ws_malloc(&beta, sizeof(double) * (size_t)R * nT, s), "alloc") ||
        !cu(ws_malloc(&rev, sizeof(double) * (size_t)Cn * nT, s), "alloc") || !cu(ws_malloc(&y, sizeof(double) * R, s), "alloc") ||
        !cu(ws_malloc(&info, sizeof(int), s), "alloc")) {
        rc = fail(EBEM_ERR_NOMEM, "direct time-marching workspace allocation failed");
        goto done;
    }
    if ((rc = solver_handle(s, &hs)) || (rc = blas_handle(s, &hb))) goto done;
    // beta_V,n = sum_j V_{n-j} g_j
    if (!cu(cudaMemsetAsync(beta, 0, sizeof(double) * (size_t)R * nT, s), "memset")) goto done;
    if ((rc = beta_gemm(hb, dV, LV, R, R, d_gV, nT, beta))) goto done;
    // A = K_0 + I_Gamma = Q_1 R_1 (thin QR, once); the least-squares solution
    // of every step is u = X y with X = R_1^{-1} Q_1^T (Cn x R), formed once
    // (the reference solves (K_0 + I_Gamma) \ y densely at every step)
    if (!cu(cudaMemcpyAsync(A, dK, sizeof(double) * RC, cudaMemcpyDeviceToDevice, s), "copy")) goto done;
    mass_add_kernel<<<(m.nt + 127) / 128, 128, 0, s>>>(m.d_dir, m.d_tris, m.nt, A);
    if (!cu(cudaGetLastError(), "mass matrix")) goto done;
    if (!sol_ok(cusolverDnDgeqrf_bufferSize(hs, R, Cn, A, R, &lwork), "QR workspace query") ||
        !sol_ok(cusolverDnDorgqr_bufferSize(hs, R, Cn, Cn, A, R, tau, &lw2), "Q workspace query"))
        goto done;
    lwork = std::max(lwork, lw2);
    if (!cu(ws_malloc(&work, sizeof(double) * (size_t)std::max(lwork, 1), s), "alloc")) goto done;
    if (!sol_ok(cusolverDnDgeqrf(hs, R, Cn, A, R, tau, work, lwork, info), "QR factorisation")) goto done;
    if (!cu(cudaMemcpyAsync(Q, A, sizeof(double) * RC, cudaMemcpyDeviceToDevice, s), "copy")) goto done;
    if (!sol_ok(cusolverDnDorgqr(hs, R, Cn, Cn, Q, R, tau, work, lwork, info), "forming Q_1")) goto done;
    // X = Q_1^T (transpose; X zeroed first although geam reads no B when
    // beta = 0), then R_1 X = Q_1^T in place
    if (!cu(cudaMemsetAsync(X, 0, sizeof(double) * RC, s), "memset")) goto done;
    if (!blas_ok(cublasDgeam(hb, CUBLAS_OP_T, CUBLAS_OP_N, Cn, R, &one, Q, R, &zero, X, Cn, X, Cn), "transpose"))
        goto done;
    if (!blas_ok(cublasDtrsm(hb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, Cn, R, &one,
                             A, R, X, Cn),
                 "triangular solve for X"))
        goto done;
    // u in reversed time order: u_n at column nT-1-n
    if (!cu(cudaMemsetAsync(rev, 0, sizeof(double) * (size_t)Cn * nT, s), "memset")) goto done;
    for (int n = 0; n < nT; n++) {
        if (!cu(cudaMemcpyAsync(y, beta + (size_t)n * R, sizeof(double) * R, cudaMemcpyDeviceToDevice, s), "copy")) goto done;
        double* un = rev + (size_t)(nT - 1 - n) * Cn;
        if (n > 0) {
            mass_apply_kernel<<<(m.nt + 127) / 128, 128, 0, s>>>(m.d_dir, m.d_tris, m.nt, un + Cn, y);
            if (!cu(cudaGetLastError(), "mass apply")) goto done;
        }
        const int M = std::min(n + 1, LK) - 1;          // K_1 .. K_M
        if (M > 0 && (rc = launch_hist_gemv(dK + RC, R, (long long)Cn * M, un + Cn, y, sms, s))) goto done;
        if (!blas_ok(cublasDgemv(hb, CUBLAS_OP_N, Cn, R, &one, X, Cn, y, 1, &zero, un, 1), "least-squares product"))
            goto done;
    }
    {
        const long long tot = (long long)Cn * nT;
        copy_cols_rev_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(rev, d_u, Cn, nT, 0);
        cu(cudaGetLastError(), "copy");
    }
    cu(cudaStreamSynchronize(s), "direct time marching");
done:
    ws_free(A, s); ws_free(Q, s); ws_free(X, s); ws_free(tau, s); ws_free(work, s); ws_free(beta, s); ws_free(rev, s);
    ws_free(y, s); ws_free(info, s);
    return rc;
}

__global__ void half_add_kernel(const double* __restrict__ rhs, double* __restrict__ out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += rhs[i] / 2;
}

int march_dd_device(const MeshData& m, const double* dV, int LV, const double* dK, int LK, const double* d_rhs,
                    const double* d_gK, int nT, double* d_phi, cudaStream_t s) {
    const int R = 3 * m.nt, Cn = 3 * m.nv;
    double* b = nullptr;
    cublasHandle_t hb = nullptr;
    int rc = EBEM_OK;
    if (int e = blas_handle(s, &hb)) return e;
    if (ws_malloc(&b, sizeof(double) * (size_t)R * nT, s) != cudaSuccess)
        return fail(EBEM_ERR_NOMEM, "right-hand side allocation failed");
    // b = rhs / 2 + beta_K, beta_K,n = sum_j K_{n-j} gK_j
    if (cudaMemsetAsync(b, 0, sizeof(double) * (size_t)R * nT, s) != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "memset failed");
    if (!rc) rc = beta_gemm(hb, dK, LK, R, Cn, d_gK, nT, b);
    if (!rc) {
        const long long n = (long long)R * nT;
        half_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_rhs, b, n);
        if (cudaGetLastError() != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "rhs combination failed");
    }
    if (!rc) rc = march_device(dV, R, LV, b, nT, d_phi, s);
    cudaStreamSynchronize(s);
    ws_free(b, s);
    return rc;
}

}  // namespace ebem
