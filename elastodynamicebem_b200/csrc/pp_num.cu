// Numerical post-processing of the indirect formulation: the displacement
// u(x, t) from the density with a composite Gauss-Hammer rule on each
// triangle (the reference's post-processing method "GPU yy z").
//
// Reference (paths relative to the reference project root; "PG/" =
// functions/BEMenerg_indir/BEMenerg_postProc/BEMenerg_postProcGPU/):
//   PG/CUDAkernels/kernelSP.cu:5-105     one point, every history instant
//                                        (launched by PG/BEMenerg_postProcGPU_calcSP.m:60-69,
//                                        summed on the host at :78-85)
//   PG/CUDAkernels/kernelLayer.cu:5-175  many points at one time, the density
//                                        contraction in the kernel
//                                        (PG/BEMenerg_postProcGPU_calcLayer.m:64-71)
//   selected by main.m:165,167 (u(:, t) -> Layer, u(x, :) -> SP).
//
// Both evaluate, for a point x, a triangle m and an instant tau = t - k dt,
//   M_k(x, m) = sum over the composite nodes y of w_y |T_m| G(y - x, tau) / (4 pi rho)
// with G the Lamé kernel integrated twice in time (kernelGHC.cu:204-259's
// nucleo), skipped when tau c_P < |x - c_m| - maxL_m.  They differ in:
//   * the clean-up: kernelSP keeps an entry only when |sum| > 1e-14 before the
//     division by 4 pi rho (kernelSP.cu:97-100), kernelLayer zeroes entries
//     below 1e-14 after it (kernelLayer.cu:93-102);
//   * the node read: kernelSP reads node 3 * subregion + l (kernelSP.cu:41,
//     right only for 3 nodes per sub-triangle; reproduced unless
//     EBEM_FIX_REFERENCE_DEFECTS), kernelLayer node subregion * n_sing + l;
//   * the time sum: kernelSP's host sum is
//       u = sum_{k < nHat} (M_k - M_{k+1}) phi_k + M_nHat phi_nHat,
//     kernelLayer's is u = sum_{k <= nHat} M_k (phi_k - phi_{k-1}), phi_{-1} = 0,
//   nHat = ceil(t / dt) - 1, and u = 0 for t <= 0.
//
// B200 design (not the reference's grid of one block per (triangle, instant)
// per point and a shared-memory tree reduction): the instants t_q - k dt of
// all requested (time, k) are formed on the host exactly as the reference
// forms them (k dt rounded, then subtracted), deduplicated by value, and M is
// evaluated once per (point, distinct instant, triangle) by one thread (the
// lanes of a warp take consecutive triangles; the rule's nodes sit in shared
// memory); a second kernel contracts, one block per (time, point).
#include "ebem_internal.h"

#include <algorithm>

namespace ebem {

namespace {

// Lamé kernel integrated twice in time at (x = y - source, r = |x|, t):
// symmetric 3x3 as (11, 12, 13, 22, 23, 33), the terms of kernelGHC.cu:204-259.
__device__ __forceinline__ void lame_kernel(double out[6], const double x[3], double r, double t, double cP, double cS) {
    const double hP = (t - (r / cP) > 0) ? 1.0 : 0.0;
    const double hS = (t - (r / cS) > 0) ? 1.0 : 0.0;
    const double ir = 1.0 / r, ir3 = ir * ir * ir, ir5 = ir3 * ir * ir;
    const double qP = (cP * cP * t * t - r * r) / (cP * cP), qS = (cS * cS * t * t - r * r) / (cS * cS);
    const double w = qP * hP - qS * hS;
    const double aP = hP / (cP * cP), aS = hS / (cS * cS);
    const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int e = 0; e < 6; e++) {
        const double xx = x[ia[e]] * x[ib[e]];
        const double d = (ia[e] == ib[e]) ? 1.0 : 0.0;
        out[e] = xx * ir3 * aP + (d * ir - xx * ir3) * aS - 0.5 * (d * ir3 - 3.0 * xx * ir5) * w;
    }
}

}  // namespace

// M for one (point, distinct instant, triangle) per thread; triangle fastest.
// At most 80 registers (6 blocks of 128 threads per SM; 116 without the
// cap): 64 points at one time on the 320-triangle sphere 0.39 -> 0.36 ms.
__global__ void __launch_bounds__(128, 6) pp_num_level_kernel(const double* __restrict__ coords,
                                                           const int32_t* __restrict__ tris,
                                                           const TriGeom* __restrict__ geo, int N,
                                                           const double* __restrict__ pts, int p0, int np, int nu,
                                                           const double* __restrict__ taus,
                                                           const double* __restrict__ nodes,   // n_sub * n_sing x 3
                                                           const double* __restrict__ w,       // n_sing
                                                           int n_sub, int n_sing, int stride, int layer, double velP,
                                                           double velS, double c4, double* __restrict__ Mbuf) {
    extern __shared__ double sh[];            // nodes (3 per node), then the n_sing weights
    const int nn = n_sub * n_sing;
    for (int q = threadIdx.x; q < 3 * nn + n_sing; q += blockDim.x) sh[q] = (q < 3 * nn) ? nodes[q] : w[q - 3 * nn];
    __syncthreads();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * np * nu) return;
    const int m = (int)(idx % N);
    const long long rr = idx / N;
    const int ui = (int)(rr % nu), pl = (int)(rr / nu);
    const int p = p0 + pl;
    const double x[3] = {pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]};
    const double tau = taus[ui];
    const TriGeom& G = geo[m];
    double S[6] = {0, 0, 0, 0, 0, 0};
    const double d0 = x[0] - G.ctr[0], d1 = x[1] - G.ctr[1], d2 = x[2] - G.ctr[2];
    const double distMin = sqrt(d0 * d0 + d1 * d1 + d2 * d2) - G.maxL;
    if (!(tau * velP < distMin)) {                 // the null test of kernelSP.cu:111-121 / kernelLayer.cu:159-170
        double V[3][3];
#pragma unroll
        for (int v = 0; v < 3; v++) {
            const int id = tris[3 * m + v];
#pragma unroll
            for (int c = 0; c < 3; c++) V[v][c] = coords[3 * id + c];
        }
        const double area = G.area;
        const double* wsh = sh + 3 * nn;
        for (int sub = 0; sub < n_sub; sub++) {
            for (int l = 0; l < n_sing; l++) {
                const double* b = sh + 3 * (sub * stride + l);
                double y[3];
#pragma unroll
                for (int c = 0; c < 3; c++) y[c] = b[0] * V[0][c] + b[1] * V[1][c] + b[2] * V[2][c] - x[c];
                const double r = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
                double K[6];
                lame_kernel(K, y, r, tau, velP, velS);
                const double wt = wsh[l] * area;
#pragma unroll
                for (int e = 0; e < 6; e++) S[e] += wt * K[e];
            }
        }
    }
    double* dst = Mbuf + (((size_t)pl * nu + ui) * N + m) * 6;
#pragma unroll
    for (int e = 0; e < 6; e++) {
        double v;
        if (layer) {
            v = S[e] / c4;
            if (fabs(v) < 1.0e-14) v = 0.0;
        } else {
            v = (fabs(S[e]) > 1.0e-14) ? S[e] / c4 : 0.0;
        }
        dst[e] = v;
    }
}

__device__ __forceinline__ void sym_apply(double acc[3], const double* M, const double d[3]) {
    acc[0] += M[0] * d[0] + M[1] * d[1] + M[2] * d[2];
    acc[1] += M[1] * d[0] + M[3] * d[1] + M[4] * d[2];
    acc[2] += M[2] * d[0] + M[4] * d[1] + M[5] * d[2];
}

// One block per (time q, point pl): the time sum of the variant.  Blocks of
// 128 threads, or of 1024 when there are too few (time, point) pairs to
// fill the GPU (one point at its 40 times: 40 blocks).
__global__ void __launch_bounds__(1024) pp_num_sum_kernel(const double* __restrict__ Mbuf, int N, int p0, int np,
                                                         int nu, const int* __restrict__ tab, int kmax,
                                                         const int* __restrict__ nhat, int npts,
                                                         const double* __restrict__ phi, int layer,
                                                         double* __restrict__ u) {
    const int q = blockIdx.x / np, pl = blockIdx.x - q * np;
    const int nh = nhat[q];
    const int* tq = tab + (size_t)q * kmax;
    const size_t n3 = 3 * (size_t)N;
    double acc[3] = {0, 0, 0};
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        for (int k = 0; k <= nh; k++) {
            const double* Mk = Mbuf + (((size_t)pl * nu + tq[k]) * N + m) * 6;
            const double* pk = phi + (size_t)k * n3 + 3 * (size_t)m;
            if (layer) {
                double d[3] = {pk[0], pk[1], pk[2]};
                if (k > 0) {
                    const double* pm = pk - n3;
                    d[0] -= pm[0]; d[1] -= pm[1]; d[2] -= pm[2];
                }
                sym_apply(acc, Mk, d);
            } else {
                double D[6];
                if (k < nh) {
                    const double* Mn = Mbuf + (((size_t)pl * nu + tq[k + 1]) * N + m) * 6;
#pragma unroll
                    for (int e = 0; e < 6; e++) D[e] = Mk[e] - Mn[e];
                } else {
#pragma unroll
                    for (int e = 0; e < 6; e++) D[e] = Mk[e];
                }
                const double d[3] = {pk[0], pk[1], pk[2]};
                sym_apply(acc, D, d);
            }
        }
    }
    __shared__ double red[3][32];
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[c][wi] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) v += red[threadIdx.x][i];
        u[((size_t)q * npts + p0 + pl) * 3 + threadIdx.x] = v;
    }
}

int launch_pp_num(const MeshData& m, const PhysParams& P, int n_sub, int n_sing, int layer, int fix,
                  const double* d_phi, const double* d_pts, int npts, const double* h_times, int ntimes, double* d_u,
                  cudaStream_t s) {
    // kernelSP reads node 3 * subregion + l (kernelSP.cu:41); with fewer than 3
    // nodes per sub-triangle that read passes the end of the node table
    const int stride = (layer || fix) ? n_sing : 3;
    if ((n_sub - 1) * stride + n_sing > n_sub * n_sing)
        return fail(EBEM_ERR_INVALID, "the reference's point post-processing reads node 3 * subregion + l "
                                      "(kernelSP.cu:41), past the node table for this rule; pass "
                                      "EBEM_FIX_REFERENCE_DEFECTS to read node subregion * n_sing + l");
    // instants t_q - k dt, formed as the reference forms them, deduplicated
    std::vector<int> nh(ntimes);
    int kmax = 1;
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
        for (int k = 0; k <= n; k++) {
            volatile double a = (double)k * P.dt;      // rounded product, then the difference
            taus.push_back(t - a);
        }
    }
    std::vector<double> uniq(taus);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    const int nu = std::max(1, (int)uniq.size());
    if (uniq.empty()) uniq.push_back(0.0);
    std::vector<int> tab((size_t)ntimes * kmax, 0);
    {
        size_t c = 0;
        for (int q = 0; q < ntimes; q++)
            for (int k = 0; k <= nh[q]; k++)
                tab[(size_t)q * kmax + k] = (int)(std::lower_bound(uniq.begin(), uniq.end(), taus[c++]) - uniq.begin());
    }
    std::vector<double> nodes((size_t)3 * n_sub * n_sing), w(n_sing);
    if (gh_composite(n_sing, n_sub, nodes.data(), w.data()))
        return fail(EBEM_ERR_INVALID, "inner rule: n_sub in {1,4,16,64}, n_sing in {1,3,7,12,19}");
    const size_t per_point = (size_t)nu * m.nt * 6 * sizeof(double);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)npts, ((size_t)1 << 30) / per_point));
    // the tables in one upload: instants, rule nodes and weights, index table, nHat
    HostPack pk;
    const size_t o_taus = pk.add(uniq.data(), nu * sizeof(double));
    std::vector<double> rule(nodes);                        // the nodes, then the weights
    rule.insert(rule.end(), w.begin(), w.end());
    const size_t o_nodes = pk.add(rule.data(), rule.size() * sizeof(double));
    const size_t o_tab = pk.add(tab.data(), tab.size() * sizeof(int));
    const size_t o_nh = pk.add(nh.data(), ntimes * sizeof(int));
    unsigned char* d_pack = nullptr;
    double* Mbuf = nullptr;
    cudaError_t e = pk.upload(&d_pack, s);
    if (e != cudaSuccess || ws_malloc(&Mbuf, per_point * chunk, s) != cudaSuccess) {
        cudaGetLastError();
        ws_free(d_pack, s);
        return fail(EBEM_ERR_NOMEM, "post-processing workspace allocation failed");
    }
    const double* d_taus = reinterpret_cast<const double*>(d_pack + o_taus);
    const double* d_rule = reinterpret_cast<const double*>(d_pack + o_nodes);
    const int* d_tab = reinterpret_cast<const int*>(d_pack + o_tab);
    const int* d_nh = reinterpret_cast<const int*>(d_pack + o_nh);
    const size_t shmem = (nodes.size() + w.size()) * sizeof(double);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device);
    for (int p0 = 0; p0 < npts && e == cudaSuccess; p0 += chunk) {
        const int np = std::min(chunk, npts - p0);
        const long long lv = (long long)m.nt * np * nu;
        pp_num_level_kernel<<<(unsigned)((lv + 127) / 128), 128, shmem, s>>>(
            m.d_coords, m.d_tris, m.d_geo, m.nt, d_pts, p0, np, nu, d_taus, d_rule, d_rule + nodes.size(), n_sub,
            n_sing, stride, layer, P.velP, P.velS, 4 * kPi * P.rho, Mbuf);
        const int sum_threads = ((long long)ntimes * np < 2LL * sms) ? 1024 : 128;
        pp_num_sum_kernel<<<(unsigned)((long long)ntimes * np), sum_threads, 0, s>>>(Mbuf, m.nt, p0, np, nu, d_tab, kmax,
                                                                             d_nh, npts, d_phi, layer, d_u);
        e = cudaGetLastError();
    }
    ws_free(Mbuf, s);
    ws_free(d_pack, s);
    if (e != cudaSuccess)
        return fail(EBEM_ERR_CUDA, std::string("numerical post-processing kernels: ") + cudaGetErrorString(e));
    return EBEM_OK;
}

}  // namespace ebem
