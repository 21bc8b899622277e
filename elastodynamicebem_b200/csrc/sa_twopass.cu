// Semi-analytic assembly of dense outputs in two passes.
//
// Pass 1 (sa_level_kernel in its level-output mode, sa_assemble.cu):
// one warp per (source, field) pair walks the pair's time levels and stores
// F(t_k), the combined kernel integral at instant k dt
// (BEMenerg_coreSA_calcMatrixSubBlock.m:101-104 summed over the outer nodes
// and rotated to global axes; 6 symmetric entries), for every level its
// non-null lags need, and the pair's non-null lags (llo, lhi) of the null
// test of BEMenerg_coreSA_calcMatrixBlock.m:57-61.
//
// Pass 2 (sa_emit_kernel): every entry of the window's blocks,
//   E_l = (F_{l+1} - 2 F_l + F_{l-1}) / (4 pi rho), clean-up |x| < 1e-14 -> 0
// (calcMatrixSubBlock.m:15,23,111; calcMatrixBlock.m:77), zero outside the
// pair's non-null lags, written (or added) one thread per block with
// consecutive threads on consecutive sources: the output is written in whole
// sectors, zeros included.  In one pass, the warp kernel wrote each
// block as 24-byte column pieces scattered 3N doubles apart and filled the
// zeros of the lags outside each pair's band the same way (sphere of 1280
// triangles, L = 40: 207 ms per step; two passes: 188 ms).
//
// The values equal those of the level kernel's direct output bit for bit
// (the same per-pair arithmetic and the same second-difference expression).
//
// The level buffer holds, per chunk of field columns, (columns) x (levels) x
// (sources) x 6 doubles plus one int2 per pair; the columns are split into
// equal chunks that keep it within what the workspace pool keeps reserved
// between calls.
#include "ebem_internal.h"

#include <algorithm>
#include <atomic>
#include <mutex>

namespace ebem {

namespace {
// Per-pass device times of the two-pass assembly (ebem_profile_*): CUDA
// events around each launch on the call's stream, read at the end of the call.
std::atomic<int> g_profile{0};
std::mutex g_prof_mu;
double g_prof_ms[2] = {0.0, 0.0};        // pass 1 (levels), pass 2 (emission)
long long g_prof_n[2] = {0, 0};
}  // namespace

void profile_enable(int on) { g_profile.store(on ? 1 : 0); }

void profile_read(double ms[2], long long n[2], int reset) {
    std::lock_guard<std::mutex> lock(g_prof_mu);
    for (int k = 0; k < 2; k++) {
        ms[k] = g_prof_ms[k];
        n[k] = g_prof_n[k];
        if (reset) { g_prof_ms[k] = 0.0; g_prof_n[k] = 0; }
    }
}

// E_l of the window from the levels of one chunk of field columns: one
// thread per (source, field, lag) block, consecutive threads on consecutive
// sources of one field column, so each of the 9 stores of a warp covers one
// contiguous 768-byte run of a column (the three row stores of a column fill
// it completely); the levels are read as 16-byte pairs.
__global__ void __launch_bounds__(128) sa_emit_kernel(const double* __restrict__ Fb, const int2* __restrict__ band,
                                                      int nsrc, int j0, int KL, int kbase, int lag0, int nlag, double c4,
                                                      double* __restrict__ E, size_t ld, size_t ld_lag,
                                                      int accumulate, const unsigned char* __restrict__ cls,
                                                      int cls_want) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= nsrc) return;
    const int jj = blockIdx.y, q = blockIdx.z, l = lag0 + q;
    const int2 b = band[(long long)jj * nsrc + ii];
    const bool inband = b.x >= 0 && l >= b.x && l <= b.y;
    if (cls) {
        // one class of a per-(pair, lag) class array (sources = all triangles)
        if (inband ? cls[((long long)(j0 + jj) * nsrc + ii) * nlag + q] != cls_want : cls_want != 0) return;
    }
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (inband) {
        const long long rec = (long long)jj * KL * nsrc + ii;          // record of level kbase
        const long long ks = nsrc;                                       // records per level
        double f1[6], f0[6] = {0, 0, 0, 0, 0, 0}, fm[6] = {0, 0, 0, 0, 0, 0};
        const double2* p1 = reinterpret_cast<const double2*>(Fb + (rec + (l + 1 - kbase) * ks) * 6);
#pragma unroll
        for (int h = 0; h < 3; h++) { const double2 t = p1[h]; f1[2 * h] = t.x; f1[2 * h + 1] = t.y; }
        if (l >= 1) {                                                      // F_0 = 0
            const double2* p0 = reinterpret_cast<const double2*>(Fb + (rec + (l - kbase) * ks) * 6);
#pragma unroll
            for (int h = 0; h < 3; h++) { const double2 t = p0[h]; f0[2 * h] = t.x; f0[2 * h + 1] = t.y; }
        }
        if (l - 1 >= 1) {
            const double2* pm = reinterpret_cast<const double2*>(Fb + (rec + (l - 1 - kbase) * ks) * 6);
#pragma unroll
            for (int h = 0; h < 3; h++) { const double2 t = pm[h]; fm[2 * h] = t.x; fm[2 * h + 1] = t.y; }
        }
#pragma unroll
        for (int e = 0; e < 6; e++) {
            const double x = ((f1[e] + (-2.0) * f0[e]) + fm[e]) / c4;
            v[e] = (fabs(x) < 1.0e-14) ? 0.0 : x;
        }
    }
    // (r, c) -> symmetric entry 11, 12, 13, 22, 23, 33
    const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    double* base = E + (size_t)q * ld_lag + 3 * (size_t)(j0 + jj) * ld + 3 * (size_t)ii;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            double* dst = base + (size_t)c * ld + r;
            const double x = v[sym[3 * c + r]];
            if (accumulate) *dst += x;
            else *dst = x;
        }
}

int launch_sa_twopass(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                      double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count, int mixed,
                      cudaStream_t s, const unsigned char* cls, int cls_want) {
    if (cls && (src0 != 0 || nsrc != m.nt)) return fail(EBEM_ERR_INVALID, "a class array needs all source rows");
    if (m.nt > 65535 || nlag > 65535) return fail(EBEM_ERR_INVALID, "mesh or lag window too large for one launch");
    const int kbase = std::max(1, lag0 - 1);
    const int KL = lag0 + nlag + 1 - kbase;           // levels kbase .. lag0 + nlag
    const size_t fbytes = (size_t)KL * nsrc * 6 * sizeof(double);
    const size_t per_col = fbytes + (size_t)nsrc * sizeof(int2);
    // within what the workspace pool keeps reserved between calls, so that a
    // repeated call maps no new memory; equal chunks of field columns
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t budget = std::max<size_t>((size_t)64 << 20, std::min<size_t>(free_b / 4, (size_t)3 << 29));
    const int most = (int)std::max<size_t>(1, std::min<size_t>((size_t)m.nt, budget / per_col));
    const int chunks = (m.nt + most - 1) / most;
    const int cols = (m.nt + chunks - 1) / chunks;
    double* Fb = nullptr;
    if (ws_malloc(&Fb, per_col * cols, s) != cudaSuccess)
        return fail(EBEM_ERR_NOMEM, "assembly workspace allocation failed");
    int2* band = reinterpret_cast<int2*>(reinterpret_cast<unsigned char*>(Fb) + fbytes * cols);
    const bool prof = g_profile.load() != 0;
    std::vector<cudaEvent_t> ev;
    auto mark = [&]() {
        if (!prof) return;
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) == cudaSuccess && cudaEventRecord(e, s) == cudaSuccess) ev.push_back(e);
        else if (e) cudaEventDestroy(e);
    };
    int rc = EBEM_OK;
    mark();
    for (int j0 = 0; j0 < m.nt && rc == EBEM_OK; j0 += cols) {
        const int nj = std::min(cols, m.nt - j0);
        rc = launch_sa_fwarp(m, P, n_gh, lag0, nlag, src0, nsrc, j0, nj, kbase, KL, Fb, band, d_count, mixed, s, cls,
                             cls_want);
        if (rc) break;
        mark();
        dim3 grid((unsigned)((nsrc + 127) / 128), (unsigned)nj, (unsigned)nlag);
        sa_emit_kernel<<<grid, 128, 0, s>>>(Fb, band, nsrc, j0, KL, kbase, lag0, nlag, 4 * kPi * P.rho, d_E, ld,
                                            ld_lag, accumulate, cls, cls_want);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, std::string("emission kernel: ") + cudaGetErrorString(e));
        mark();
    }
    ws_free(Fb, s);
    if (prof) {
        // events alternate: start, after pass 1, after pass 2, after pass 1, ...
        double add[2] = {0.0, 0.0};
        long long cnt[2] = {0, 0};
        if (rc == EBEM_OK && !ev.empty() && cudaEventSynchronize(ev.back()) == cudaSuccess) {
            for (size_t k = 1; k < ev.size(); k++) {
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, ev[k - 1], ev[k]) == cudaSuccess) {
                    add[(k - 1) & 1] += ms;
                    cnt[(k - 1) & 1]++;
                }
            }
        }
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        cudaGetLastError();
        std::lock_guard<std::mutex> lock(g_prof_mu);
        for (int k = 0; k < 2; k++) {
            g_prof_ms[k] += add[k];
            g_prof_n[k] += cnt[k];
        }
    }
    return rc;
}

}  // namespace ebem
