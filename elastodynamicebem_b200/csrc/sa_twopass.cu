// Semi-analytic assembly of dense outputs in two passes.
//
// Pass 1 (sa_assemble_warp_kernel in its level-output mode, sa_assemble.cu):
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
// pair's non-null lags, written (or added) one thread per entry with
// consecutive threads on consecutive rows of a column: the output is written
// in whole sectors, zeros included.  In one pass, the warp kernel wrote each
// block as 24-byte column pieces scattered 3N doubles apart and filled the
// zeros of the lags outside each pair's band the same way (sphere of 1280
// triangles, L = 40: 207 ms per step; two passes: 188 ms).
//
// The values equal the one-pass kernel's bit for bit (the same per-pair
// arithmetic and the same second-difference expression).
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

// E_l of the window from the levels of one chunk of field columns.
__global__ void __launch_bounds__(256) sa_emit_kernel(const double* __restrict__ Fb, const int2* __restrict__ band,
                                                      int nsrc, int j0, int KL, int kbase, int lag0, double c4,
                                                      double* __restrict__ E, size_t ld, size_t ld_lag,
                                                      int accumulate) {
    const long long rows = 3LL * nsrc;
    const long long r3 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r3 >= rows) return;
    const int col = blockIdx.y;                   // 3 jj + c
    const int jj = col / 3, c = col - 3 * jj;
    const int q = blockIdx.z, l = lag0 + q;
    const int ii = (int)(r3 / 3), r = (int)(r3 - 3LL * ii);
    const int2 b = band[(long long)jj * nsrc + ii];
    double v = 0.0;
    if (b.x >= 0 && l >= b.x && l <= b.y) {
        const int e = (r == 0) ? c : (c == 0 ? r : r + c + 1);        // (r, c) -> 11, 12, 13, 22, 23, 33
        const double* f = Fb + ((long long)jj * KL * nsrc + ii) * 6 + e;
        const long long ks = (long long)nsrc * 6;                       // one level
        const double fk1 = f[(l + 1 - kbase) * ks];
        const double fk = (l >= 1) ? f[(l - kbase) * ks] : 0.0;            // F_0 = 0
        const double fkm = (l - 1 >= 1) ? f[(l - 1 - kbase) * ks] : 0.0;
        v = ((fk1 + (-2.0) * fk) + fkm) / c4;
        if (fabs(v) < 1.0e-14) v = 0.0;
    }
    double* dst = E + (size_t)q * ld_lag + (3 * (size_t)(j0 + jj) + c) * ld + (size_t)r3;
    if (accumulate) *dst += v;
    else *dst = v;
}

int launch_sa_twopass(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                      double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count, int mixed,
                      cudaStream_t s) {
    if (3LL * m.nt > 65535 || nlag > 65535) return fail(EBEM_ERR_INVALID, "mesh or lag window too large for one launch");
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
        rc = launch_sa_fwarp(m, P, n_gh, lag0, nlag, src0, nsrc, j0, nj, kbase, KL, Fb, band, d_count, mixed, s);
        if (rc) break;
        mark();
        const long long rows = 3LL * nsrc;
        dim3 grid((unsigned)((rows + 255) / 256), (unsigned)(3 * nj), (unsigned)nlag);
        sa_emit_kernel<<<grid, 256, 0, s>>>(Fb, band, nsrc, j0, KL, kbase, lag0, 4 * kPi * P.rho, d_E, ld, ld_lag,
                                            accumulate);
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
