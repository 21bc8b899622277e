// ORACLE — test infrastructure only.  Host launchers for the reference's own
// direct-formulation CUDA kernels, compiled from the reference's source files
// in place (the build recipe passes the path of exactly one of them as
// REF_KERNEL_K, REF_KERNEL_G or REF_KERNEL_P; no reference source is copied
// here).  Argument lists and launch shapes follow
//   kernelK: functions/BEMenerg_dir/BEMenerg_dir_timeMarchingN.m:186-206 and
//            BEMenerg_dir_launchKernelK.m:1-20 (grid (N, Nv, lags), block (nSub, nSing))
//   kernelG: functions/BEMenerg_dirPP/BEMenerg_ppN_calc.m:80-93 (grid (N, nHat), block nSub)
//   kernelP: functions/BEMenerg_dirPP/BEMenerg_ppN_calc.m:96-109 (grid (Nv, nHat), block nSub)
#include <cuda_runtime.h>
#include <vector>

static float g_last_ms = -1.0f;   // device time of the last reference kernel launch (CUDA events)

extern "C" float ref_last_kernel_ms() { return g_last_ms; }

// CUDA events around one launch; the elapsed time lands in g_last_ms.
struct KernelTimer {
    cudaEvent_t e0, e1;
    KernelTimer() {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
    }
    void stop() {
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&g_last_ms, e0, e1);
    }
    ~KernelTimer() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
};

#if defined(REF_KERNEL_K)
#include REF_KERNEL_K
#elif defined(REF_KERNEL_G)
#include REF_KERNEL_G
#elif defined(REF_KERNEL_P)
#include REF_KERNEL_P
#endif

namespace {
struct Dev {
    std::vector<void*> ptrs;
    bool ok = true;
    double* put(const double* h, size_t n) {
        void* d = nullptr;
        if (cudaMalloc(&d, (n ? n : 1) * sizeof(double)) != cudaSuccess) { ok = false; return nullptr; }
        ptrs.push_back(d);
        if (n) cudaMemcpy(d, h, n * sizeof(double), cudaMemcpyHostToDevice);
        return (double*)d;
    }
    int* puti(const int* h, size_t n) {
        void* d = nullptr;
        if (cudaMalloc(&d, (n ? n : 1) * sizeof(int)) != cudaSuccess) { ok = false; return nullptr; }
        ptrs.push_back(d);
        if (n) cudaMemcpy(d, h, n * sizeof(int), cudaMemcpyHostToDevice);
        return (int*)d;
    }
    ~Dev() { for (void* p : ptrs) cudaFree(p); }
};
void split3(const double* n3, int n, std::vector<double>& x, std::vector<double>& y, std::vector<double>& z) {
    x.resize(n); y.resize(n); z.resize(n);
    for (int k = 0; k < n; k++) { x[k] = n3[3 * k]; y[k] = n3[3 * k + 1]; z[k] = n3[3 * k + 2]; }
}
}  // namespace

#if defined(REF_KERNEL_K)
// matrix: 9 N Nv nlag doubles, column-major (3N) x (3Nv) per lag; indSM: Nv*N
// (index s*N + m, 1..3 or 0); matCoeff: 9N (9m + 3j + i = M(i,j)); vetCoeff 3N.
extern "C" int ref_k(double* matrix, int N, int Nv, int nlag, double deltaT, double velP, double velS, double lambda,
                     double mu, double rho, const double* GHw, const double* GHn, int nGH, const double* GHCw,
                     const double* GHCn, int nSub, int nSing, const double* vertsT, const double* areeT,
                     const double* normT, const int* indSM, const double* matCoeff, const double* vetCoeff,
                     int offsetZ, int numBlocks, const double* nodesMesh, double maxLen) {
    const size_t nm = (size_t)9 * N * Nv * nlag;
    const int nInt = nSub * nSing;
    std::vector<double> gx, gy, gz, cx, cy, cz;
    split3(GHn, nGH, gx, gy, gz);
    split3(GHCn, nInt, cx, cy, cz);
    Dev D;
    double* d_m = D.put(matrix, nm);
    double *w = D.put(GHw, nGH), *x = D.put(gx.data(), nGH), *y = D.put(gy.data(), nGH), *z = D.put(gz.data(), nGH);
    double *cw = D.put(GHCw, nSing), *ccx = D.put(cx.data(), nInt), *ccy = D.put(cy.data(), nInt),
           *ccz = D.put(cz.data(), nInt);
    double *v = D.put(vertsT, 9 * (size_t)N), *a = D.put(areeT, N), *nr = D.put(normT, 3 * (size_t)N);
    int* ism = D.puti(indSM, (size_t)N * Nv);
    double *mc = D.put(matCoeff, 9 * (size_t)N), *vc = D.put(vetCoeff, 3 * (size_t)N),
           *nm3 = D.put(nodesMesh, 3 * (size_t)Nv);
    if (!D.ok) return -3;
    dim3 grid(N, Nv, nlag), block(nSub, nSing);
    KernelTimer timer;
    kernelK<<<grid, block, nSub * nSing * 9 * sizeof(double)>>>(d_m, deltaT, velP, velS, lambda, mu, rho,
                                                                4 * 3.141592653589793 * deltaT, w, x, y, z, nGH, cw,
                                                                ccx, ccy, ccz, v, a, nr, ism, mc, vc, offsetZ,
                                                                numBlocks, nm3, maxLen);
    timer.stop();
    cudaError_t e = cudaGetLastError();               // a launch the block shape does not allow fails here
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(matrix, d_m, nm * sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : -2;
}
#endif

#if defined(REF_KERNEL_G)
// matrix: (3 nHat) x (3N) column-major.  The kernel reads node 3 tid + l, so
// the launcher refuses n_sing < 3 with n_sub > 1 (the read would leave the
// node table).
extern "C" int ref_g(double* matrix, int N, int nHat, double velP, double velS, double rho, const double* x3,
                     const double* diffTemp /* nHat + 2 */, const double* PPw, const double* PPn, int nSub, int nSing,
                     const double* vertsT, const double* areeT, const double* centerT, const double* maxLenT) {
    if (3 * (nSub - 1) + nSing > nSub * nSing) return -1;
    const int nInt = nSub * nSing;
    std::vector<double> px, py, pz;
    split3(PPn, nInt, px, py, pz);
    Dev D;
    const size_t nm = (size_t)9 * nHat * N;
    double* d_m = D.put(matrix, nm);
    double *sp = D.put(x3, 3), *dtm = D.put(diffTemp, nHat + 2);
    double *w = D.put(PPw, nSing), *x = D.put(px.data(), nInt), *y = D.put(py.data(), nInt), *z = D.put(pz.data(), nInt);
    double *v = D.put(vertsT, 9 * (size_t)N), *a = D.put(areeT, N), *c = D.put(centerT, 3 * (size_t)N),
           *ml = D.put(maxLenT, N);
    if (!D.ok) return -3;
    dim3 grid(N, nHat, 1), block(nSub, 1, 1);
    KernelTimer timer;
    kernelPPNEWG<<<grid, block, nSub * 9 * sizeof(double)>>>(d_m, velP, velS, 4 * 3.141592653589793 * rho, sp, dtm, w,
                                                             x, y, z, nSing, v, a, c, ml);
    timer.stop();
    cudaError_t e = cudaGetLastError();               // a launch the block shape does not allow fails here
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(matrix, d_m, nm * sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : -2;
}
#endif

#if defined(REF_KERNEL_P)
// matrix: (3 nHat) x (3 Nv) column-major; indSM index s*N + m.
extern "C" int ref_p(double* matrix, int N, int Nv, int nHat, double velP, double velS, double lambda, double mu,
                     double rho, double deltaT, const double* x3, const double* diffTemp, const double* PPw,
                     const double* PPn, int nSub, int nSing, const double* vertsT, const double* areeT,
                     const double* normT, const int* indSM, const double* matCoeff, const double* vetCoeff) {
    const int nInt = nSub * nSing;
    std::vector<double> px, py, pz;
    split3(PPn, nInt, px, py, pz);
    Dev D;
    const size_t nm = (size_t)9 * nHat * Nv;
    double* d_m = D.put(matrix, nm);
    double *sp = D.put(x3, 3), *dtm = D.put(diffTemp, nHat + 2);
    double *w = D.put(PPw, nSing), *x = D.put(px.data(), nInt), *y = D.put(py.data(), nInt), *z = D.put(pz.data(), nInt);
    double *v = D.put(vertsT, 9 * (size_t)N), *a = D.put(areeT, N), *nr = D.put(normT, 3 * (size_t)N);
    int* ism = D.puti(indSM, (size_t)N * Nv);
    double *mc = D.put(matCoeff, 9 * (size_t)N), *vc = D.put(vetCoeff, 3 * (size_t)N);
    if (!D.ok) return -3;
    dim3 grid(Nv, nHat, 1), block(nSub, 1, 1);
    KernelTimer timer;
    kernelPPNEWP<<<grid, block, nSub * 9 * sizeof(double)>>>(d_m, velP, velS, lambda, mu,
                                                             4 * 3.141592653589793 * rho * deltaT, (double)N, sp, dtm,
                                                             w, x, y, z, nSing, v, a, nr, ism, mc, vc);
    timer.stop();
    cudaError_t e = cudaGetLastError();               // a launch the block shape does not allow fails here
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(matrix, d_m, nm * sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : -2;
}
#endif
