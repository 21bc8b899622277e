// ORACLE — test infrastructure only.  Host launchers for the reference's own
// numerical post-processing kernels, compiled from the reference's source
// files in place (the build recipe passes the path; no reference source is
// copied here), one library per kernel because both are named kernelPP:
//   REF_KERNEL_SP     functions/BEMenerg_indir/BEMenerg_postProc/BEMenerg_postProcGPU/
//                     CUDAkernels/kernelSP.cu, launched as
//                     BEMenerg_postProcGPU_calcSP.m:29-75 does: grid (N, numIst),
//                     block (numSubRegionPP), one matrix [3 numIst x 3N] per (x, t)
//   REF_KERNEL_LAYER  .../CUDAkernels/kernelLayer.cu, launched as
//                     BEMenerg_postProcGPU_calcLayer.m:27-72 does: grid (#points),
//                     block (numIst), u [3 x #points] for one t
// Kernel time of the last launch by CUDA events.
#if defined(REF_KERNEL_SP)
#include REF_KERNEL_SP
#elif defined(REF_KERNEL_LAYER)
#include REF_KERNEL_LAYER
#endif

#include <cuda_runtime.h>
#include <vector>

static float g_last_ms = -1.0f;

extern "C" float ref_last_kernel_ms() { return g_last_ms; }

namespace {
struct Dev {
    std::vector<void*> bufs;
    double* put(const double* h, size_t n) {
        void* d = nullptr;
        if (cudaMalloc(&d, n * sizeof(double) > 0 ? n * sizeof(double) : 8) != cudaSuccess) return nullptr;
        bufs.push_back(d);
        if (h) cudaMemcpy(d, h, n * sizeof(double), cudaMemcpyHostToDevice);
        else cudaMemset(d, 0, n * sizeof(double));
        return (double*)d;
    }
    ~Dev() { for (void* p : bufs) cudaFree(p); }
};
}  // namespace

// Common inputs: PPw (nSing), PPn (nSub*nSing x 3, row-major), vertsT (9N,
// vertsT[9t + 3*coord + vertex]), areeT (N), centerT (3N), maxLenT (N).
#if defined(REF_KERNEL_SP)
extern "C" int ref_sp(double* matrix_host /* 9 numIst N, column-major [3 numIst x 3N] */, int N, int numIst,
                      double velP, double velS, double const4PiRho, const double* x /* 3 */,
                      const double* diffTemp /* numIst */, const double* PPw, const double* PPn, int nSub, int nSing,
                      const double* vertsT, const double* areeT, const double* centerT, const double* maxLenT) {
    const int nn = nSub * nSing;
    // kernelSP reads node 3 * threadIdx.x + l (kernelSP.cu:41): refuse rules
    // where that read would pass the end of the node table
    if (3 * (nSub - 1) + nSing > nn || nSub > 1024) return -4;
    std::vector<double> nx(nn), ny(nn), nz(nn);
    for (int k = 0; k < nn; k++) { nx[k] = PPn[3 * k]; ny[k] = PPn[3 * k + 1]; nz[k] = PPn[3 * k + 2]; }
    Dev d;
    const size_t nm = (size_t)9 * numIst * N;
    double *dm = d.put(nullptr, nm), *dx = d.put(x, 3), *dt = d.put(diffTemp, numIst), *dw = d.put(PPw, nSing),
           *dnx = d.put(nx.data(), nn), *dny = d.put(ny.data(), nn), *dnz = d.put(nz.data(), nn),
           *dv = d.put(vertsT, 9 * (size_t)N), *da = d.put(areeT, N), *dc = d.put(centerT, 3 * (size_t)N),
           *dl = d.put(maxLenT, N);
    if (!dm || !dx || !dt || !dw || !dnx || !dny || !dnz || !dv || !da || !dc || !dl) return -3;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    kernelPP<<<dim3(N, numIst), dim3(nSub), nSub * 9 * sizeof(double)>>>(dm, velP, velS, const4PiRho, dx, dt, dw, dnx,
                                                                          dny, dnz, nSing, dv, da, dc, dl);
    cudaEventRecord(e1);
    cudaError_t e = cudaGetLastError();               // a launch the block shape does not allow fails here
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaEventElapsedTime(&g_last_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e == cudaSuccess) e = cudaMemcpy(matrix_host, dm, nm * sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : -2;
}
#endif

#if defined(REF_KERNEL_LAYER)
extern "C" int ref_layer(double* u_host /* 3 npts */, int N, int npts, int numIst, double velP, double velS,
                         double const4PiRho, const double* pts /* 3 npts */, const double* diffTemp /* numIst */,
                         const double* PPw, const double* PPn, int nSub, int nSing, const double* vertsT,
                         const double* areeT, const double* centerT, const double* maxLenT,
                         const double* densityLin /* 3N numIst, [(3m + c) numIst + k] */) {
    const int nn = nSub * nSing;
    if (numIst < 1 || numIst > 1024) return -4;           // one thread per history instant
    std::vector<double> nx(nn), ny(nn), nz(nn);
    for (int k = 0; k < nn; k++) { nx[k] = PPn[3 * k]; ny[k] = PPn[3 * k + 1]; nz[k] = PPn[3 * k + 2]; }
    Dev d;
    double *du = d.put(nullptr, 3 * (size_t)npts), *dp = d.put(pts, 3 * (size_t)npts), *dt = d.put(diffTemp, numIst),
           *dw = d.put(PPw, nSing), *dnx = d.put(nx.data(), nn), *dny = d.put(ny.data(), nn),
           *dnz = d.put(nz.data(), nn), *dv = d.put(vertsT, 9 * (size_t)N), *da = d.put(areeT, N),
           *dc = d.put(centerT, 3 * (size_t)N), *dl = d.put(maxLenT, N),
           *dd = d.put(densityLin, 3 * (size_t)N * numIst);
    if (!du || !dp || !dt || !dw || !dnx || !dny || !dnz || !dv || !da || !dc || !dl || !dd) return -3;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    kernelPP<<<dim3(npts), dim3(numIst), numIst * 3 * sizeof(double)>>>(du, velP, velS, const4PiRho, dp, dt, N, nSub,
                                                                        nSing, dw, dnx, dny, dnz, dv, da, dc, dl, dd);
    cudaEventRecord(e1);
    cudaError_t e = cudaGetLastError();               // a launch the block shape does not allow fails here
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaEventElapsedTime(&g_last_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e == cudaSuccess) e = cudaMemcpy(u_host, du, 3 * (size_t)npts * sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : -2;
}
#endif
