// ORACLE — test infrastructure only.  Host launcher for the reference's own
// numerical-inner kernel, kernelGHC (functions/BEMenerg_indir/BEMenerg_core/
// BEMenerg_coreGPU/CUDAkernels/kernelGHC.cu), compiled from the reference's
// source file in place (the build recipe passes its path as REF_KERNEL_GHC;
// no reference source is copied here).  Arguments and launch shape follow
// BEMenerg_coreGPU_timeMarching.m:40-85 and BEMenerg_coreGPU_launchKernel.m:1-15.
#include REF_KERNEL_GHC

#include <cuda_runtime.h>
#include <vector>

static float g_last_ms = -1.0f;   // device time of the last reference kernel launch (CUDA events)

extern "C" float ref_last_kernel_ms() { return g_last_ms; }

extern "C" int ref_ghc(double* matrix_host, int N, int nlag, double deltaT, double velP, double velS,
                       double const4PiRho, const double* GHw, const double* GHn /* nGH x 3 */, int nGH,
                       const double* GHCw, const double* GHCn /* nSub*nSing x 3 */, int nSub, int nSing,
                       const double* vertsT /* 9N */, const double* areeT /* N */, int offsetZ, int numBlocks) {
    size_t nm = (size_t)9 * N * N * nlag;
    int nInt = nSub * nSing;
    std::vector<double> gx(nGH), gy(nGH), gz(nGH), cx(nInt), cy(nInt), cz(nInt);
    for (int k = 0; k < nGH; k++) { gx[k] = GHn[3 * k]; gy[k] = GHn[3 * k + 1]; gz[k] = GHn[3 * k + 2]; }
    for (int k = 0; k < nInt; k++) { cx[k] = GHCn[3 * k]; cy[k] = GHCn[3 * k + 1]; cz[k] = GHCn[3 * k + 2]; }
    double *d_m, *d_w, *d_x, *d_y, *d_z, *d_cw, *d_cx, *d_cy, *d_cz, *d_v, *d_a;
    if (cudaMalloc(&d_m, nm * 8) || cudaMalloc(&d_w, nGH * 8) || cudaMalloc(&d_x, nGH * 8) || cudaMalloc(&d_y, nGH * 8) ||
        cudaMalloc(&d_z, nGH * 8) || cudaMalloc(&d_cw, nSing * 8) || cudaMalloc(&d_cx, nInt * 8) ||
        cudaMalloc(&d_cy, nInt * 8) || cudaMalloc(&d_cz, nInt * 8) || cudaMalloc(&d_v, 9 * (size_t)N * 8) ||
        cudaMalloc(&d_a, (size_t)N * 8))
        return -3;
    cudaMemcpy(d_m, matrix_host, nm * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_w, GHw, nGH * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_x, gx.data(), nGH * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_y, gy.data(), nGH * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_z, gz.data(), nGH * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_cw, GHCw, nSing * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_cx, cx.data(), nInt * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_cy, cy.data(), nInt * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_cz, cz.data(), nInt * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_v, vertsT, 9 * (size_t)N * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_a, areeT, (size_t)N * 8, cudaMemcpyHostToDevice);
    dim3 grid(N, N, nlag), block(nSub, nSing);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    kernelGHC<<<grid, block, nSub * nSing * 9 * sizeof(double)>>>(d_m, deltaT, velP, velS, const4PiRho, d_w, d_x, d_y,
                                                                  d_z, nGH, d_cw, d_cx, d_cy, d_cz, d_v, d_a,
                                                                  offsetZ, numBlocks);
    cudaEventRecord(e1);
    cudaError_t e = cudaGetLastError();               // a launch the block shape does not allow fails here
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaEventElapsedTime(&g_last_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e == cudaSuccess) e = cudaMemcpy(matrix_host, d_m, nm * 8, cudaMemcpyDeviceToHost);
    cudaFree(d_m); cudaFree(d_w); cudaFree(d_x); cudaFree(d_y); cudaFree(d_z); cudaFree(d_cw);
    cudaFree(d_cx); cudaFree(d_cy); cudaFree(d_cz); cudaFree(d_v); cudaFree(d_a);
    return e == cudaSuccess ? 0 : -2;
}
