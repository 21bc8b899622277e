/*
 * ebem_mex.c — MATLAB gateway of libebem: ebem_mex(cmd, ...) forwards to the
 * C ABI of include/ebem.h.  The replacement bodies of the reference's MATLAB
 * entry points (the .m files beside this file) call it; their signatures stay
 * those of the reference.
 *
 * Build on a MATLAB host (interleaved complex API, R2018a and later):
 *   mex -R2018a -I<repo>/include ebem_mex.c -L<repo>/elastodynamicebem_b200 -lebem
 *
 * Conventions of every command:
 *   P      vertex coordinates, Nv x 3 (domainMesh.coordinates)
 *   T      triangles, N x 3 or more columns, 1-based (domainMesh.triangles)
 *   q      [rho mu lambda Tfin nT] (pbParam.rho, .mu, .lambda, .Tfin, .nT)
 *   arrays are host double arrays in the reference's layouts (the library
 *   stages them through device memory): E 3N x 3N x L, density 3N x nT,
 *   points npts x 3, displacement 3 x npts x ntimes.
 * Every library error becomes mexErrMsgIdAndTxt("ebem:<cmd>", message) after
 * the mesh handle of the call has been destroyed.
 *
 * Commands (-> C ABI):
 *   v = ebem_mex('version')                                    ebem_version
 *   [n, w] = ebem_mex('quad_gh', nNodes, nSub)                 ebem_quad_gh
 *   L = ebem_mex('num_blocks', P, T, q)                        ebem_num_blocks
 *   E = ebem_mex('assemble_sa', P, T, q, nGH, lag0, nlag[, prec])   ebem_assemble_sa_ex
 *   E = ebem_mex('assemble_ghc', P, T, q, nGH, nSub, nSing, lag0, nlag)   ebem_assemble_ghc (SA diagonal)
 *   b = ebem_mex('rhs', P, T, q, nGH, datum)                   ebem_rhs
 *   phi = ebem_mex('march', E, b)                              ebem_march
 *   phi = ebem_mex('timemarch_sa', P, T, q, nGH, datum[, prec])     ebem_timemarch_sa_ex
 *   phi = ebem_mex('timemarch_ghc', P, T, q, nGH, nSub, nSing, datum)
 *                                                              ebem_assemble_ghc + ebem_rhs + ebem_march
 *   phi = ebem_mex('timemarch_banded', P, T, q, nGH, datum[, prec])
 *                                                              ebem_banded_assemble + ebem_rhs + ebem_banded_march
 *   u = ebem_mex('pp_sa', P, T, q, phi, X, t)                  ebem_pp_sa
 *   u = ebem_mex('pp_gpu', P, T, q, phi, X, t, nSub, nSing, variant[, flags])   ebem_pp_gpu
 *   [LV, LK] = ebem_mex('num_blocks_dir', P, T, q)             ebem_num_blocks_dir
 *   V = ebem_mex('assemble_v', P, T, q, rules, lag0, nlag)     ebem_assemble_v
 *   K = ebem_mex('assemble_k', P, T, q, rules, lag0, nlag[, flags])   ebem_assemble_k
 *   u = ebem_mex('march_dn', P, T, q, rules, gV[, flags])      ebem_assemble_v + _k + ebem_march_dn
 *   phi = ebem_mex('march_dd', P, T, q, rules, rhs, gK[, flags])     ebem_assemble_v + _k + ebem_march_dd
 *   u = ebem_mex('pp_dir', P, T, q, nSub, nSing, a, b, X, t[, flags])   ebem_pp_dir
 *   ebem_mex('release'[, device])                              ebem_release_workspace / ebem_device_release
 * rules = [nGH nSub nSing nDiag] ("FN nGH nSub nSing nDiag"); datum as ebem_rhs.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "mex.h"
#include "ebem.h"

static ebem_mesh* g_mesh = NULL;          /* the current command's mesh, destroyed on error */
static char g_cmd[32] = "";

static void fail_now(const char* msg) {
    char id[64];
    if (g_mesh) {
        ebem_mesh_destroy(g_mesh);
        g_mesh = NULL;
    }
    snprintf(id, sizeof id, "ebem:%s", g_cmd[0] ? g_cmd : "call");
    mexErrMsgIdAndTxt(id, "%s", msg);
}

static void check(int rc) {
    if (rc != EBEM_OK) fail_now(ebem_last_error());
}

static void need(int cond, const char* msg) {
    if (!cond) fail_now(msg);
}

static const double* dbl(const mxArray* a, const char* what) {
    need(a != NULL && mxIsDouble(a), what);
    return mxGetDoubles(a);
}

static int iarg(const mxArray* a, const char* what) {
    need(a != NULL && mxIsDouble(a) && mxGetNumberOfElements(a) == 1, what);
    return (int)mxGetScalar(a);
}

/* q = [rho mu lambda Tfin nT] */
static ebem_problem prob_arg(const mxArray* a) {
    ebem_problem p;
    const double* q = dbl(a, "problem must be [rho mu lambda Tfin nT]");
    need(mxGetNumberOfElements(a) == 5, "problem must be [rho mu lambda Tfin nT]");
    p.rho = q[0];
    p.mu = q[1];
    p.lambda = q[2];
    p.tfin = q[3];
    p.nt = (int)q[4];
    return p;
}

/* Mesh from MATLAB's column-major coordinates (Nv x 3) and 1-based
 * triangles (N x >= 3); the handle lives until the command ends. */
static ebem_mesh* mesh_arg(const mxArray* Pa, const mxArray* Ta) {
    const double* P = dbl(Pa, "coordinates must be a double Nv x 3 array");
    const double* T = dbl(Ta, "triangles must be a double N x 3 array");
    int nv = (int)mxGetM(Pa), nt = (int)mxGetM(Ta);
    need(mxGetN(Pa) == 3 && mxGetN(Ta) >= 3, "coordinates Nv x 3 and triangles N x 3 expected");
    double* coords = (double*)mxMalloc(sizeof(double) * 3 * (size_t)nv);
    int32_t* tris = (int32_t*)mxMalloc(sizeof(int32_t) * 3 * (size_t)nt);
    for (int i = 0; i < nv; i++)
        for (int c = 0; c < 3; c++) coords[3 * i + c] = P[(size_t)c * nv + i];
    for (int i = 0; i < nt; i++)
        for (int c = 0; c < 3; c++) tris[3 * i + c] = (int32_t)T[(size_t)c * nt + i] - 1;
    int rc = ebem_mesh_create(coords, nv, tris, nt, &g_mesh);
    mxFree(coords);
    mxFree(tris);
    check(rc);
    return g_mesh;
}

static int ntri(void) {
    int nv = 0, nt = 0;
    ebem_mesh_info(g_mesh, &nv, &nt);
    return nt;
}

static int nvert(void) {
    int nv = 0, nt = 0;
    ebem_mesh_info(g_mesh, &nv, &nt);
    return nv;
}

static mxArray* zeros3(size_t a, size_t b, size_t c) {
    mwSize dims[3];
    dims[0] = a;
    dims[1] = b;
    dims[2] = c;
    return mxCreateNumericArray(3, dims, mxDOUBLE_CLASS, mxREAL);
}

/* npts x 3 (column-major) -> row-major copy for the C ABI */
static double* points_arg(const mxArray* Xa, int* npts) {
    const double* X = dbl(Xa, "points must be a double npts x 3 array");
    int n = (int)mxGetM(Xa);
    need(mxGetN(Xa) == 3 && n >= 1, "points must be npts x 3");
    double* p = (double*)mxMalloc(sizeof(double) * 3 * (size_t)n);
    for (int i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) p[3 * i + c] = X[(size_t)c * n + i];
    *npts = n;
    return p;
}

static void rules_arg(const mxArray* a, int r[4]) {
    const double* v = dbl(a, "rules must be [nGH nSub nSing nDiag]");
    need(mxGetNumberOfElements(a) == 4, "rules must be [nGH nSub nSing nDiag]");
    for (int k = 0; k < 4; k++) r[k] = (int)v[k];
}

static void release_at_exit(void) { ebem_release_workspace(); }

/* ---------------------------------------------------------------------
 * indirect formulation */

static void cmd_assemble_sa(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 7, "usage: E = ebem_mex('assemble_sa', P, T, q, nGH, lag0, nlag[, prec])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int ngh = iarg(prhs[4], "nGH"), lag0 = iarg(prhs[5], "lag0"), nlag = iarg(prhs[6], "nlag");
    int prec = nrhs > 7 ? iarg(prhs[7], "prec") : EBEM_PREC_FP64;
    need(nlag >= 1 && lag0 >= 0, "need lag0 >= 0 and nlag >= 1");
    int n = ntri();
    plhs[0] = zeros3(3 * (size_t)n, 3 * (size_t)n, (size_t)nlag);
    check(ebem_assemble_sa_ex(g_mesh, &p, ngh, lag0, nlag, 0, n, mxGetDoubles(plhs[0]), 3LL * n, 0, prec, NULL, NULL));
}

static void cmd_assemble_ghc(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 9, "usage: E = ebem_mex('assemble_ghc', P, T, q, nGH, nSub, nSing, lag0, nlag)");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int ngh = iarg(prhs[4], "nGH"), nsub = iarg(prhs[5], "nSub"), nsing = iarg(prhs[6], "nSing");
    int lag0 = iarg(prhs[7], "lag0"), nlag = iarg(prhs[8], "nlag");
    need(nlag >= 1 && lag0 >= 0, "need lag0 >= 0 and nlag >= 1");
    int n = ntri();
    plhs[0] = zeros3(3 * (size_t)n, 3 * (size_t)n, (size_t)nlag);       /* kernelGHC accumulates into zeros */
    check(ebem_assemble_ghc(g_mesh, &p, ngh, nsub, nsing, lag0, nlag, mxGetDoubles(plhs[0]), 1, NULL));
}

static void cmd_rhs(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 6, "usage: b = ebem_mex('rhs', P, T, q, nGH, datum)");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    plhs[0] = mxCreateDoubleMatrix(3 * (size_t)ntri(), (size_t)p.nt, mxREAL);
    check(ebem_rhs(g_mesh, &p, iarg(prhs[4], "nGH"), iarg(prhs[5], "datum"), mxGetDoubles(plhs[0]), NULL));
}

static void cmd_march(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 3, "usage: phi = ebem_mex('march', E, b)");
    const double* E = dbl(prhs[1], "E must be a double 3N x 3N x L array");
    const double* b = dbl(prhs[2], "b must be a double 3N x nT array");
    size_t n3 = mxGetM(prhs[1]), nT = mxGetN(prhs[2]);
    need(n3 > 0 && mxGetM(prhs[2]) == n3 && mxGetNumberOfElements(prhs[1]) % (n3 * n3) == 0,
         "E (3N x 3N x L) and b (3N x nT) do not match");
    int L = (int)(mxGetNumberOfElements(prhs[1]) / (n3 * n3));
    plhs[0] = mxCreateDoubleMatrix(n3, nT, mxREAL);
    check(ebem_march(E, (int)n3, L, b, (int)nT, mxGetDoubles(plhs[0]), NULL));
}

static void cmd_timemarch_sa(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 6, "usage: phi = ebem_mex('timemarch_sa', P, T, q, nGH, datum[, prec])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int prec = nrhs > 6 ? iarg(prhs[6], "prec") : EBEM_PREC_FP64;
    plhs[0] = mxCreateDoubleMatrix(3 * (size_t)ntri(), (size_t)p.nt, mxREAL);
    check(ebem_timemarch_sa_ex(g_mesh, &p, iarg(prhs[4], "nGH"), iarg(prhs[5], "datum"), prec, mxGetDoubles(plhs[0]),
                               NULL, NULL));
}

/* The reference's GPU method: numerical inner rule off the diagonal,
 * semi-analytic diagonal, LU marching (BEMenerg_coreGPU_timeMarching.m). */
static void cmd_timemarch_ghc(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 8, "usage: phi = ebem_mex('timemarch_ghc', P, T, q, nGH, nSub, nSing, datum)");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int ngh = iarg(prhs[4], "nGH"), nsub = iarg(prhs[5], "nSub"), nsing = iarg(prhs[6], "nSing");
    int datum = iarg(prhs[7], "datum"), L = 0, n = ntri();
    check(ebem_num_blocks(g_mesh, &p, &L));
    mxArray* E = zeros3(3 * (size_t)n, 3 * (size_t)n, (size_t)L);
    mxArray* b = mxCreateDoubleMatrix(3 * (size_t)n, (size_t)p.nt, mxREAL);
    plhs[0] = mxCreateDoubleMatrix(3 * (size_t)n, (size_t)p.nt, mxREAL);
    check(ebem_assemble_ghc(g_mesh, &p, ngh, nsub, nsing, 0, L, mxGetDoubles(E), 1, NULL));
    check(ebem_rhs(g_mesh, &p, ngh, datum, mxGetDoubles(b), NULL));
    check(ebem_march(mxGetDoubles(E), 3 * n, L, mxGetDoubles(b), p.nt, mxGetDoubles(plhs[0]), NULL));
    mxDestroyArray(E);
    mxDestroyArray(b);
}

/* Banded block storage: 6 doubles per non-null pair-lag. */
static void cmd_timemarch_banded(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 6, "usage: phi = ebem_mex('timemarch_banded', P, T, q, nGH, datum[, prec])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int ngh = iarg(prhs[4], "nGH"), datum = iarg(prhs[5], "datum");
    int prec = nrhs > 6 ? iarg(prhs[6], "prec") : EBEM_PREC_FP64;
    size_t n3 = 3 * (size_t)ntri();
    mxArray* b = mxCreateDoubleMatrix(n3, (size_t)p.nt, mxREAL);
    plhs[0] = mxCreateDoubleMatrix(n3, (size_t)p.nt, mxREAL);
    check(ebem_rhs(g_mesh, &p, ngh, datum, mxGetDoubles(b), NULL));
    ebem_banded* op = NULL;
    check(ebem_banded_assemble(g_mesh, &p, ngh, prec, NULL, &op));
    int rc = ebem_banded_march(op, mxGetDoubles(b), p.nt, mxGetDoubles(plhs[0]), NULL);
    ebem_banded_destroy(op);
    mxDestroyArray(b);
    check(rc);
}

static void cmd_pp_sa(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 7, "usage: u = ebem_mex('pp_sa', P, T, q, phi, X, t)");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    const double* phi = dbl(prhs[4], "phi must be a double 3N x nT array");
    need(mxGetM(prhs[4]) == 3 * (size_t)ntri() && mxGetN(prhs[4]) == (size_t)p.nt, "phi must be 3N x nT");
    int np = 0;
    double* X = points_arg(prhs[5], &np);
    const double* t = dbl(prhs[6], "times must be a double vector");
    int nt = (int)mxGetNumberOfElements(prhs[6]);
    plhs[0] = zeros3(3, (size_t)np, (size_t)nt);
    int rc = ebem_pp_sa(g_mesh, &p, phi, X, np, t, nt, mxGetDoubles(plhs[0]), NULL);
    mxFree(X);
    check(rc);
}

static void cmd_pp_gpu(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 10, "usage: u = ebem_mex('pp_gpu', P, T, q, phi, X, t, nSub, nSing, variant[, flags])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    const double* phi = dbl(prhs[4], "phi must be a double 3N x nT array");
    need(mxGetM(prhs[4]) == 3 * (size_t)ntri() && mxGetN(prhs[4]) == (size_t)p.nt, "phi must be 3N x nT");
    int np = 0;
    double* X = points_arg(prhs[5], &np);
    const double* t = dbl(prhs[6], "times must be a double vector");
    int nt = (int)mxGetNumberOfElements(prhs[6]);
    int flags = nrhs > 10 ? iarg(prhs[10], "flags") : 0;
    plhs[0] = zeros3(3, (size_t)np, (size_t)nt);
    int rc = ebem_pp_gpu(g_mesh, &p, iarg(prhs[7], "nSub"), iarg(prhs[8], "nSing"), iarg(prhs[9], "variant"), flags,
                         phi, X, np, t, nt, mxGetDoubles(plhs[0]), NULL);
    mxFree(X);
    check(rc);
}

/* ---------------------------------------------------------------------
 * direct formulation */

static void cmd_assemble_v(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 7, "usage: V = ebem_mex('assemble_v', P, T, q, rules, lag0, nlag)");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int r[4];
    rules_arg(prhs[4], r);
    int lag0 = iarg(prhs[5], "lag0"), nlag = iarg(prhs[6], "nlag"), n = ntri();
    need(nlag >= 1 && lag0 >= 0, "need lag0 >= 0 and nlag >= 1");
    plhs[0] = zeros3(3 * (size_t)n, 3 * (size_t)n, (size_t)nlag);
    check(ebem_assemble_v(g_mesh, &p, r[0], r[1], r[2], r[3], lag0, nlag, mxGetDoubles(plhs[0]), NULL));
}

static void cmd_assemble_k(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 7, "usage: K = ebem_mex('assemble_k', P, T, q, rules, lag0, nlag[, flags])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int r[4];
    rules_arg(prhs[4], r);
    int lag0 = iarg(prhs[5], "lag0"), nlag = iarg(prhs[6], "nlag");
    int flags = nrhs > 7 ? iarg(prhs[7], "flags") : 0;
    need(nlag >= 1 && lag0 >= 0, "need lag0 >= 0 and nlag >= 1");
    plhs[0] = zeros3(3 * (size_t)ntri(), 3 * (size_t)nvert(), (size_t)nlag);
    check(ebem_assemble_k(g_mesh, &p, r[0], r[1], r[2], r[3], lag0, nlag, flags, mxGetDoubles(plhs[0]), 0, NULL));
}

/* V_0..V_{LV-1} and K_0..K_{LK-1} of the mesh (host arrays owned by the caller). */
static void dir_operators(const ebem_problem* p, const int r[4], int flags, mxArray** V, int* LV, mxArray** K,
                          int* LK) {
    int n = ntri(), nv = nvert();
    check(ebem_num_blocks_dir(g_mesh, p, LV, LK));
    *V = zeros3(3 * (size_t)n, 3 * (size_t)n, (size_t)*LV);
    *K = zeros3(3 * (size_t)n, 3 * (size_t)nv, (size_t)*LK);
    check(ebem_assemble_v(g_mesh, p, r[0], r[1], r[2], r[3], 0, *LV, mxGetDoubles(*V), NULL));
    check(ebem_assemble_k(g_mesh, p, r[0], r[1], r[2], r[3], 0, *LK, flags, mxGetDoubles(*K), 0, NULL));
}

/* BEMenerg_dir_timeMarchingN.m: Neumann datum gV (3N x nT) -> u (3Nv x nT). */
static void cmd_march_dn(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 6, "usage: u = ebem_mex('march_dn', P, T, q, rules, gV[, flags])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int r[4];
    rules_arg(prhs[4], r);
    const double* gV = dbl(prhs[5], "gV must be a double 3N x nT array");
    need(mxGetM(prhs[5]) == 3 * (size_t)ntri() && mxGetN(prhs[5]) == (size_t)p.nt, "gV must be 3N x nT");
    int flags = nrhs > 6 ? iarg(prhs[6], "flags") : 0;
    mxArray *V, *K;
    int LV = 0, LK = 0;
    dir_operators(&p, r, flags, &V, &LV, &K, &LK);
    plhs[0] = mxCreateDoubleMatrix(3 * (size_t)nvert(), (size_t)p.nt, mxREAL);
    check(ebem_march_dn(g_mesh, &p, mxGetDoubles(V), LV, mxGetDoubles(K), LK, gV, mxGetDoubles(plhs[0]), NULL));
    mxDestroyArray(V);
    mxDestroyArray(K);
}

/* BEMenerg_dir_timeMarchingD.m: rhs (3N x nT), Dirichlet datum gK (3Nv x nT) -> phi (3N x nT). */
static void cmd_march_dd(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 7, "usage: phi = ebem_mex('march_dd', P, T, q, rules, rhs, gK[, flags])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    int r[4];
    rules_arg(prhs[4], r);
    const double* rhs = dbl(prhs[5], "rhs must be a double 3N x nT array");
    const double* gK = dbl(prhs[6], "gK must be a double 3Nv x nT array");
    need(mxGetM(prhs[5]) == 3 * (size_t)ntri() && mxGetN(prhs[5]) == (size_t)p.nt, "rhs must be 3N x nT");
    need(mxGetM(prhs[6]) == 3 * (size_t)nvert() && mxGetN(prhs[6]) == (size_t)p.nt, "gK must be 3Nv x nT");
    int flags = nrhs > 7 ? iarg(prhs[7], "flags") : 0;
    mxArray *V, *K;
    int LV = 0, LK = 0;
    dir_operators(&p, r, flags, &V, &LV, &K, &LK);
    plhs[0] = mxCreateDoubleMatrix(3 * (size_t)ntri(), (size_t)p.nt, mxREAL);
    check(ebem_march_dd(g_mesh, &p, mxGetDoubles(V), LV, mxGetDoubles(K), LK, rhs, gK, mxGetDoubles(plhs[0]), NULL));
    mxDestroyArray(V);
    mxDestroyArray(K);
}

/* BEMenerg_ppN_setup.m (a = gV, b = u) / BEMenerg_ppD_setup.m (a = phi, b = gK). */
static void cmd_pp_dir(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 10, "usage: u = ebem_mex('pp_dir', P, T, q, nSub, nSing, a, b, X, t[, flags])");
    mesh_arg(prhs[1], prhs[2]);
    ebem_problem p = prob_arg(prhs[3]);
    const double* a = dbl(prhs[6], "a must be a double 3N x nT array");
    const double* b = dbl(prhs[7], "b must be a double 3Nv x nT array");
    need(mxGetM(prhs[6]) == 3 * (size_t)ntri() && mxGetN(prhs[6]) == (size_t)p.nt, "a must be 3N x nT");
    need(mxGetM(prhs[7]) == 3 * (size_t)nvert() && mxGetN(prhs[7]) == (size_t)p.nt, "b must be 3Nv x nT");
    int np = 0;
    double* X = points_arg(prhs[8], &np);
    const double* t = dbl(prhs[9], "times must be a double vector");
    int nt = (int)mxGetNumberOfElements(prhs[9]);
    int flags = nrhs > 10 ? iarg(prhs[10], "flags") : 0;
    plhs[0] = zeros3(3, (size_t)np, (size_t)nt);
    int rc = ebem_pp_dir(g_mesh, &p, iarg(prhs[4], "nSub"), iarg(prhs[5], "nSing"), flags, a, b, X, np, t, nt,
                         mxGetDoubles(plhs[0]), NULL);
    mxFree(X);
    check(rc);
}

/* ---------------------------------------------------------------------
 * dispatch */

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    static int registered = 0;
    if (!registered) {
        mexAtExit(release_at_exit);          /* `clear mex` / MATLAB exit: hand the reserved workspace back */
        registered = 1;
    }
    g_mesh = NULL;
    g_cmd[0] = '\0';
    if (nrhs < 1 || !mxIsChar(prhs[0]) || mxGetString(prhs[0], g_cmd, sizeof g_cmd) != 0)
        fail_now("usage: ebem_mex(cmd, ...) with cmd a command name");
    if (!strcmp(g_cmd, "version")) {
        plhs[0] = mxCreateDoubleScalar((double)ebem_version());
    } else if (!strcmp(g_cmd, "quad_gh")) {
        need(nrhs >= 3, "usage: [n, w] = ebem_mex('quad_gh', nNodes, nSub)");
        int nn = iarg(prhs[1], "nNodes"), ns = iarg(prhs[2], "nSub");
        need(nn >= 1 && nn <= 28 && ns >= 1 && ns <= 4096, "unsupported Gauss-Hammer rule");
        double* nodes = (double*)mxMalloc(sizeof(double) * 3 * (size_t)nn * ns);
        mxArray* w = mxCreateDoubleMatrix((size_t)nn, 1, mxREAL);
        int rc = ebem_quad_gh(nn, ns, nodes, mxGetDoubles(w));
        if (rc != EBEM_OK) {
            mxFree(nodes);
            check(rc);
        }
        plhs[0] = mxCreateDoubleMatrix((size_t)nn * ns, 3, mxREAL);     /* MATLAB's (nSub nNodes) x 3 */
        double* o = mxGetDoubles(plhs[0]);
        for (size_t i = 0; i < (size_t)nn * ns; i++)
            for (int c = 0; c < 3; c++) o[(size_t)c * nn * ns + i] = nodes[3 * i + c];
        mxFree(nodes);
        if (nlhs > 1) plhs[1] = w;
        else mxDestroyArray(w);
    } else if (!strcmp(g_cmd, "num_blocks")) {
        need(nrhs >= 4, "usage: L = ebem_mex('num_blocks', P, T, q)");
        mesh_arg(prhs[1], prhs[2]);
        ebem_problem p = prob_arg(prhs[3]);
        int L = 0;
        check(ebem_num_blocks(g_mesh, &p, &L));
        plhs[0] = mxCreateDoubleScalar((double)L);
    } else if (!strcmp(g_cmd, "num_blocks_dir")) {
        need(nrhs >= 4, "usage: [LV, LK] = ebem_mex('num_blocks_dir', P, T, q)");
        mesh_arg(prhs[1], prhs[2]);
        ebem_problem p = prob_arg(prhs[3]);
        int LV = 0, LK = 0;
        check(ebem_num_blocks_dir(g_mesh, &p, &LV, &LK));
        plhs[0] = mxCreateDoubleScalar((double)LV);
        if (nlhs > 1) plhs[1] = mxCreateDoubleScalar((double)LK);
    } else if (!strcmp(g_cmd, "assemble_sa")) {
        cmd_assemble_sa(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "assemble_ghc")) {
        cmd_assemble_ghc(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "rhs")) {
        cmd_rhs(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "march")) {
        cmd_march(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "timemarch_sa")) {
        cmd_timemarch_sa(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "timemarch_ghc")) {
        cmd_timemarch_ghc(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "timemarch_banded")) {
        cmd_timemarch_banded(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "pp_sa")) {
        cmd_pp_sa(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "pp_gpu")) {
        cmd_pp_gpu(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "assemble_v")) {
        cmd_assemble_v(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "assemble_k")) {
        cmd_assemble_k(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "march_dn")) {
        cmd_march_dn(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "march_dd")) {
        cmd_march_dd(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "pp_dir")) {
        cmd_pp_dir(nlhs, plhs, nrhs, prhs);
    } else if (!strcmp(g_cmd, "release")) {
        check(ebem_release_workspace());
        if (nrhs > 1) check(ebem_device_release(iarg(prhs[1], "device")));
    } else {
        fail_now("unknown command");
    }
    if (g_mesh) {
        ebem_mesh_destroy(g_mesh);
        g_mesh = NULL;
    }
}
