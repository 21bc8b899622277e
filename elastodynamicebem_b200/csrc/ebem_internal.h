// Internal declarations shared by the CUDA translation units of libebem.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ebem.h"
#include "sa_device.cuh"

struct cusolverDnContext;   // cuSOLVER dense handle (cusolverDnHandle_t)
struct cublasContext;       // cuBLAS handle (cublasHandle_t)

namespace ebem { struct NodeW; }

namespace ebem {

// Thread-local error message returned by ebem_last_error().
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

// Generation of device dev's cached state, bumped by ebem_device_release:
// per-thread library handles and the allocation-free scratch address cached
// under an older generation are abandoned and rebuilt on next use.
unsigned device_generation(int dev);
// Destroys the calling thread's cuSOLVER / cuBLAS handles of device dev.
void release_thread_handles(int dev);

// Per-call device workspace, stream-ordered, from a memory pool the library
// keeps for each device.  Up to kWorkspaceKeep bytes stay reserved in the pool
// between calls, so a repeated call allocates without a driver call and
// without the device-wide synchronisation of cudaMalloc / cudaFree.  A buffer
// is released with ws_free on the stream that last uses it (on the current
// device, as when it was allocated).  ebem_release_workspace() hands the
// reserved memory back.
constexpr unsigned long long kWorkspaceKeep = 2ull << 30;
cudaError_t ws_malloc(void** p, size_t bytes, cudaStream_t s);
cudaError_t ws_free(void* p, cudaStream_t s);
template <class T>
cudaError_t ws_malloc(T** p, size_t bytes, cudaStream_t s) {
    return ws_malloc(reinterpret_cast<void**>(p), bytes, s);
}

// Several small host tables uploaded as one workspace block with one copy
// (each table on a 16-byte boundary): a call that needs a handful of them
// then pays one allocation and one host-to-device copy instead of one each.
struct HostPack {
    std::vector<unsigned char> bytes;
    // appends n bytes from p; returns the table's byte offset in the block
    size_t add(const void* p, size_t n) {
        const size_t o = (bytes.size() + 15) & ~(size_t)15;
        bytes.resize(o + n);
        if (n) std::memcpy(bytes.data() + o, p, n);
        return o;
    }
    // device copy on stream s into a new workspace block (ws_free it)
    cudaError_t upload(unsigned char** d, cudaStream_t s) const {
        cudaError_t e = ws_malloc(d, bytes.size() ? bytes.size() : 16, s);
        if (e == cudaSuccess && !bytes.empty())
            e = cudaMemcpyAsync(*d, bytes.data(), bytes.size(), cudaMemcpyHostToDevice, s);
        return e;
    }
};

#define EBEM_CUDA_TRY(expr)                                                        \
    do {                                                                           \
        cudaError_t _e = (expr);                                                   \
        if (_e != cudaSuccess)                                                     \
            return ::ebem::fail(EBEM_ERR_CUDA, std::string(#expr) + ": " +         \
                                cudaGetErrorString(_e));                           \
    } while (0)

struct MeshData {
    int nv = 0, nt = 0;
    int device = 0;
    double* d_coords = nullptr;   // nv x 3
    int32_t* d_tris = nullptr;    // nt x 3 (0-based)
    TriGeom* d_geo = nullptr;     // nt
    // mapped outer nodes, (x, y, z, weight) per (triangle, node): one table
    // per Gauss-Hammer rule, built on first use and freed only with the mesh,
    // so that a pointer held by a batch plan stays valid when the mesh is
    // later used with another rule.  d_nodes / nodes_rule name the table of
    // the last map_nodes call.
    static constexpr int kNodeRules = 6;          // rules of 1, 3, 7, 12, 19, 28 nodes
    NodeW* d_node_tables[kNodeRules] = {};
    // composite rules (n_gh nodes on n_sub sub-triangles, n_sub > 1), the same
    // lifetime: key n_gh * 4096 + n_sub
    static constexpr int kCompRules = 16;
    int comp_key[kCompRules] = {};
    NodeW* d_comp_tables[kCompRules] = {};
    int nodes_rule = 0;
    NodeW* d_nodes = nullptr;     // nt x nodes_rule
    // direct formulation (built on first use): per-triangle P1 data and the
    // vertex -> triangles adjacency (CSR)
    struct DirTri* d_dir = nullptr;
    int32_t* d_vt_off = nullptr;  // nv + 1
    int32_t* d_vt_tri = nullptr;  // 3 nt
    double max_len = 0.0;         // largest triangle edge
};

// Gauss-Hammer base rules (barycentric nodes, weights summing to 1/2).
int gh_base(int n, double bary[][3], double w[]);
// Composite rule on n_sub congruent sub-triangles, weights scaled by 2/n_sub.
int gh_composite(int n_nodes, int n_sub, double* nodes, double* weights);

// Device preparation of the per-triangle geometry.
int prep_mesh(MeshData& m, cudaStream_t s);
int map_nodes(MeshData& m, int n_gh, cudaStream_t s);
// The same for GaussHammerComposite(n_sub, n_gh): n_gh * n_sub nodes per
// triangle in m.d_nodes (n_sub = 1 is map_nodes).
int map_nodes_composite(MeshData& m, int n_gh, int n_sub, cudaStream_t s);

struct PhysParams {
    double rho, velP, velS, dt;
    int nT;
    double lam = 0.0, mu = 0.0;
};
PhysParams phys_from(const ebem_problem* p);

// SA assembly of source rows [src0, src0+nsrc) into a device buffer
// (column-major 3 nsrc x 3N per lag, leading dimension ld, lag stride ld_lag).
int launch_sa_assemble(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                       double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count,
                       cudaStream_t s, int diag_only = 0, int mixed = 0, const int2* pairs = nullptr,
                       long long npairs = 0);
// The same assembly in two passes (sa_twopass.cu): F(t_k) of every (pair,
// level) into a workspace, then the second difference written column by
// column.  Dense outputs only (no pair list, no diagonal-only mode).
// With a class array cls (device, cls[(j N + i) nlag + l - lag0] for field j,
// source i; src0 = 0, nsrc = N) only the lags of class cls_want are written
// (and the zeros outside the non-null lags when cls_want is 0), with the
// outer rule in m.d_nodes (n_gh nodes per triangle, composite or not).
int launch_sa_twopass(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                     double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count, int mixed,
                     cudaStream_t s, const unsigned char* cls = nullptr, int cls_want = -1);
// Per-pass device times of the two-pass assembly (ebem_profile_enable / _read).
void profile_enable(int on);
void profile_read(double ms[2], long long n[2], int reset);
// Pass 1 of that assembly by the one-warp-per-pair kernel (sa_assemble.cu):
// F(t_k) and the non-null lags of the pairs of field columns [j0, j0 + nj).
int launch_sa_fwarp(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc, int j0,
                    int nj, int kbase, int KL, double* d_F, int2* d_band, unsigned long long* d_count, int mixed,
                    cudaStream_t s, const unsigned char* cls = nullptr, int cls_want = -1);
// Blocks of explicit (source, field) pairs (int2 list, device) at lags
// [0, nlag) with the rule in m.d_nodes: out[(p nlag + l) 6 + e], 6 symmetric
// entries per block, zero outside the pair's non-null lags.
int launch_sa_pair_blocks(const MeshData& m, const PhysParams& P, int n_gh, const int2* d_pairs, long long npairs,
                          int nlag, double* d_out, cudaStream_t s);
// Allocation-free variant of the full assembly (device E, ld = 3N): mapped
// nodes and the counter live in a static device array (sa_assemble.cu).
int launch_sa_assemble_noalloc(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, double* d_E,
                               int accumulate, bool count, unsigned long long* host_count, cudaStream_t s);
size_t noalloc_max_nodes();

// One instance of a batched assembly (device table entry).
struct BatchInst {
    const TriGeom* geo;
    const NodeW* nodes;
    double* E;              // 9 N^2 nlag doubles, lags 0..nlag-1
    int N, nlag;
    double velP, velS, dt, c4pirho;
    long long pair_begin;   // first index of this instance in the concatenated pair space
};
// Persistent batched assembly over all instances; d_next must be zero.
int launch_sa_batch(const BatchInst* d_insts, int ninst, long long total, int n_gh, int mixed, int wpb, int chunk,
                    unsigned long long* d_next, int device, cudaStream_t s);
int launch_ghc_assemble(const MeshData& m, const PhysParams& P, int n_gh, int n_sub, int n_sing, int lag0, int nlag,
                        double* d_E, size_t ld, size_t ld_lag, cudaStream_t s);

int launch_rhs(const MeshData& m, const PhysParams& P, int n_gh, int datum, double* d_rhs, cudaStream_t s);
// factor: EBEM_FACTOR_LU (partial pivoting, the reference's lu) or
// EBEM_FACTOR_CHOLESKY (of the symmetric part (E_0 + E_0^T) / 2).
int march_device(const double* dE, int n3, int L, const double* drhs, int nT, double* dphi, cudaStream_t s,
                 int factor = EBEM_FACTOR_LU);
// A square system solved many times: A^{-1} formed once from the LU factors
// (partial pivoting), so that each solve is one matrix-vector (or matrix)
// product instead of a row-interchange pass and two triangular solves, which
// for one right-hand side are latency-bound.  `pooled` plans (the marching's
// own) keep the inverse in the workspace pool, released on `st`.
struct LuPlan {
    int n = 0;
    double* inv = nullptr;      // A^{-1}, column-major n x n
    bool pooled = false;
    cudaStream_t st = nullptr;
};
// cuSOLVER / cuBLAS handles of the calling host thread on the current device,
// created on first use and kept for the life of the thread (creating one costs
// milliseconds and allocates device memory), bound to stream s on return.
int solver_handle(cudaStream_t s, ::cusolverDnContext** h);
int blas_handle(cudaStream_t s, ::cublasContext** h);
// Banded Toeplitz blocks (csrc/banded.cu): pair p = i N + j owns the blocks
// [off[p], off[p+1]) of Eb, one per lag of its band starting at lo[p], the 6
// symmetric entries (11,12,13,22,23,33) of each.
struct BandOp {
    int N = 0, L = 0;
    long long nblocks = 0;
    double* Eb = nullptr;
    long long* off = nullptr;
    int* lo = nullptr;
};
int band_structure(const MeshData& m, const PhysParams& P, int L, BandOp* op, cudaStream_t s);
// In-place exclusive prefix sum of n values on stream s (banded.cu); returns
// after the stream has finished it.
int exclusive_scan(long long* d, long long n, cudaStream_t s);
void band_free(BandOp* op);
int band_to_dense(const BandOp& op, int lag0, int nlag, double* d_E, cudaStream_t s);
int band_march(const BandOp& op, const double* d_rhs, int nT, double* d_phi, cudaStream_t s);
int launch_sa_assemble_banded(const MeshData& m, const PhysParams& P, int n_gh, int L, double* d_Eb,
                              const long long* d_boff, const int* d_blo, int mixed, cudaStream_t s);
int lu_plan_create(const double* dA, int n, cudaStream_t s, LuPlan* plan, bool pooled = false, bool cholesky = false);
int lu_plan_solve(LuPlan* plan, double* db, int nrhs, cudaStream_t s);
void lu_plan_destroy(LuPlan* plan);
int launch_pp_sa(const MeshData& m, const PhysParams& P, const double* d_phi, const double* d_pts, int npts,
                 const double* h_times, int ntimes, double* d_u, cudaStream_t s);
// Numerical post-processing (pp_num.cu): composite rule (n_sub, n_sing) per
// triangle, kernelLayer's semantics when layer != 0, else kernelSP's (node
// stride 3 unless fix); u (ntimes x npts x 3) fully written.
int launch_pp_num(const MeshData& m, const PhysParams& P, int n_sub, int n_sing, int layer, int fix,
                  const double* d_phi, const double* d_pts, int npts, const double* h_times, int ntimes, double* d_u,
                  cudaStream_t s);

// ---------------------------------------------------------------------------
// direct formulation (direct.cu)

// Per-triangle data of the direct formulation: vertices, unit normal and area
// (readSpaceMesh.m:114-121), P1 basis phi_k(y) = v[k] + M[3k..3k+2] . y, longest edge.
struct DirTri {
    double V[3][3];
    double n[3];
    double area;
    double M[9];
    double v[3];
    double maxL;
};

int prep_direct(MeshData& m, cudaStream_t s);
void free_direct(MeshData& m);
// K_l (3N x 3Nv per lag, column-major, ld = 3N): off-singular part with the
// outer GH rule n_gh and composite inner rule (n_sub, n_sing), then, when
// n_diag > 0, the same-triangle parts on the DIAG rule.  Accumulates (+=).
int launch_k_assemble(const MeshData& m, const PhysParams& P, int n_gh, int n_sub, int n_sing, int n_diag, int lag0,
                      int nlag, int nblocks, int fix, double* d_K, cudaStream_t s);
// Diagonal blocks of V_l on the DIAG rule, written into a 3N x 3N per lag buffer.
int launch_v_diag(const MeshData& m, const PhysParams& P, int n_gh, int n_diag, int lag0, int nlag, double* d_V,
                  cudaStream_t s);
// Direct post-processing.  mode 0: u(t_q, x_p) = sum_n G_n a_n - P_n b_n into
// d_u (ntimes x npts x 3); mode 1: the matrices G (3 nHat x 3N) and P
// (3 nHat x 3Nv) of one (x, t) into d_G, d_P.
int launch_pp_dir(const MeshData& m, const PhysParams& P, int n_sub, int n_sing, int fix, const double* d_pts, int npts,
                  const double* h_times, int ntimes, const double* d_a, const double* d_b, double* d_u, double* d_G,
                  double* d_P, int mode, cudaStream_t s);
// Direct time marching.  DN: least squares (K_0 + I) u_n = beta_V,n + I u_{n-1}
// - sum K_l u_{n-l}; DD: V_0 phi_n = rhs_n / 2 + beta_K,n - sum V_l phi_{n-l}.
int march_dn_device(const MeshData& m, const double* dV, int LV, const double* dK, int LK, const double* d_gV, int nT,
                    double* d_u, cudaStream_t s);
int march_dd_device(const MeshData& m, const double* dV, int LV, const double* dK, int LK, const double* d_rhs,
                    const double* d_gK, int nT, double* d_phi, cudaStream_t s);
int launch_hist_gemv(const double* A, int n3, long long K, const double* x, double* y, int sm_count, cudaStream_t s);

// ---------------------------------------------------------------------------
// learned quadrature selector (selector.cu)
// features of samples[3 q + 0..2] = (source, field, lag)
int selector_features(const MeshData& m, const PhysParams& P, const int* d_samples, long long n, float* d_out,
                      cudaStream_t s);
// 1 where a wavefront sweeps the sample's distance window (those lags take the maximal rule)
int selector_sweeps(const MeshData& m, const PhysParams& P, const int* d_samples, long long n, unsigned char* d_out,
                    cudaStream_t s);
// labels from the samples' blocks at the four rules (blocks[(c n + q) 6 + e])
int selector_labels(const double* d_blocks, long long n, double tol, double scale, const double* d_scales,
                    int* d_labels, cudaStream_t s);
int selector_grad(const float* d_params, const float* d_feats, const int* d_labels, long long n, float* d_grad,
                  float* d_loss, cudaStream_t s);
int selector_train(float* d_params, const float* d_feats, const int* d_labels, long long n, int epochs, int batch,
                   float lr, unsigned long long seed, float* h_losses, cudaStream_t s);
int selector_infer(const float* d_params, const MeshData& m, const PhysParams& P, float threshold, int lag0, int nlag,
                   unsigned char* d_cls, long long* h_counts, cudaStream_t s);
int assemble_selected(MeshData& m, const PhysParams& P, const int* h_rules, int nclass, const unsigned char* d_cls,
                      int lag0, int nlag, double* d_E, int prec, long long* h_counts, cudaStream_t s);
void selector_init(float* h_params, unsigned long long seed);

}  // namespace ebem
