// Device preparation of the mesh and the semi-analytic (SA) assembly kernel.
//
// Reference (paths relative to the reference project root; "SA/" =
// functions/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/):
//   mesh fields      functions/utility/fileRead/readSpaceMesh.m:93-148
//   frame            SA/calcoloMatrice/operazioniGeometriche/calcoloSistemaRiferimento.m
//   Euler matrix     SA/calcoloMatrice/operazioniGeometriche/rotazioneInversaEulero.m:23-176
//   mapped nodes     SA/BEMenerg_coreSA_calcCostantData.m:8-23
//   null test        SA/calcoloMatrice/BEMenerg_coreSA_calcMatrixBlock.m:57-61, clean-up :77
//   sub-block        SA/calcoloMatrice/BEMenerg_coreSA_calcMatrixSubBlock.m:1-111
//   projection       SA/calcoloMatrice/operazioniGeometriche/preparazioneTriangolo.m:1-115
//   edge distance    SA/calcoloMatrice/operazioniGeometriche/calcoloDistanzaTriangolo.m
//   children         SA/calcoloMatrice/BEMenerg_coreSA_calcIntgInt_fieldTriangle.m:13-84
//
// Work decomposition (B200 design, not the reference's): one thread per
// (source i, field j) pair; consecutive lanes take consecutive source
// triangles of the same field triangle, so a warp writes 3 x 32 x 3
// contiguous doubles per block column.  A thread walks the time levels
// t_k = k dt of its pair once, in increasing order; F(t_k) (the combined
// kernel integral at one instant) depends on k only, so each level is
// evaluated once and E_l = F_{l+1} - 2 F_l + F_{l-1} is emitted from a
// three-level sliding window (the reference evaluates every instant three
// times, once per lag that uses it).
#include "ebem_internal.h"
#include "sa_pair.cuh"

namespace ebem {

// ---------------------------------------------------------------------------
// mesh preparation

__global__ void prep_kernel(const double* __restrict__ coords, const int32_t* __restrict__ tris, int nt,
                            TriGeom* __restrict__ geo) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    double V[3][3];
    for (int v = 0; v < 3; v++) {
        int id = tris[3 * t + v];
        for (int c = 0; c < 3; c++) V[v][c] = coords[3 * id + c];
    }
    TriGeom g;
    tri_geom(V, g);
    geo[t] = g;
}

__global__ void map_nodes_kernel(const double* __restrict__ coords, const int32_t* __restrict__ tris, int nt,
                                 const TriGeom* __restrict__ geo, const double* __restrict__ bary,
                                 const double* __restrict__ w, int n_gh, NodeW* __restrict__ out) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nt * n_gh) return;
    int t = idx / n_gh, g = idx % n_gh;
    double V[3][3];
    for (int v = 0; v < 3; v++) {
        int id = tris[3 * t + v];
        for (int c = 0; c < 3; c++) V[v][c] = coords[3 * id + c];
    }
    double b0 = bary[3 * g], b1 = bary[3 * g + 1], b2 = bary[3 * g + 2];
    NodeW o;
    o.x = b0 * V[0][0] + b1 * V[1][0] + b2 * V[2][0];
    o.y = b0 * V[0][1] + b1 * V[1][1] + b2 * V[2][1];
    o.z = b0 * V[0][2] + b1 * V[1][2] + b2 * V[2][2];
    o.w = geo[t].area * w[g];
    out[idx] = o;
}

int prep_mesh(MeshData& m, cudaStream_t s) {
    int threads = 128, blocks = (m.nt + threads - 1) / threads;
    prep_kernel<<<blocks, threads, 0, s>>>(m.d_coords, m.d_tris, m.nt, m.d_geo);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

int map_nodes(MeshData& m, int n_gh, cudaStream_t s) {
    if (m.nodes_rule == n_gh && m.d_nodes) return EBEM_OK;
    double bary[28 * 3], w[28];
    int rc = gh_composite(n_gh, 1, bary, w);
    if (rc) return fail(rc, "unsupported Gauss-Hammer rule");
    if (m.d_nodes) { cudaFree(m.d_nodes); m.d_nodes = nullptr; }
    double* d_tab = nullptr;
    EBEM_CUDA_TRY(cudaMalloc(&m.d_nodes, sizeof(NodeW) * (size_t)m.nt * n_gh));
    EBEM_CUDA_TRY(cudaMalloc(&d_tab, sizeof(double) * 4 * n_gh));
    EBEM_CUDA_TRY(cudaMemcpyAsync(d_tab, bary, sizeof(double) * 3 * n_gh, cudaMemcpyHostToDevice, s));
    EBEM_CUDA_TRY(cudaMemcpyAsync(d_tab + 3 * n_gh, w, sizeof(double) * n_gh, cudaMemcpyHostToDevice, s));
    int total = m.nt * n_gh, threads = 128;
    map_nodes_kernel<<<(total + threads - 1) / threads, threads, 0, s>>>(m.d_coords, m.d_tris, m.nt, m.d_geo, d_tab,
                                                                           d_tab + 3 * n_gh, n_gh, m.d_nodes);
    EBEM_CUDA_TRY(cudaGetLastError());
    EBEM_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(d_tab);
    m.nodes_rule = n_gh;
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// assembly

struct SAArgs {
    const TriGeom* geo;
    const NodeW* nodes;
    int N, n_gh;
    double velP, velS, dt, c4pirho;
    int lag0, nlag;
    int src0, nsrc;         // source rows [src0, src0 + nsrc) of the panel
    int diag_only;          // 1: only the diagonal pairs (i, i), i in the panel
    double* E;
    size_t ld;              // leading dimension (>= 3 nsrc)
    size_t ld_lag;          // doubles between consecutive lags
    int accumulate;
    unsigned long long* count;
};

__device__ __forceinline__ void store_block(const SAArgs& A, int q, int i, int j, const double b[6]) {
    // symmetric entries (11,12,13,22,23,33) -> column-major 3x3 at (3(i - src0), 3j)
    const size_t n3 = A.ld;
    double* base = A.E + (size_t)q * A.ld_lag + (3 * (size_t)j) * n3 + 3 * (size_t)(i - A.src0);
    const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};   // (r, c) column-major -> sym index
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            double v = b[map[3 * c + r]];
            if (A.accumulate) base[c * n3 + r] += v;
            else base[c * n3 + r] = v;
        }
}

__global__ void __launch_bounds__(128) sa_assemble_kernel(SAArgs A) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long NN = A.diag_only ? (long long)A.nsrc : (long long)A.nsrc * A.N;
    const bool valid = p < NN;
    const int i = valid ? A.src0 + (int)(p % A.nsrc) : A.src0;   // source (row block)
    const int j = A.diag_only ? i : (valid ? (int)(p / A.nsrc) : 0);   // field (column block)
    const TriGeom& F = A.geo[j];
    const TriGeom& Sg = A.geo[i];
    double v0 = F.ctr[0] - Sg.ctr[0], v1 = F.ctr[1] - Sg.ctr[1], v2 = F.ctr[2] - Sg.ctr[2];
    double d = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    double distMin = d - F.maxL - Sg.maxL;
    double distMax = d + F.maxL + Sg.maxL;
    // contiguous range of non-null lags inside [lag0, lag0 + nlag)
    int llo = -1, lhi = -2;
    for (int q = 0; q < A.nlag; q++) {
        int l = A.lag0 + q;
        if (lag_nonnull(l, A.velP, A.velS, A.dt, distMin, distMax)) {
            if (llo < 0) llo = l;
            lhi = l;
        }
    }
    if (A.count) {
        unsigned cnt = (valid && llo >= 0) ? (unsigned)(lhi - llo + 1) : 0u;
        unsigned tot = __reduce_add_sync(0xffffffffu, cnt);
        if ((threadIdx.x & 31) == 0 && tot) atomicAdd(A.count, (unsigned long long)tot);
    }
    if (!valid) return;
    const double zero[6] = {0, 0, 0, 0, 0, 0};
    if (llo < 0) {
        if (!A.accumulate)
            for (int q = 0; q < A.nlag; q++) store_block(A, q, i, j, zero);
        return;
    }
    if (!A.accumulate) {
        for (int l = A.lag0; l < llo; l++) store_block(A, l - A.lag0, i, j, zero);
        for (int l = lhi + 1; l < A.lag0 + A.nlag; l++) store_block(A, l - A.lag0, i, j, zero);
    }
    const int klo = max(1, llo - 1), khi = lhi + 1;
    // sliding window F_{k-2}, F_{k-1}, F_k; F_k = 0 for k <= 0
    double Fm2[6] = {0, 0, 0, 0, 0, 0}, Fm1[6] = {0, 0, 0, 0, 0, 0}, Fk[6];
    const double c4 = A.c4pirho;
    for (int k = klo; k <= khi; k++) {
        level_value(Fk, k, A.velP, A.velS, A.dt, F, A.nodes + (size_t)i * A.n_gh, A.n_gh);
        const int l = k - 1;                     // lag completed by F_k
        if (l >= llo && l <= lhi) {
            double b[6];
#pragma unroll
            for (int e = 0; e < 6; e++) {
                double prev = (l - 1 >= 1) ? Fm2[e] : 0.0;
                double v = ((Fk[e] + (-2.0) * Fm1[e]) + prev) / c4;
                b[e] = (fabs(v) < 1.0e-14) ? 0.0 : v;
            }
            store_block(A, l - A.lag0, i, j, b);
        }
#pragma unroll
        for (int e = 0; e < 6; e++) { Fm2[e] = Fm1[e]; Fm1[e] = Fk[e]; }
    }
}

int launch_sa_assemble(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                       double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count,
                       cudaStream_t s, int diag_only) {
    SAArgs A;
    A.geo = m.d_geo;
    A.nodes = m.d_nodes;
    A.N = m.nt;
    A.n_gh = n_gh;
    A.velP = P.velP;
    A.velS = P.velS;
    A.dt = P.dt;
    A.c4pirho = 4 * kPi * P.rho;
    A.lag0 = lag0;
    A.nlag = nlag;
    A.src0 = src0;
    A.nsrc = nsrc;
    A.diag_only = diag_only;
    A.E = d_E;
    A.ld = ld;
    A.ld_lag = ld_lag;
    A.accumulate = accumulate;
    A.count = d_count;
    long long NN = diag_only ? (long long)nsrc : (long long)nsrc * m.nt;
    int threads = 128;
    long long blocks = (NN + threads - 1) / threads;
    if (blocks > 0x7fffffffLL) return fail(EBEM_ERR_INVALID, "mesh too large for one launch");
    sa_assemble_kernel<<<(unsigned)blocks, threads, 0, s>>>(A);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

}  // namespace ebem
