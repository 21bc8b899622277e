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
// Work decomposition (B200 design, not the reference's): one warp per
// (source i, field j) pair walks the pair's time levels t_k = k dt once, in
// increasing order, with the lanes on the children of the outer nodes
// (sa_warp.cuh; level_pair below).  F(t_k), the combined kernel integral at
// one instant, depends on k only, so each level is evaluated once and
// E_l = F_{l+1} - 2 F_l + F_{l-1} is formed from three levels (the
// reference evaluates every instant three times, once per lag that uses
// it).  Dense outputs store the levels and write the blocks in a second,
// coalesced pass (sa_twopass.cu); the other modes write the blocks directly.
// A thread-per-pair kernel (sa_assemble_kernel) remains for builds with
// EBEM_SA_KERNEL=1.
#include "ebem_internal.h"

#include <algorithm>
#include <mutex>
#include "sa_pair.cuh"
#include "sa_warp.cuh"

#ifndef EBEM_SA_KERNEL
#define EBEM_SA_KERNEL 0    // 0: the warp-per-pair level kernel, 1: thread per pair
#endif
#ifndef EBEM_SA_TWOPASS
#define EBEM_SA_TWOPASS 1   // 1: dense assemblies store F(t_k) and emit the blocks in a second pass (sa_twopass.cu)
#endif

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
    static const int kSlotRule[MeshData::kNodeRules] = {1, 3, 7, 12, 19, 28};
    int slot = -1;
    for (int k = 0; k < MeshData::kNodeRules; k++)
        if (kSlotRule[k] == n_gh) slot = k;
    if (slot < 0) return fail(EBEM_ERR_INVALID, "unsupported Gauss-Hammer rule");
    if (NodeW* t = m.d_node_tables[slot]) {
        m.d_nodes = t;
        m.nodes_rule = n_gh;
        return EBEM_OK;
    }
    double bary[28 * 3], w[28];
    int rc = gh_composite(n_gh, 1, bary, w);
    if (rc) return fail(rc, "unsupported Gauss-Hammer rule");
    // the table enters the cache only once the mapping has finished, so a
    // failed call leaves no half-built table behind
    NodeW* table = nullptr;
    double* d_tab = nullptr;
    if (cudaMalloc(&table, sizeof(NodeW) * (size_t)m.nt * n_gh) != cudaSuccess ||
        cudaMalloc(&d_tab, sizeof(double) * 4 * n_gh) != cudaSuccess) {
        cudaGetLastError();
        if (table) cudaFree(table);
        return fail(EBEM_ERR_NOMEM, "outer-node table allocation failed");
    }
    cudaError_t e = cudaMemcpyAsync(d_tab, bary, sizeof(double) * 3 * n_gh, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_tab + 3 * n_gh, w, sizeof(double) * n_gh, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        int total = m.nt * n_gh, threads = 128;
        map_nodes_kernel<<<(total + threads - 1) / threads, threads, 0, s>>>(m.d_coords, m.d_tris, m.nt, m.d_geo, d_tab,
                                                                               d_tab + 3 * n_gh, n_gh, table);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_tab);
    if (e != cudaSuccess) {
        cudaFree(table);
        return fail(EBEM_ERR_CUDA, std::string("outer-node mapping: ") + cudaGetErrorString(e));
    }
    m.d_node_tables[slot] = table;
    m.d_nodes = table;
    m.nodes_rule = n_gh;
    return EBEM_OK;
}

int map_nodes_composite(MeshData& m, int n_gh, int n_sub, cudaStream_t s) {
    if (n_sub == 1) return map_nodes(m, n_gh, s);
    const int key = n_gh * 4096 + n_sub;
    for (int k = 0; k < MeshData::kCompRules; k++)
        if (m.d_comp_tables[k] && m.comp_key[k] == key) {
            m.d_nodes = m.d_comp_tables[k];
            m.nodes_rule = n_gh * n_sub;
            return EBEM_OK;
        }
    int slot = -1;
    for (int k = 0; k < MeshData::kCompRules && slot < 0; k++)
        if (!m.d_comp_tables[k]) slot = k;
    if (slot < 0) return fail(EBEM_ERR_INVALID, "too many composite outer rules cached on one mesh");
    if (n_sub < 1 || n_sub > 1024) return fail(EBEM_ERR_INVALID, "composite rule: n_sub out of range");
    const int nn = n_gh * n_sub;
    std::vector<double> bary(3 * (size_t)nn), w((size_t)nn), wb(n_gh);
    int rc = gh_composite(n_gh, n_sub, bary.data(), wb.data());
    if (rc) return fail(rc, "unsupported composite Gauss-Hammer rule (n_sub must be a square)");
    for (int q = 0; q < n_sub; q++)
        for (int g = 0; g < n_gh; g++) w[(size_t)q * n_gh + g] = wb[g];
    NodeW* table = nullptr;
    double* d_tab = nullptr;
    if (cudaMalloc(&table, sizeof(NodeW) * (size_t)m.nt * nn) != cudaSuccess ||
        cudaMalloc(&d_tab, sizeof(double) * 4 * (size_t)nn) != cudaSuccess) {
        cudaGetLastError();
        if (table) cudaFree(table);
        return fail(EBEM_ERR_NOMEM, "outer-node table allocation failed");
    }
    cudaError_t e = cudaMemcpyAsync(d_tab, bary.data(), sizeof(double) * 3 * nn, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_tab + 3 * (size_t)nn, w.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const long long total = (long long)m.nt * nn;
        const int threads = 128;
        map_nodes_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(
            m.d_coords, m.d_tris, m.nt, m.d_geo, d_tab, d_tab + 3 * (size_t)nn, nn, table);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_tab);
    if (e != cudaSuccess) {
        cudaFree(table);
        return fail(EBEM_ERR_CUDA, std::string("outer-node mapping: ") + cudaGetErrorString(e));
    }
    m.d_comp_tables[slot] = table;
    m.comp_key[slot] = key;
    m.d_nodes = table;
    m.nodes_rule = nn;
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
    const int2* pairs;      // optional explicit (source, field) list (npairs entries)
    long long npairs;
    // banded output (instead of E): pair p = (i - src0) N + j owns the blocks
    // [boff[p], boff[p+1]) of Eb, one per lag of its band starting at blo[p],
    // 6 symmetric entries (11,12,13,22,23,33) each
    double* Eb = nullptr;
    const long long* boff = nullptr;
    const int* blo = nullptr;
    // level output (instead of E): field columns [j0, j0 + nj) of the panel;
    // F(t_k) of pair (i, j) at Fout[(((j - j0) KL + k - kbase) nsrc + i - src0) 6 + e]
    // for every level it needs, its non-null lags (llo, lhi) at band[(j - j0) nsrc + i - src0]
    double* Fout = nullptr;
    int2* band = nullptr;
    int j0 = 0, nj = 0, kbase = 0, KL = 0;
    // level output restricted to one class of a per-(pair, lag) class array:
    // cls[(j N + i) nlag + l - lag0] (fields j, sources i); only the levels
    // that lags of class cls_want use are computed, only those lags counted
    const unsigned char* cls = nullptr;
    int cls_want = -1;
    // direct dense output into a buffer already zeroed: only the band's blocks are written
    int zeros_written = 0;
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

__device__ __forceinline__ void store_entry(const SAArgs& A, int q, int i, int j, int e, double v) {
    // entry e = 3 c + r of the column-major 3x3 block at (3(i - src0), 3j)
    const int c = e / 3, r = e - 3 * c;
    double* dst = A.E + (size_t)q * A.ld_lag + (3 * (size_t)j + c) * A.ld + 3 * (size_t)(i - A.src0) + r;
    if (A.accumulate) *dst += v;
    else *dst = v;
}


// ---------------------------------------------------------------------------
// Level pass of the two-pass assembly, outer nodes in groups.
//
// One warp per (source, field) pair walks the pair's time levels with the
// schedule of sa_warp.cuh (lane = child of one outer node; per level the
// per-child decision phase, the whole-range moments, the warp-wide list of
// Gauss-Legendre nodes and one warp reduction), for the children of at most
// 10 outer nodes at a time, so composite outer rules of any size
// (GaussHammerComposite.m) run group after group with each group's per-level
// sums added in shared memory.  After the levels of a chunk, one lane per
// level forms F(t_k) (the rotation to global axes) and stores it for the
// emission pass.  With a per-(pair, lag) class array only the levels used by
// lags of the wanted class are walked.
//
// Two alternative schedules were measured and not kept.  Compacted (child,
// level) items, 32 per round, each lane on its own item: sphere of 1280
// triangles 224 ms per step against 186 ms (ncu: 9 % fewer warp
// instructions, but more instruction-fetch stalls, the items of a round
// taking more distinct branches than the children of one level).  Groups
// of 10 consecutive outer nodes of up to three pairs of one field column
// (30 lanes busy instead of 21 with the 7-node rule, per-pair level sums):
// 165.9 ms against 167.2 ms with the 7-node rule, 104.7 against 135.4 ms
// with the 3-node rule; the children of different pairs take more distinct
// branches per pass than those of one pair, which cancels most of the lanes
// gained, and the results then depend on how pairs fall into groups (a
// source-row sub-panel no longer reproduces the full assembly bit for bit).

// Levels per chunk (per-level sums in shared memory).  24 rather than 48:
// the 4 warps' sums take 5.4 KB less shared memory per block, which leaves
// the 3 blocks per SM a larger L1 for the kernel's stack and loads (sphere
// N=1280, L=40: 163.5 -> 160.2 ms per step, two A/B rounds on one box; 16
// levels gave 163.2 ms: the chunks' set-up then costs what L1 gains).
#ifndef EBEM_LEVEL_KC
#define EBEM_LEVEL_KC 24
#endif
#ifndef EBEM_LEVEL_WPB
#define EBEM_LEVEL_WPB 4
#endif
#ifndef EBEM_LEVEL_MINB
#define EBEM_LEVEL_MINB 3
#endif
#ifndef EBEM_LEVEL_SKIP_IDLE
#define EBEM_LEVEL_SKIP_IDLE 1   // 1: levels at which no child works skip the decision and node phases
#endif
constexpr int kGroupNodes = 10;  // outer nodes per group: 30 children on 32 lanes

struct LevelShared {
    WarpShared<1> W;
    double acc[7][EBEM_LEVEL_KC];
    double carry[2][6];          // direct output: F of the two levels before the chunk
};

// Whether level k is used by a lag of the wanted class (lags k-1, k, k+1 of
// the pair's non-null range [llo, lhi]).
EBEM_DI bool level_wanted(const SAArgs& A, const unsigned char* cls, int k, int llo, int lhi) {
    if (!cls) return true;
    for (int l = max(k - 1, llo); l <= min(k + 1, lhi); l++)
        if (cls[l - A.lag0] == A.cls_want) return true;
    return false;
}

// Pair p of the launch: (source i, field j); its record in A.band and its
// levels in A.Fout (record rec, level k at (rec + (k - kbase) kstride) 6):
// field columns of a panel (rec = (j - j0) KL nsrc + i - src0, kstride =
// nsrc) or an explicit pair list (rec = p KL, kstride = 1).
// The dynamic shared memory opt-in of a kernel, before every launch that is
// not being captured: it belongs to the context, which a caller may have
// reset since the last call; a captured launch relies on the uncaptured one
// before it (the batch plan runs its launch before capturing it).
template <class K>
static int opt_in_smem(K kernel, size_t smem, cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) return EBEM_OK;
    EBEM_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return EBEM_OK;
}

template <bool MIXED>
__device__ __forceinline__ void level_pair(const SAArgs& A, LevelShared& Ls, const double* glx, const double* glw,
                                           long long p, int i, int j, int lane, unsigned long long& my_count) {
    WarpShared<1>& W = Ls.W;
    const TriGeom& F = A.geo[j];
    const TriGeom& Sg = A.geo[i];
    int llo = -1, lhi = -2;
    long long bbase = 0;
    if (A.Eb) {
        // banded output: the band comes from the structure pass, so writes stay in the pair's blocks
        const long long pb = (long long)(i - A.src0) * A.N + j;
        bbase = A.boff[pb];
        const int nb = (int)(A.boff[pb + 1] - bbase);
        if (nb > 0) {
            llo = A.blo[pb];
            lhi = llo + nb - 1;
        }
    } else {
        pair_band(F, Sg, A.velP, A.velS, A.dt, A.lag0, A.nlag, &llo, &lhi);
    }
    const long long brec = A.pairs ? p : (long long)(j - A.j0) * A.nsrc + (i - A.src0);
    const long long frec = A.pairs ? p * A.KL : (long long)(j - A.j0) * A.KL * A.nsrc + (i - A.src0);
    const long long kstride = A.pairs ? 1 : A.nsrc;
    if (A.band && lane == 0) A.band[brec] = make_int2(llo, lhi);
    // direct dense output: the zeros of the window's lags outside the band
    const bool dense = !A.Fout && !A.Eb;
    if (dense && !A.accumulate && !A.zeros_written) {
        for (int idx = lane; idx < A.nlag * 9; idx += 32) {
            const int q = idx / 9, e = idx - 9 * q, l = A.lag0 + q;
            if (llo < 0 || l < llo || l > lhi) store_entry(A, q, i, j, e, 0.0);
        }
    }
    if (llo < 0) return;
    if (!A.Fout && lane < 12) (&Ls.carry[0][0])[lane] = 0.0;
    const unsigned char* cls = A.cls ? A.cls + ((long long)j * A.N + i) * A.nlag : nullptr;
    if (cls) {
        int n = 0;
        for (int l = llo; l <= lhi; l++) n += (cls[l - A.lag0] == A.cls_want);
        if (lane == 0) my_count += (unsigned long long)n;
        if (n == 0) return;
    } else if (lane == 0) {
        my_count += (unsigned long long)(lhi - llo + 1);
    }
    const double vp2 = A.velP * A.velP, vs2 = A.velS * A.velS, den = vp2 * vs2;
    const double k1 = 1.0 / vp2, k5 = (vp2 + vs2) / den, k6 = (vp2 - vs2) / den;
    const int ngroups = (A.n_gh + kGroupNodes - 1) / kGroupNodes;
    const int klo = max(1, llo - 1), khi = lhi + 1;
    const int slot = lane;
    LaneChild Cu;
    bool hasmom = false, is_stat = false;
    for (int kc0 = klo; kc0 <= khi; kc0 += EBEM_LEVEL_KC) {
        const int kc1 = min(khi, kc0 + EBEM_LEVEL_KC - 1), nk = kc1 - kc0 + 1;
        for (int x = lane; x < 7 * EBEM_LEVEL_KC; x += 32) (&Ls.acc[0][0])[x] = 0.0;
        for (int grp = 0; grp < ngroups; grp++) {
            const int g0 = kGroupNodes * grp, gn = min(kGroupNodes, A.n_gh - g0);
            if (ngroups > 1 || kc0 == klo) {
                // children of outer nodes [g0, g0 + gn): slot = 3 (g - g0) + child
                __syncwarp();
                Cu.live = false;
                Cu.zeta = 0.0; Cu.sigma = 0.0; Cu.dMIN = 0.0; Cu.w = 0.0;
                hasmom = false;
                is_stat = false;
                const int g = g0 + slot / 3, c = slot - 3 * (slot / 3);
                if (slot < 3 * gn) {
                    NodeW sp = A.nodes[(size_t)i * A.n_gh + g];
                    NodeGeo G;
                    node_geo(G, sp, F);
                    Cu.zeta = G.zeta;
                    Cu.sigma = G.sigma;
                    Cu.dMIN = G.dMIN;
                    Cu.w = sp.w;
                    if (node_child_e(Cu.g, G, c)) {
                        Cu.live = true;
                        m_sincos(Cu.g.gamma, &Cu.sg, &Cu.cg);
                    }
                }
                if (Cu.live) {
                    const ChildE& gg = Cu.g;
                    LevelCtx L0;
                    L0.k5 = k5;
                    L0.k6 = k6;
                    const W4 w0 = origin_weights(Cu.zeta, L0);
                    W.w0[0][slot] = w0.sc;
                    W.w0[1][slot] = w0.in;
                    W.w0[2][slot] = w0.mx;
                    W.w0[3][slot] = w0.zz;
                    W.amax[slot] = gg.amax;
                    W.F[slot] = gg.F;
                    W.cbp[slot] = gg.cb * gg.ct + gg.sb * gg.st;     // cos(beta - theta_V1)
                    W.sbp[slot] = gg.sb * gg.ct - gg.cb * gg.st;     // sin(beta - theta_V1)
                    W.zeta[slot] = Cu.zeta;
                    W.zs[slot] = Cu.zeta * Cu.sigma;
                    W.scale[slot] = Cu.w * gg.sgnC;
                    if (MIXED) {
                        W.Ff[slot] = (float)W.F[slot];
                        W.cbpf[slot] = (float)W.cbp[slot];
                        W.sbpf[slot] = (float)W.sbp[slot];
                        W.zetaf[slot] = (float)W.zeta[slot];
                        W.zsf[slot] = (float)W.zs[slot];
                        W.scalef[slot] = (float)W.scale[slot];
                    }
                }
            }
            __syncwarp();
            for (int k = kc0; k <= kc1; k++) {
                if (!level_wanted(A, cls, k, llo, lhi)) continue;
                const double t = k * A.dt;
                LevelCtx L;
                L.t2 = t * t;
                L.RP = A.velP * t;
                L.RS = A.velS * t;
                L.k1 = k1;
                L.k5 = k5;
                L.k6 = k6;
                double S = 0.0, T[6] = {0, 0, 0, 0, 0, 0};
                Piece pc[3];
                int np = 0, nsubs[3], ngs[3];
                double hs[3];
                int nn = 0;
                // decision phase (per child)
                int type = T_NONE;
                double rhoP = -1.0, rhoS = -1.0;
                if (Cu.live && !is_stat) type = classify(Cu.zeta, L.RP, L.RS, Cu.dMIN, rhoP, rhoS);
                // no child at work at this level (about half the levels of a pair's
                // band: the null test's distance bounds are conservative): F is the
                // sum of the static children, zero when there are none
                if (EBEM_LEVEL_SKIP_IDLE && __ballot_sync(0xffffffffu, type != T_NONE) == 0u) {
                    if (__ballot_sync(0xffffffffu, is_stat) != 0u) {
                        double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                        if (is_stat) {
#pragma unroll
                            for (int e = 0; e < 7; e++) v[e] = W.sv[e][slot];
                        }
                        const double tot = warp_reduce_scatter8(v, lane);
                        const int e = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
                        if ((lane & 3) == 0 && e < 7) Ls.acc[e][k - kc0] += tot;
                    }
                    continue;
                }
                AccE Ac = {0, 0, 0, 0, 0, 0, 0};
                int full = 0;
                if (type != T_NONE) {
                    W4 w0;
                    w0.sc = W.w0[0][slot];
                    w0.in = W.w0[1][slot];
                    w0.mx = W.w0[2][slot];
                    w0.zz = W.w0[3][slot];
                    child_decide(Ac, pc, np, full, Cu, L, rhoP, rhoS, type, w0, W.amax[slot]);
                }
                // whole-range moments, computed by the whole warp once per child
                const bool need = full && !hasmom;
                unsigned mm = __ballot_sync(0xffffffffu, need);
                while (mm) {
                    const int b = __ffs(mm) - 1;
                    mm &= mm - 1;
                    const double Fb = __shfl_sync(0xffffffffu, Cu.g.F, b), cbb = __shfl_sync(0xffffffffu, Cu.g.cb, b);
                    const double sbb = __shfl_sync(0xffffffffu, Cu.g.sb, b), zb = __shfl_sync(0xffffffffu, Cu.zeta, b);
                    const double s1b = __shfl_sync(0xffffffffu, Cu.g.s1, b), s0b = __shfl_sync(0xffffffffu, Cu.g.s0, b);
                    double m[16];
                    moment_share(m, Fb, cbb, sbb, zb, s1b, s0b, lane, glx, glw);
                    m[14] = 0.0;
                    m[15] = 0.0;
                    const double tot = warp_reduce_scatter16(m, lane);
                    const int e = scatter16_index(lane);
                    if (!(lane & 1) && e < 14) W.mom[e][b] = tot;
                }
                __syncwarp();
                if (need) hasmom = true;
                const double zs = Cu.zeta * Cu.sigma;
                if (full & 1) apply_moments(Ac, W, slot, true, L, zs);
                if (full & 2) apply_moments(Ac, W, slot, false, L, zs);
                if (type != T_NONE) {
                    double Sc = 0.0, Tc[6] = {0, 0, 0, 0, 0, 0};
                    child_to_plane(Sc, Tc, Ac, Cu.g, Cu.w * Cu.g.sgnC);
                    S += Sc;
#pragma unroll
                    for (int e = 0; e < 6; e++) T[e] += Tc[e];
                    // inside the S front with its whole edge (only the full S piece):
                    // level-independent from now on (the fronts only grow)
                    if (type == T_SP_SP && full == 2 && np == 0) {
                        W.sv[0][slot] = Sc;
#pragma unroll
                        for (int e = 0; e < 6; e++) W.sv[1 + e][slot] = Tc[e];
                        is_stat = true;
                    }
                } else if (is_stat) {
                    S += W.sv[0][slot];
#pragma unroll
                    for (int e = 0; e < 6; e++) T[e] += W.sv[1 + e][slot];
                }
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    nsubs[q] = 0;
                    ngs[q] = 10;
                    hs[q] = 0.0;
                    if (q < np) {
                        double len = pc[q].shi - pc[q].slo;
                        int ns = (int)ceil(len * (1.0 / EBEM_EDGE_H));
                        ns = max(1, min(ns, 4096));
                        // nodes per sub-piece: 6 up to length 1/4, 8 up to 1/2 (gl6_x)
                        if (EBEM_GL_ADAPT && ns == 1) ngs[q] = len <= 0.25 ? 6 : (len <= 0.5 ? 8 : 10);
                        nsubs[q] = ns;
                        hs[q] = len / ns;
                        nn += ngs[q] * ns;
                    }
                }
                // partial edge pieces of all children -> per-warp list
                int totp, totn;
                int pb = warp_excl_scan(np, lane, totp);
                int o = warp_excl_scan(nn, lane, totn);
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    if (q < np) {
                        W.slo[pb] = pc[q].slo;
                        W.h[pb] = hs[q];
                        W.off[pb] = o;
                        W.who[pb] = slot | (pc[q].pterm ? 64 : 0) | (((ngs[q] - 6) >> 1) << 7);
                        o += ngs[q] * nsubs[q];
                        pb++;
                    }
                }
                if (lane == 31) W.off[totp] = totn;
                __syncwarp();
                // all lanes: Gauss-Legendre nodes of the list, plane frame
                int pp = 0;
                if (MIXED) {
                    float Sf = 0.0f, Tf[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                    const float fk1 = (float)L.k1, ft2 = (float)L.t2, fk5 = (float)L.k5, fk6 = (float)L.k6;
                    for (int idx = lane; idx < totn; idx += 32) {
                        while (idx >= W.off[pp + 1]) pp++;
                        const int who = W.who[pp], cl = who & 63, code = who >> 7;
                        const int u = idx - W.off[pp], sub = code == 2 ? u / 10 : 0;
                        const int q = u - (6 + 2 * code) * sub + (code == 0 ? 0 : (code == 1 ? 6 : 14));
                        const double h = W.h[pp];
                        const double s = W.slo[pp] + (sub + 0.5) * h + 0.5 * h * glx[q];
                        edge_node_f32(Sf, Tf, s, (float)(0.5 * h * glw[q]), W.Ff[cl], W.cbpf[cl], W.sbpf[cl],
                                      W.zetaf[cl], W.zsf[cl], W.scalef[cl], (who & 64) != 0, fk1, ft2, fk5, fk6);
                    }
                    S += (double)Sf;
#pragma unroll
                    for (int e = 0; e < 6; e++) T[e] += (double)Tf[e];
                    totn = 0;    // the FP64 loop below has nothing left to do
                }
                for (int idx = lane; idx < totn; idx += 32) {
                    while (idx >= W.off[pp + 1]) pp++;
                    const int who = W.who[pp], cl = who & 63, code = who >> 7;
                    const int u = idx - W.off[pp], sub = code == 2 ? u / 10 : 0;
                    const int q = u - (6 + 2 * code) * sub + (code == 0 ? 0 : (code == 1 ? 6 : 14));
                    const double h = W.h[pp];
                    const double s = W.slo[pp] + (sub + 0.5) * h + 0.5 * h * glx[q];
                    double sech, th;
                    Rad v;
                    edge_point(s, W.F[cl], W.zeta[cl], sech, th, v);
                    const double cbq = W.cbp[cl], sbq = W.sbp[cl];
                    const double cq = th * cbq + sech * sbq, sq = sech * cbq - th * sbq;
                    W4 w = weigh(v, (who & 64) != 0, L);
                    const double f = 0.5 * h * glw[q] * sech * W.scale[cl];
                    const double fin = f * w.in, fmx = -W.zs[cl] * f * w.mx;
                    S += f * w.sc;
                    T[0] += fin * cq * cq;
                    T[1] += fin * sq * cq;
                    T[2] += fin * sq * sq;
                    T[3] += fmx * cq;
                    T[4] += fmx * sq;
                    T[5] += f * w.zz;
                }
                __syncwarp();
                // warp sums; lane scatter8_lane(e) holds entry e (S, T11, T12, T22, T13, T23, T33)
                double v[8] = {S, T[0], T[1], T[2], T[3], T[4], T[5], 0.0};
                const double tot = warp_reduce_scatter8(v, lane);
                const int e = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
                if ((lane & 3) == 0 && e < 7) Ls.acc[e][k - kc0] += tot;
            }
            __syncwarp();
        }
        // F(t_k) = (S I + C^T M C) / 2 in global axes, one lane per level
        for (int kl = lane; kl < nk; kl += 32) {
            const int k = kc0 + kl;
            if (!level_wanted(A, cls, k, llo, lhi)) continue;
            const double S = Ls.acc[0][kl];
            double T[6];
#pragma unroll
            for (int e = 0; e < 6; e++) T[e] = Ls.acc[1 + e][kl];
            double M[3][3] = {{T[0], T[1], T[3]}, {T[1], T[2], T[4]}, {T[3], T[4], T[5]}};
            const double* Cm = F.C;
            double MC[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int cc = 0; cc < 3; cc++)
                    MC[r][cc] = M[r][0] * Cm[cc] + M[r][1] * Cm[3 + cc] + M[r][2] * Cm[6 + cc];
            double Rm[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int cc = r; cc < 3; cc++)
                    Rm[r][cc] = Cm[r] * MC[0][cc] + Cm[3 + r] * MC[1][cc] + Cm[6 + r] * MC[2][cc];
            const double Fk[6] = {0.5 * (S + Rm[0][0]), 0.5 * Rm[0][1], 0.5 * Rm[0][2],
                                  0.5 * (S + Rm[1][1]), 0.5 * Rm[1][2], 0.5 * (S + Rm[2][2])};
            if (A.Fout) {
                double2* dst = reinterpret_cast<double2*>(A.Fout + (frec + (k - A.kbase) * kstride) * 6);
                dst[0] = make_double2(Fk[0], Fk[1]);
                dst[1] = make_double2(Fk[2], Fk[3]);
                dst[2] = make_double2(Fk[4], Fk[5]);
            } else {
#pragma unroll
                for (int e = 0; e < 6; e++) Ls.acc[e][kl] = Fk[e];     // this lane's level only
            }
        }
        __syncwarp();
        if (!A.Fout) {
            // direct output: E_l = (F_{l+1} - 2 F_l + F_{l-1}) / (4 pi rho) for the
            // lags l = k - 1 completed by the chunk's levels k, clean-up |x| < 1e-14
            // (calcMatrixSubBlock.m:15,23,111; calcMatrixBlock.m:77); F_0 = 0
            const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
            for (int kl = lane; kl < nk; kl += 32) {
                const int k = kc0 + kl, l = k - 1;
                if (l < llo || l > lhi) continue;
                double b[6];
#pragma unroll
                for (int e = 0; e < 6; e++) {
                    const double f1 = Ls.acc[e][kl];
                    const double f0 = (k - 1 < 1) ? 0.0 : (kl >= 1 ? Ls.acc[e][kl - 1] : Ls.carry[1][e]);
                    const double fm = (k - 2 < 1) ? 0.0 : (kl >= 2 ? Ls.acc[e][kl - 2] : Ls.carry[kl][e]);
                    const double v = ((f1 + (-2.0) * f0) + fm) / A.c4pirho;
                    b[e] = (fabs(v) < 1.0e-14) ? 0.0 : v;
                }
                if (A.Eb) {
#pragma unroll
                    for (int e = 0; e < 6; e++) A.Eb[(bbase + (l - llo)) * 6 + e] = b[e];
                } else {
#pragma unroll
                    for (int e9 = 0; e9 < 9; e9++) store_entry(A, l - A.lag0, i, j, e9, b[map[e9]]);
                }
            }
            __syncwarp();
            if (lane < 6) {
                const double c1 = Ls.carry[1][lane];
                Ls.carry[0][lane] = (nk >= 2) ? Ls.acc[lane][nk - 2] : c1;
                Ls.carry[1][lane] = Ls.acc[lane][nk - 1];
            }
            __syncwarp();
        }
    }
}

template <int WPB, int MINB, bool MIXED>
__global__ void __launch_bounds__(32 * WPB, MINB) sa_level_kernel(SAArgs A) {
    extern __shared__ __align__(16) unsigned char level_smem[];
    LevelShared* Lsh = reinterpret_cast<LevelShared*>(level_smem);
    __shared__ double gt[48];          // Gauss-Legendre nodes and weights (gl_table_entry)
    __shared__ unsigned long long blk_count;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    LevelShared& Ls = Lsh[wib];
    if (threadIdx.x < 24) gl_table_entry(threadIdx.x, gt[threadIdx.x], gt[24 + threadIdx.x]);
    if (threadIdx.x == 0) blk_count = 0;
    __syncthreads();
    const long long NP = A.pairs ? A.npairs : A.diag_only ? (long long)A.nsrc : (long long)A.nsrc * A.nj;
    const long long nwarps = (long long)gridDim.x * WPB;
    unsigned long long my_count = 0;
    for (long long p = (long long)blockIdx.x * WPB + wib; p < NP; p += nwarps) {
        int i, j;
        if (A.pairs) {
            const int2 pj = A.pairs[p];
            i = pj.x;
            j = pj.y;
        } else {
            i = A.src0 + (int)(p % A.nsrc);
            j = A.diag_only ? i : A.j0 + (int)(p / A.nsrc);
        }
        level_pair<MIXED>(A, Ls, gt, gt + 24, p, i, j, lane, my_count);
    }
    if (A.count) {
        if (lane == 0 && my_count) atomicAdd(&blk_count, my_count);
        __syncthreads();
        if (threadIdx.x == 0 && blk_count) atomicAdd(A.count, blk_count);
    }
}

template <int WPB, int MINB, bool MIXED>
static int launch_level(const SAArgs& A, long long NN, int device, cudaStream_t s) {
    const size_t smem = sizeof(LevelShared) * WPB;
    if (int rc = opt_in_smem(sa_level_kernel<WPB, MINB, MIXED>, smem, s)) return rc;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    long long want = (NN + WPB - 1) / WPB;
    long long cap = (long long)sms * MINB * 16;
    unsigned blocks = (unsigned)(want < cap ? want : cap);
    if (blocks == 0) blocks = 1;
    sa_level_kernel<WPB, MINB, MIXED><<<blocks, 32 * WPB, smem, s>>>(A);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}
int launch_sa_assemble(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                       double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count,
                       cudaStream_t s, int diag_only, int mixed, const int2* pairs, long long npairs) {
    if (EBEM_SA_TWOPASS && EBEM_SA_KERNEL == 0 && !diag_only && !pairs)
        return launch_sa_twopass(m, P, n_gh, lag0, nlag, src0, nsrc, d_E, ld, ld_lag, accumulate, d_count, mixed, s);
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
    A.pairs = pairs;
    A.npairs = npairs;
    A.j0 = 0;
    A.nj = m.nt;
    long long NN = diag_only ? (long long)nsrc : (long long)nsrc * m.nt;
    if (pairs) NN = npairs;
    if (EBEM_SA_KERNEL == 0)
        return mixed ? launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, true>(A, NN, m.device, s)
                     : launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, false>(A, NN, m.device, s);
    if (pairs || mixed) return fail(EBEM_ERR_INVALID, "pair lists and mixed precision need the warp kernel");
    int threads = 128;
    long long blocks = (NN + threads - 1) / threads;
    if (blocks > 0x7fffffffLL) return fail(EBEM_ERR_INVALID, "mesh too large for one launch");
    sa_assemble_kernel<<<(unsigned)blocks, threads, 0, s>>>(A);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

// Level output for the two-pass assembly (sa_twopass.cu): F(t_k) of the pairs
// (sources [src0, src0 + nsrc), fields [j0, j0 + nj)) at every level their
// non-null lags in [lag0, lag0 + nlag) need, and those lags.
int launch_sa_fwarp(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc, int j0,
                    int nj, int kbase, int KL, double* d_F, int2* d_band, unsigned long long* d_count, int mixed,
                    cudaStream_t s, const unsigned char* cls, int cls_want) {
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
    A.diag_only = 0;
    A.E = nullptr;
    A.ld = 0;
    A.ld_lag = 0;
    A.accumulate = 0;
    A.count = d_count;
    A.pairs = nullptr;
    A.npairs = 0;
    A.Fout = d_F;
    A.band = d_band;
    A.j0 = j0;
    A.nj = nj;
    A.kbase = kbase;
    A.KL = KL;
    A.cls = cls;
    A.cls_want = cls_want;
    const long long NN = (long long)nsrc * nj;
    return mixed ? launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, true>(A, NN, m.device, s)
                 : launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, false>(A, NN, m.device, s);
}

// Blocks of an explicit list of (source, field) pairs at every lag [0, nlag)
// with the outer rule in m.d_nodes (n_gh nodes per triangle, composite or
// not): out[(p nlag + l) 6 + e], the 6 symmetric entries (11, 12, 13, 22, 23,
// 33) of E_l, zero outside the pair's non-null lags.
__global__ void pair_emit_kernel(const double* __restrict__ Fb, const int2* __restrict__ band, long long np, int nlag,
                                 int KL, double c4, double* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np * nlag) return;
    const long long p = t / nlag;
    const int l = (int)(t - p * nlag);
    const int2 b = band[p];
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (b.x >= 0 && l >= b.x && l <= b.y) {
        // level k of pair p at (p KL + k - 1) 6 (kbase = 1); F_0 = 0
        const double* rec = Fb + p * KL * 6;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            const double a1 = rec[l * 6 + e];
            const double a0 = (l >= 1) ? rec[(l - 1) * 6 + e] : 0.0;
            const double am = (l >= 2) ? rec[(l - 2) * 6 + e] : 0.0;
            const double x = ((a1 + (-2.0) * a0) + am) / c4;
            v[e] = (fabs(x) < 1.0e-14) ? 0.0 : x;
        }
    }
#pragma unroll
    for (int e = 0; e < 6; e++) out[t * 6 + e] = v[e];
}

int launch_sa_pair_blocks(const MeshData& m, const PhysParams& P, int n_gh, const int2* d_pairs, long long npairs,
                          int nlag, double* d_out, cudaStream_t s) {
    if (npairs <= 0) return EBEM_OK;
    const int KL = nlag;                          // levels 1 .. nlag
    const long long chunk = std::max<long long>(1, ((long long)256 << 20) / ((long long)KL * 48 + 8));
    const long long np0 = std::min(npairs, chunk);
    double* Fb = nullptr;
    if (ws_malloc(&Fb, (size_t)np0 * KL * 48 + (size_t)np0 * sizeof(int2), s) != cudaSuccess)
        return fail(EBEM_ERR_NOMEM, "pair-block workspace allocation failed");
    int2* band = reinterpret_cast<int2*>(reinterpret_cast<unsigned char*>(Fb) + (size_t)np0 * KL * 48);
    int rc = EBEM_OK;
    for (long long q0 = 0; q0 < npairs && rc == EBEM_OK; q0 += np0) {
        const long long nq = std::min(np0, npairs - q0);
        SAArgs A;
        A.geo = m.d_geo;
        A.nodes = m.d_nodes;
        A.N = m.nt;
        A.n_gh = n_gh;
        A.velP = P.velP;
        A.velS = P.velS;
        A.dt = P.dt;
        A.c4pirho = 4 * kPi * P.rho;
        A.lag0 = 0;
        A.nlag = nlag;
        A.src0 = 0;
        A.nsrc = m.nt;
        A.diag_only = 0;
        A.E = nullptr;
        A.ld = 0;
        A.ld_lag = 0;
        A.accumulate = 0;
        A.count = nullptr;
        A.pairs = d_pairs + q0;
        A.npairs = nq;
        A.Fout = Fb;
        A.band = band;
        A.j0 = 0;
        A.nj = 0;
        A.kbase = 1;
        A.KL = KL;
        rc = launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, false>(A, nq, m.device, s);
        if (rc) break;
        const long long nt = nq * nlag;
        pair_emit_kernel<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(Fb, band, nq, nlag, KL, 4 * kPi * P.rho,
                                                                     d_out + q0 * nlag * 6);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, std::string("pair blocks: ") + cudaGetErrorString(e));
    }
    ws_free(Fb, s);
    return rc;
}

// Banded output: all lags [0, L) of every pair, written into the band
// layout that band_structure() built (only the warp kernel has this mode).
int launch_sa_assemble_banded(const MeshData& m, const PhysParams& P, int n_gh, int L, double* d_Eb,
                              const long long* d_boff, const int* d_blo, int mixed, cudaStream_t s) {
    SAArgs A;
    A.geo = m.d_geo;
    A.nodes = m.d_nodes;
    A.N = m.nt;
    A.n_gh = n_gh;
    A.velP = P.velP;
    A.velS = P.velS;
    A.dt = P.dt;
    A.c4pirho = 4 * kPi * P.rho;
    A.lag0 = 0;
    A.nlag = L;
    A.src0 = 0;
    A.nsrc = m.nt;
    A.diag_only = 0;
    A.E = nullptr;
    A.ld = 0;
    A.ld_lag = 0;
    A.accumulate = 0;
    A.count = nullptr;
    A.pairs = nullptr;
    A.npairs = 0;
    A.Eb = d_Eb;
    A.boff = d_boff;
    A.blo = d_blo;
    A.j0 = 0;
    A.nj = m.nt;
    const long long NN = (long long)m.nt * m.nt;
    return mixed ? launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, true>(A, NN, m.device, s)
                 : launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, false>(A, NN, m.device, s);
}

// ---------------------------------------------------------------------------
// Assembly without device allocations (ebem_assemble_sa_noalloc).
//
// The ordinary assembly allocates two small device buffers of its own: the
// mapped outer nodes of the mesh (cached per rule) and, when the caller asks
// for the non-null count, an 8-byte counter.  This variant keeps both in one
// statically allocated device array, so that a call allocates nothing.  The
// array belongs to every GPU that loads the library until the process exits.
//
// Layout (bytes): [0, 8) counter, zeroed by each call that counts; from
// byte 256 on, the mapped node table, rewritten by each call.  Every call on
// a device shares the array: calls whose work overlaps on the GPU race.

constexpr size_t kNoAllocScratchBytes = size_t(1) << 20;        // 1 MiB per device
constexpr size_t kNoAllocNodeOffset = 256;
constexpr size_t kNoAllocMaxNodes = (kNoAllocScratchBytes - kNoAllocNodeOffset) / sizeof(NodeW);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

size_t noalloc_max_nodes() { return kNoAllocMaxNodes; }

// Device address of the scratch array on the current device, looked up once
// per device (the host-side name of the array is not a device address) and
// again after ebem_device_release, whose caller may reset the device (a new
// context may place the array elsewhere).
static int noalloc_scratch(int device, unsigned char** out) {
    constexpr int kMaxDevices = 64;
    static unsigned char* addr[kMaxDevices] = {};
    static unsigned gen[kMaxDevices] = {};
    static std::mutex mu;
    if (device < 0 || device >= kMaxDevices) return fail(EBEM_ERR_INVALID, "device ordinal beyond the supported range");
    std::lock_guard<std::mutex> lock(mu);
    const unsigned g = device_generation(device);
    if (!addr[device] || gen[device] != g) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(EBEM_ERR_CUDA, std::string("scratch address lookup failed: ") + cudaGetErrorString(e));
        addr[device] = (unsigned char*)p;
        gen[device] = g;
    }
    *out = addr[device];
    return EBEM_OK;
}

// Outer rule passed by value (no device table).
struct RuleParam {
    double b[28][3];
    double w[28];
};

__global__ void map_nodes_param_kernel(const double* __restrict__ coords, const int32_t* __restrict__ tris, int nt,
                                       const TriGeom* __restrict__ geo, RuleParam rule, int n_gh,
                                       NodeW* __restrict__ out) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nt * n_gh) return;
    int t = idx / n_gh, g = idx % n_gh;
    double V[3][3];
    for (int v = 0; v < 3; v++) {
        int id = tris[3 * t + v];
        for (int c = 0; c < 3; c++) V[v][c] = coords[3 * id + c];
    }
    const double b0 = rule.b[g][0], b1 = rule.b[g][1], b2 = rule.b[g][2];
    NodeW o;
    o.x = b0 * V[0][0] + b1 * V[1][0] + b2 * V[2][0];
    o.y = b0 * V[0][1] + b1 * V[1][1] + b2 * V[2][1];
    o.z = b0 * V[0][2] + b1 * V[1][2] + b2 * V[2][2];
    o.w = geo[t].area * rule.w[g];
    out[idx] = o;
}

int launch_sa_assemble_noalloc(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, double* d_E,
                               int accumulate, bool count, unsigned long long* host_count, cudaStream_t s) {
    if ((size_t)m.nt * n_gh > kNoAllocMaxNodes)
        return fail(EBEM_ERR_INVALID, "mesh too large for the allocation-free assembly: N x n_gh = " +
                                          std::to_string((long long)m.nt * n_gh) + " outer nodes, at most " +
                                          std::to_string(kNoAllocMaxNodes) + " fit in its 1 MiB scratch array");
    if (3 * n_gh > 64) return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    unsigned char* base = nullptr;
    if (int rc = noalloc_scratch(m.device, &base)) return rc;
    unsigned long long* d_count = (unsigned long long*)base;
    NodeW* d_nodes = (NodeW*)(base + kNoAllocNodeOffset);
    RuleParam rule;
    if (int rc = gh_composite(n_gh, 1, &rule.b[0][0], rule.w)) return fail(rc, "unsupported Gauss-Hammer rule");
    const int total = m.nt * n_gh;
    map_nodes_param_kernel<<<(total + 127) / 128, 128, 0, s>>>(m.d_coords, m.d_tris, m.nt, m.d_geo, rule, n_gh, d_nodes);
    EBEM_CUDA_TRY(cudaGetLastError());
    if (count) EBEM_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s));
    SAArgs A;
    A.geo = m.d_geo;
    A.nodes = d_nodes;
    A.N = m.nt;
    A.n_gh = n_gh;
    A.velP = P.velP;
    A.velS = P.velS;
    A.dt = P.dt;
    A.c4pirho = 4 * kPi * P.rho;
    A.lag0 = lag0;
    A.nlag = nlag;
    A.src0 = 0;
    A.nsrc = m.nt;
    A.diag_only = 0;
    A.E = d_E;
    A.ld = 3 * (size_t)m.nt;
    A.ld_lag = A.ld * A.ld;
    A.accumulate = accumulate;
    A.count = count ? d_count : nullptr;
    A.pairs = nullptr;
    A.npairs = 0;
    A.j0 = 0;
    A.nj = m.nt;
    const long long NN = (long long)m.nt * m.nt;
    int rc = launch_level<EBEM_LEVEL_WPB, EBEM_LEVEL_MINB, false>(A, NN, m.device, s);
    if (rc) return rc;
    if (count) {
        EBEM_CUDA_TRY(cudaMemcpyAsync(host_count, d_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        EBEM_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// Batched assembly: many meshes (instances) in one persistent launch.  Each
// warp grabs `chunk` consecutive pairs of the concatenated pair space
// (instance b owns pairs [pair_begin[b], pair_begin[b] + N_b^2)) from a global
// counter and assembles them with level_pair's per-pair walk (direct output),
// so a batch result equals the single-mesh results to rounding: per pair the
// per-level sums of level_pair, one lane per level forming F(t_k) and writing
// the blocks of the lags it completes.
template <int WPB, int MINB, bool MIXED>
__global__ void __launch_bounds__(32 * WPB, MINB)
sa_batch_level_kernel(const BatchInst* __restrict__ insts, int ninst, long long total, int n_gh, int chunk,
                      unsigned long long* next) {
    extern __shared__ __align__(16) unsigned char batch_smem[];
    LevelShared* Lsh = reinterpret_cast<LevelShared*>(batch_smem);
    __shared__ double gt[48];          // Gauss-Legendre nodes and weights (gl_table_entry)
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    LevelShared& Ls = Lsh[wib];
    if (threadIdx.x < 24) gl_table_entry(threadIdx.x, gt[threadIdx.x], gt[24 + threadIdx.x]);
    __syncthreads();
    unsigned long long unused = 0;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(next, (unsigned long long)chunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((long long)base >= total) break;
        const long long end = min((long long)base + chunk, total);
        for (long long p = (long long)base; p < end; p++) {
            int lo = 0, hi = ninst - 1;                 // last instance with pair_begin <= p
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (insts[mid].pair_begin <= p) lo = mid;
                else hi = mid - 1;
            }
            const BatchInst& I = insts[lo];
            SAArgs A;
            A.geo = I.geo;
            A.nodes = I.nodes;
            A.N = I.N;
            A.n_gh = n_gh;
            A.velP = I.velP;
            A.velS = I.velS;
            A.dt = I.dt;
            A.c4pirho = I.c4pirho;
            A.lag0 = 0;
            A.nlag = I.nlag;
            A.src0 = 0;
            A.nsrc = I.N;
            A.diag_only = 0;
            A.E = I.E;
            A.ld = 3 * (size_t)I.N;
            A.ld_lag = A.ld * A.ld;
            A.accumulate = 0;
            A.count = nullptr;
            A.pairs = nullptr;
            A.npairs = 0;
            A.j0 = 0;
            A.nj = I.N;
            A.zeros_written = 1;
            const long long q = p - I.pair_begin;
            level_pair<MIXED>(A, Ls, gt, gt + 24, q, (int)(q % I.N), (int)(q / I.N), lane, unused);
        }
    }
}

template <int WPB, int MINB, bool MIXED>
static int launch_batch_level(const BatchInst* d_insts, int ninst, long long total, int n_gh, int chunk,
                              unsigned long long* d_next, int device, cudaStream_t s) {
    const size_t smem = sizeof(LevelShared) * WPB;
    if (int rc = opt_in_smem(sa_batch_level_kernel<WPB, MINB, MIXED>, smem, s)) return rc;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const unsigned blocks = (unsigned)(sms * MINB);       // one resident wave: persistent
    sa_batch_level_kernel<WPB, MINB, MIXED><<<blocks, 32 * WPB, smem, s>>>(d_insts, ninst, total, n_gh, chunk, d_next);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

// Zeros of every instance's output (the output pointers read from the device
// table at run time, as the assembly reads them): blockIdx.y = instance,
// 16-byte stores over its 9 N^2 nlag doubles.  The assembly then writes only
// the blocks of each pair's non-null lags; zeroing the whole buffer at copy
// bandwidth costs less than the scattered zero blocks of the direct output.
__global__ void batch_zero_kernel(const BatchInst* __restrict__ insts) {
    const BatchInst& I = insts[blockIdx.y];
    const long long n = 9LL * I.N * I.N * I.nlag;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    if ((reinterpret_cast<size_t>(I.E) & 15) == 0) {
        double2* E2 = reinterpret_cast<double2*>(I.E);
        const double2 z = make_double2(0.0, 0.0);
        for (long long k = t0; k < n / 2; k += stride) E2[k] = z;
        if ((n & 1) && t0 == 0) I.E[n - 1] = 0.0;
    } else {
        // an output that starts off a 16-byte boundary: 8-byte stores
        for (long long k = t0; k < n; k += stride) I.E[k] = 0.0;
    }
}

int launch_sa_batch(const BatchInst* d_insts, int ninst, long long total, int n_gh, int mixed, int wpb, int chunk,
                    unsigned long long* d_next, int device, cudaStream_t s) {
    (void)n_gh;
    if (ninst > 65535) return fail(EBEM_ERR_INVALID, "too many batch instances for one launch");
    batch_zero_kernel<<<dim3(148, (unsigned)ninst), 256, 0, s>>>(d_insts);
    EBEM_CUDA_TRY(cudaGetLastError());
    if (wpb == 2)
        return mixed ? launch_batch_level<2, 6, true>(d_insts, ninst, total, n_gh, chunk, d_next, device, s)
                     : launch_batch_level<2, 6, false>(d_insts, ninst, total, n_gh, chunk, d_next, device, s);
    return mixed ? launch_batch_level<4, 3, true>(d_insts, ninst, total, n_gh, chunk, d_next, device, s)
                 : launch_batch_level<4, 3, false>(d_insts, ninst, total, n_gh, chunk, d_next, device, s);
}

}  // namespace ebem
