/*
 * libebem — C ABI of the B200-native energetic space-time Galerkin BEM for 3D
 * elastodynamics (Lamé single-layer operator, piecewise-constant space/time).
 *
 * Plain C types only: host or device pointers and sizes.  Every function
 * returns an int status (EBEM_OK = 0, negative on error) and leaves a
 * thread-local message for ebem_last_error().  Matrices use the reference's
 * byte layouts so that a MATLAB/MEX caller can `reshape` them unchanged:
 *
 *   E   column-major 3N x 3N per lag, lags slowest:
 *       E[l*(3N)^2 + (3*j + c)*3N + 3*i + r] = block (source i, field j, lag l),
 *       row component r, column component c
 *       (reference: functions/BEMenerg_indir/BEMenerg_core/BEMenerg_coreGPU/
 *        CUDAkernels/kernelGHC.cu:162, BEMenerg_coreSA_calcMatrixBlock.m:41,80)
 *   phi column-major 3N x nT, phi[n*3N + 3*i + c]
 *       (BEMenerg_coreGPU_timeMarching.m:156)
 *
 * Output pointers may be device pointers (the call is asynchronous on
 * `stream` unless it returns a count) or host pointers (the library stages
 * through device memory and returns after the copy).  `stream` is a
 * cudaStream_t passed as void*; NULL is the legacy default stream.
 *
 * Reference paths are relative to the IvanDB/ElastodynamicEBEM project root;
 * "f/" abbreviates "functions/".
 */
#ifndef EBEM_H
#define EBEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EBEM_VERSION 1

#define EBEM_OK 0
#define EBEM_ERR_INVALID (-1)   /* bad argument, unsupported rule, size limit */
#define EBEM_ERR_CUDA (-2)      /* CUDA runtime/library failure */
#define EBEM_ERR_NOMEM (-3)     /* device or host allocation failed */
#define EBEM_ERR_NODEVICE (-4)  /* no CUDA device visible */
#define EBEM_ERR_SINGULAR (-5)  /* E_0 factorisation found a zero pivot */

/* Opaque device-resident mesh: vertices, triangles and per-triangle frames.
 * It caches device data built on first use (the mapped outer nodes of each
 * rule, the direct formulation's vertex adjacency), so one handle must not
 * be used by two host threads at once; distinct handles are independent. */
typedef struct ebem_mesh ebem_mesh;

/* The reference's pbParam (f/utility/fileRead/readInputFile.m:12-74):
 * c_P = sqrt((lambda+2 mu)/rho), c_S = sqrt(mu/rho), dt = tfin/nt. */
typedef struct ebem_problem {
    double rho;
    double mu;
    double lambda;
    double tfin;
    int nt;
} ebem_problem;

/* Library version (EBEM_VERSION). */
int ebem_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* ebem_last_error(void);

/* Per-call device workspace comes from a stream-ordered memory pool that the
 * library keeps for each device; up to 2 GiB per device stay reserved between
 * calls so that repeated calls neither allocate nor synchronise the device.
 * ebem_release_workspace returns every device's reserved workspace memory
 * that no call in flight uses (after the calls in flight have finished). */
int ebem_release_workspace(void);

/* Bytes the workspace pool of `device` holds reserved and in use (both 0
 * when the library has not used that device).  No counterpart in the
 * reference. */
int ebem_workspace_info(int device, unsigned long long* reserved, unsigned long long* used);

/* Device-time profile of the semi-analytic assembly of dense outputs, which
 * runs in two passes (per chunk of field columns: the level kernel that stores
 * F(t_k) of every pair and level, then the emission kernel that writes the
 * blocks).  While enabled, each such call records CUDA events around its
 * launches on its stream and waits for them at its end; ebem_profile_read
 * returns the summed milliseconds and launch counts of both passes since the
 * last reset (ms[0], launches[0]: levels; ms[1], launches[1]: emission) and
 * resets them when reset != 0.  No counterpart in the reference (it has no
 * timing code). */
int ebem_profile_enable(int on);
int ebem_profile_read(double* ms, long long* launches, int reset);

/* Release everything the library keeps for `device` between calls, before
 * its CUDA context is reset (cudaDeviceReset, or the reset(gpuDevice) that
 * f/BEMenerg_indir/BEMenerg_core/BEMenerg_coreGPU/BEMenerg_coreGPU_timeMarching.m:7,170
 * runs at entry and exit): waits for the device, destroys the workspace pool
 * and the calling thread's cuSOLVER / cuBLAS handles, and forgets the device
 * address of the allocation-free assembly's scratch array.  Handles of other
 * host threads are abandoned (not destroyed) at their next use.  Later calls
 * rebuild all of it.  Objects the caller holds (meshes, batch plans, banded
 * operators, LU plans) own device memory of that context: destroy them
 * before the reset.  No counterpart in the reference. */
int ebem_device_release(int device);

/* Gauss-Hammer composite rule.  Replaces f/utility/quadRules/
 * GaussHammerComposite.m:1 (with the base tables of GaussHammer_base.m).
 * n_nodes in {1,3,7,12,19,28}; n_sub in {1,4,16,64,...} (a square);
 * nodes: host array n_sub*n_nodes x 3 barycentric coordinates (row-major);
 * weights: host array n_nodes, (2/n_sub) x base weights. */
int ebem_quad_gh(int n_nodes, int n_sub, double* nodes, double* weights);

/* Upload a surface mesh and derive normals, areas, centroids, longest edges
 * and in-plane frames on the device.  Replaces the derived-field part of
 * f/utility/fileRead/readSpaceMesh.m:93-151 and the per-triangle constants of
 * .../BEMenerg_coreSA/BEMenerg_coreSA_calcCostantData.m:1-26.
 * coords: host n_vertices x 3; tris: host n_triangles x 3, 0-based. */
int ebem_mesh_create(const double* coords, int n_vertices, const int32_t* tris, int n_triangles,
                     ebem_mesh** out);
int ebem_mesh_destroy(ebem_mesh* mesh);
int ebem_mesh_info(const ebem_mesh* mesh, int* n_vertices, int* n_triangles);
/* Derived fields copied to host arrays (any may be NULL): normal (N x 3),
 * area (N), center (N x 3), maxl (N); readSpaceMesh.m:114-139. */
int ebem_mesh_derived(const ebem_mesh* mesh, double* normal, double* area, double* center, double* maxl);
/* Device data the mesh handle holds: rules_cached bit k set when the mapped
 * outer-node table of rule k (1, 3, 7, 12, 19, 28 nodes) is cached, and the
 * device bytes held (geometry, cached tables including composite rules,
 * direct-formulation data).
 * No counterpart in the reference. */
int ebem_mesh_cache_info(const ebem_mesh* mesh, int* rules_cached, long long* device_bytes);

/* Number of non-zero Toeplitz blocks L = min(nT, ceil(maxDist/(c_S dt)) + 1).
 * Replaces .../BEMenerg_coreGPU/BEMenerg_coreGPU_calcNumBlocks.m:1-20. */
int ebem_num_blocks(const ebem_mesh* mesh, const ebem_problem* prob, int* num_blocks);

/* Semi-analytic assembly of E_lag0 ... E_{lag0+nlag-1}: outer Gauss-Hammer
 * rule with n_gh nodes (3, 7, 12 or 19) on the source triangle, closed-form
 * inner integral on the field triangle, P- and S-fronts, energetic second
 * difference in time, null test and 1e-14 clean-up of the reference.
 * Replaces BEMenerg_coreSA_calcMatrixBlock(matrix, methodInfo, indTemp,
 * deltaT, pbParam, domainMesh, constValues)
 * (.../BEMenerg_coreSA/calcoloMatrice/BEMenerg_coreSA_calcMatrixBlock.m:1),
 * one call per lag there, and the feval of the assembly kernel in
 * .../BEMenerg_coreGPU/BEMenerg_coreGPU_launchKernel.m:11 (same layout).
 * E: 9 N^2 nlag doubles, host or device.  accumulate = 0 overwrites every
 * entry (zeros included); 1 adds (E += block), as the reference kernels do.
 * nonnull (may be NULL): number of (source, field, lag) blocks that pass the
 * null test; requesting it synchronises the stream, so it must be NULL on a
 * stream under capture (EBEM_ERR_INVALID otherwise).  A device E must belong
 * to the mesh's device (EBEM_ERR_INVALID otherwise); so must every device
 * buffer passed to a mesh-based entry point below. */
int ebem_assemble_sa(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int lag0, int nlag,
                     double* E, int accumulate, void* stream, long long* nonnull);

/* Row panel of the same assembly: source triangles [src0, src0+nsrc) only,
 * written column-major as (3 nsrc) x 3N per lag with leading dimension ld
 * (ld >= 3 nsrc; lag stride ld*3N).  E + 3*src0 with ld = 3N writes the
 * panel into a full matrix.  Used to shard the assembly across GPUs by
 * source rows; the reference's parfor over all N^2 pairs
 * (BEMenerg_coreSA_calcMatrixBlock.m:38) restricted to one row range.
 * Host E requires ld == 3 nsrc. */
int ebem_assemble_sa_panel(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int lag0, int nlag,
                           int src0, int nsrc, double* E, long long ld, int accumulate, void* stream,
                           long long* nonnull);

/* Precision of the semi-analytic assembly.  EBEM_PREC_FP64 is the reference's
 * arithmetic.  EBEM_PREC_MIXED evaluates the bulk quadrature, the Gauss-
 * Legendre nodes of the edge-bounded pieces (after the node position e^s,
 * which stays FP64), in FP32 with FP32 per-lane accumulation, and keeps FP64
 * for the closed-form pieces at the wavefronts and the singularity (crossing
 * angles, logarithmic terms), the whole-edge moments, the level combination
 * F_{l+1} - 2 F_l + F_{l-1}, the E_0 factorisation and the time-marching
 * right-hand side.  No counterpart in the reference (the mixed-precision form
 * of the assembly). */
#define EBEM_PREC_FP64 0
#define EBEM_PREC_MIXED 1

/* The full assembly of ebem_assemble_sa (FP64, all source rows), for callers
 * that may not allocate device memory while they run: code that executes
 * inside a host framework whose device memory is all handed out by its own
 * pool, or a time-critical loop where a cudaMalloc/cudaFree (which can
 * synchronise the device) is not allowed.  No counterpart in the reference.
 *
 * It allocates nothing: the two small device buffers the ordinary assembly
 * allocates for itself (the mesh's mapped outer nodes and the non-null
 * counter) live here in one statically allocated 1 MiB device array that
 * every GPU loading the library keeps until the process exits.  Limit:
 * N x n_gh <= 32760 outer nodes (e.g. 2800 triangles with 7 nodes, 1280 with
 * 19); larger meshes are rejected with EBEM_ERR_INVALID.  E must be a device
 * buffer of 9 N^2 nlag doubles.
 *
 * The first call on a device looks up the device address of the array (a
 * one-time set-up, repeated once after ebem_device_release); make that first
 * call before any stream capture.  nonnull must be NULL on a stream under
 * capture (the count is read back and waited for).  All calls on a device
 * share the array and each call rewrites it (the counter is zeroed by every
 * call that asks for nonnull): calls whose work can overlap on the GPU
 * (different streams, no ordering between them) race and must be serialised
 * by the caller. */
int ebem_assemble_sa_noalloc(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int lag0, int nlag,
                             double* E, int accumulate, void* stream, long long* nonnull);

/* Batched assembly of many instances (meshes with their own problem data and
 * lag counts) in one persistent, graph-captured launch.  No counterpart in
 * the reference (it assembles one mesh per run, BEMenerg_coreSA_timeMarching.m).
 * Every warp takes a few pairs at a time from a global counter across all
 * instances, so small and large meshes share the GPU without tail effects.
 * ebem_batch_create records the instances (nlag may be NULL: L of each
 * instance; instance k assembles lags 0..nlag[k]-1) with one outer rule and
 * precision mode.  The first ebem_batch_assemble tunes the schedule: the
 * persistent launch's tile shape (warps per block x pairs per grab) and, as
 * one more candidate, one two-pass assembly per instance, each timed once on
 * the batch; it captures the fastest in a CUDA graph and every call replays
 * the graph (the persistent launch reads the outputs from a device table at
 * run time; the per-instance schedule is recaptured when a call passes other
 * output buffers than the captured ones).  E[k]:
 * device buffer of 9 N_k^2 nlag[k] doubles, same layout as ebem_assemble_sa,
 * every entry written; results equal ebem_assemble_sa's to rounding (the
 * same per-pair computation in another kernel).  The plan reads its meshes'
 * device data at every replay: destroy it before any of its meshes (using
 * the meshes in other calls meanwhile, with any rule, is fine).
 * ebem_batch_info reports the chosen shape (0 and 0 for the per-instance
 * schedule), its tuning time and the pair count. */
typedef struct ebem_batch ebem_batch;
int ebem_batch_create(const ebem_mesh* const* meshes, const ebem_problem* probs, const int* nlag, int n, int n_gh,
                      int prec, ebem_batch** out);
int ebem_batch_assemble(ebem_batch* batch, double* const* E, void* stream);
int ebem_batch_info(const ebem_batch* batch, int* warps_per_block, int* pairs_per_grab, float* tuned_ms,
                    long long* pairs);
int ebem_batch_destroy(ebem_batch* batch);

/* Learned quadrature selector (no counterpart in the reference, which uses
 * one outer rule for every pair and lag, BEMenerg_setupCore.m:13-28).
 * Outer rules are (n_gh, n_sub) pairs: the n_gh-node Gauss-Hammer rule on
 * n_sub congruent sub-triangles of the source triangle (n_sub a square,
 * GaussHammerComposite.m:1-55).  A small MLP (12 -> 64 -> 64 -> 4, ReLU,
 * softmax, FP32; EBEM_SELECTOR_PARAMS floats: W1[64][12], b1[64],
 * W2[64][64], b2[64], W3[4][64], b3[4]) maps the 12 features of a
 * (source, field, lag) to one of four rules (class 0..3, class 3 the
 * maximal one).  All buffers below are device buffers unless stated.
 *   ebem_sa_pair_blocks  the plain method's blocks of explicit pairs
 *              (pairs[2 p] = source, pairs[2 p + 1] = field) at lags
 *              0..nlag-1 with rule (n_gh, n_sub): out[(p nlag + l) 6 + e],
 *              the 6 symmetric entries 11, 12, 13, 22, 23, 33 of E_l, zero
 *              outside the pair's non-null lags.
 *   _init      He-initialised parameters (host or device buffer).
 *   _features  n x 12 features of samples[3 q .. 3 q + 2] = (source, field, lag).
 *   _sweeps    flags[q] = 1 where a wavefront sweeps sample q's distance
 *              window during its lag (c t, t from (l-1) dt to (l+1) dt,
 *              meets [d - h_i - h_j, d + h_i + h_j] for c = c_P or c_S; d
 *              the centroid distance, h the longest edges): the outer rule
 *              converges slowly there and inference gives those lags the
 *              maximal rule.
 *   _labels    labels of n samples from their blocks at the four rules
 *              (blocks[(c n + q) 6 + e]): the smallest rule whose block
 *              differs from the maximal rule's by at most tol * scale (times
 *              scales[q] when the per-sample array is not NULL) in every
 *              entry, else 3.
 *   _grad      gradient of the mean cross-entropy over n samples (+ loss).
 *   _train     Adam over shuffled mini-batches; losses (host, may be NULL)
 *              receives the full-set loss after each epoch.
 *   _infer     class of every (pair, lag) of a mesh for lags lag0..lag0+nlag-1:
 *              cls[(field N + source) nlag + l - lag0] (bytes); the maximal
 *              rule where a front sweeps the lag (as _sweeps) or where the
 *              largest probability is below threshold; 0 at null lags.  counts (host, 4 entries, may be NULL): non-null
 *              lags per class.
 * ebem_assemble_sa_selected assembles every lag of every pair with the rule
 * of its class, rules[2 c], rules[2 c + 1] (host, nclass pairs) for class c
 * (E as ebem_assemble_sa, device, every entry written); counts (host, nclass
 * entries, may be NULL) receives the non-null lags per class.  With every
 * class byte 0 it is the plain assembly with rule (rules[0], rules[1]). */
#define EBEM_SELECTOR_FEATURES 12
#define EBEM_SELECTOR_CLASSES 4
#define EBEM_SELECTOR_PARAMS 5252
int ebem_sa_pair_blocks(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int n_sub, const int* pairs,
                        long long npairs, int nlag, double* out, void* stream);
int ebem_selector_init(float* params, unsigned long long seed);
int ebem_selector_features(const ebem_mesh* mesh, const ebem_problem* prob, const int* samples, long long n,
                           float* feats, void* stream);
int ebem_selector_sweeps(const ebem_mesh* mesh, const ebem_problem* prob, const int* samples, long long n,
                         unsigned char* flags, void* stream);
int ebem_selector_labels(const double* blocks, long long n, double tol, double scale, const double* scales,
                         int* labels, void* stream);
int ebem_selector_grad(const float* params, const float* feats, const int* labels, long long n, float* grad,
                       float* loss, void* stream);
int ebem_selector_train(float* params, const float* feats, const int* labels, long long n, int epochs, int batch,
                        float lr, unsigned long long seed, float* losses, void* stream);
int ebem_selector_infer(const float* params, const ebem_mesh* mesh, const ebem_problem* prob, float threshold,
                        int lag0, int nlag, unsigned char* cls, long long* counts, void* stream);
int ebem_assemble_sa_selected(const ebem_mesh* mesh, const ebem_problem* prob, const int* rules, int nclass,
                              const unsigned char* cls, int lag0, int nlag, double* E, int prec, void* stream,
                              long long* counts);

/* ebem_assemble_sa_panel with a precision mode. */
int ebem_assemble_sa_ex(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int lag0, int nlag, int src0,
                        int nsrc, double* E, long long ld, int accumulate, int prec, void* stream, long long* nonnull);

/* Numerical-inner assembly (the reference's GPU method "GPU xx yy z"): outer
 * Gauss-Hammer rule with n_gh nodes on the source triangle, composite rule of
 * n_sub sub-triangles x n_sing nodes on the field triangle, Lamé kernel with
 * P/S Heaviside fronts, off-diagonal pairs only, added to E (E += block,
 * entries with |value| <= 1e-14 before the 1/(4 pi rho) skipped).  Replaces
 * the kernelGHC feval of
 * f/BEMenerg_indir/BEMenerg_core/BEMenerg_coreGPU/BEMenerg_coreGPU_launchKernel.m:11
 * (kernel: .../CUDAkernels/kernelGHC.cu:5; the same kernel is kernelV.cu of
 * f/BEMenerg_dir).  sa_diagonal = 1 also writes the diagonal blocks with the
 * semi-analytic result, as BEMenerg_coreGPU_timeMarching.m:101-131 inserts
 * its CPU semi-analytic diagonal.  E: host or device, 9 N^2 nlag doubles. */
int ebem_assemble_ghc(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int n_sub, int n_sing, int lag0,
                      int nlag, double* E, int sa_diagonal, void* stream);

/* Right-hand side b_n, n = 0..nT-1: b_n[3i+c] = sum_g w_g (g(x_g, t_{n+1}) -
 * g(x_g, t_n)) over the outer nodes of triangle i, entries below 1e-14 set
 * to 0.  Replaces BEMenerg_core_calcTnBlock(rhs, methodInfo, indTemp, deltaT,
 * pbParam, domainMesh, constValues)
 * (f/BEMenerg_indir/BEMenerg_core/BEMenerg_core_calcTn/BEMenerg_core_calcTnBlock.m:1),
 * all steps at once.  datum selects g (f/.../BEMenerg_core_calcNucleoTn.m:196-244):
 * 0 (0,0,t^4 e^{-2t}), 1 x sin(2 pi t) H(t), 2 'sphereUniform', 3 'screenUniform',
 * 4 'barH1', 5 'barH3', 6 'sphereWave', 7 'elementoIndustriale', 8 'TEST' (the
 * manufactured case of :13-132 whose solution is phi = (1, 1, 1), defined on
 * the screen [-1,1]^2 at z = 0; other meshes are rejected).
 * rhs: 3N x nT column-major, host or device. */
int ebem_rhs(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int datum, double* rhs, void* stream);

/* Time marching: LU of E_0 once (and from it E_0^{-1}, as ebem_lu_create
 * does), then phi_n = E_0^{-1}(b_n - sum_{l=1}^{min(n,L-1)} E_l phi_{n-l}).
 * Replaces the marching loop of
 * f/BEMenerg_indir/BEMenerg_core/BEMenerg_coreGPU/BEMenerg_coreGPU_timeMarching.m:151-169
 * (and of BEMenerg_coreSA_timeMarching.m:46-113).  E: n3 x n3 x L (the
 * layout of ebem_assemble_sa), rhs and phi: n3 x nT; host or device.
 * Returns EBEM_ERR_SINGULAR when E_0 has a zero pivot. */
int ebem_march(const double* E, int n3, int L, const double* rhs, int nT, double* phi, void* stream);

/* ebem_march with a choice of factorisation of E_0.  EBEM_FACTOR_LU is the
 * reference's lu with partial pivoting (BEMenerg_coreSA_timeMarching.m:46);
 * EBEM_FACTOR_CHOLESKY factors the symmetric part (E_0 + E_0^T) / 2 by
 * Cholesky (half the work of the LU): E_0 of the semi-analytic
 * assembly (outer quadrature, exact inner integral) is not exactly symmetric,
 * so the two differ by the asymmetry's effect on the density.  Returns
 * EBEM_ERR_SINGULAR when the symmetric part is not positive definite. */
#define EBEM_FACTOR_LU 0
#define EBEM_FACTOR_CHOLESKY 1
int ebem_march_ex(const double* E, int n3, int L, const double* rhs, int nT, double* phi, int factor, void* stream);

/* Pieces of ebem_march for callers that drive the steps themselves (the
 * row-panel marching across ranks, where each rank holds the rows
 * [r0, r0 + rows) of every E_l and one all-gather per step assembles the
 * right-hand side).
 *
 * ebem_lu_create: the factorisation of the device matrix A (column-major
 * n x n) for repeated solves; replaces [L, U, P] = lu(sparse(matrix)) of
 * f/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/BEMenerg_coreSA_timeMarching.m:46
 * (BEMenerg_coreGPU_timeMarching.m:153).  LU with partial pivoting, from
 * which A^{-1} is formed once and kept on the device (n^2 doubles), so that
 * a solve is one matrix-vector product rather than two triangular solves of
 * one right-hand side.  Returns EBEM_ERR_SINGULAR on a zero pivot.
 * ebem_lu_solve overwrites the device columns b (n x nrhs) with A^{-1} b
 * (U\(L\(P*b)) of :59, equal to rounding: the two differ by about
 * cond(A) times the unit roundoff).  ebem_lu_destroy frees the inverse.
 *
 * ebem_history_gemv: y -= A x for device A (rows x K, column-major, leading
 * dimension rows), x (K) and y (rows): the history sum
 * tnf = tnf - matrixSaved{indMat} * density(:, currInd - indMat + 1) of
 * BEMenerg_coreGPU_timeMarching.m:160-166 for all lags at once when A is
 * [E_1 E_2 ... E_M] restricted to a row panel and x = (phi_{n-1}; ...;
 * phi_{n-M}). */
/* Banded (block-sparse) Toeplitz blocks and the marching on them.  The
 * reference keeps every E_l dense (matrixSaved{l},
 * f/BEMenerg_indir/BEMenerg_core/BEMenerg_coreGPU/BEMenerg_coreGPU_timeMarching.m:139-147;
 * one .mat file per block in BEMenerg_coreSA_timeMarching.m:96-99), although
 * a (source, field) block is zero outside the lags that pass the null test of
 * BEMenerg_coreSA_calcMatrixBlock.m:57-61.  That test is monotone in the lag,
 * so each pair's non-null lags form one band, and the blocks are symmetric:
 * this storage keeps 6 doubles per non-null pair-lag (plus 12 bytes per pair
 * of structure) instead of 9 doubles per pair and lag.
 *
 * ebem_banded_assemble: E_0..E_{L-1} (L from ebem_num_blocks) by the
 * semi-analytic method, FP64 or EBEM_PREC_MIXED, into a device-resident
 * operator; the values equal those of ebem_assemble_sa.
 * ebem_banded_info: triangles, L, non-null pair-lags and device bytes held.
 * ebem_banded_to_dense: E_lag0..E_{lag0+nlag-1} in the layout of
 * ebem_assemble_sa (host or device).
 * ebem_banded_march: the marching of ebem_march (LU of E_0 once, history
 * sum_{l>=1} E_l phi_{n-l} per step) on the banded blocks; rhs and phi
 * 3N x nT, host or device.
 * No counterpart in the reference beyond the dense equivalents cited. */
typedef struct ebem_banded ebem_banded;
int ebem_banded_assemble(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int prec, void* stream,
                         ebem_banded** out);
int ebem_banded_info(const ebem_banded* op, int* n_triangles, int* num_blocks, long long* nonnull, long long* bytes);
int ebem_banded_to_dense(const ebem_banded* op, int lag0, int nlag, double* E, void* stream);
int ebem_banded_march(const ebem_banded* op, const double* rhs, int nT, double* phi, void* stream);
void ebem_banded_destroy(ebem_banded* op);

typedef struct ebem_lu ebem_lu;
int ebem_lu_create(const double* A, int n, void* stream, ebem_lu** out);
int ebem_lu_solve(ebem_lu* lu, double* b, int nrhs, void* stream);
void ebem_lu_destroy(ebem_lu* lu);
int ebem_history_gemv(const double* A, int rows, long long K, const double* x, double* y, void* stream);

/* The semi-analytic indirect solve end to end: assembly of E_0..E_{L-1}
 * (L from ebem_num_blocks), right-hand side, time marching.  Replaces
 * density = BEMenerg_coreSA_timeMarching(pbParam, domainMesh, methodInfo, GHn, GHw)
 * (f/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/BEMenerg_coreSA_timeMarching.m:1).
 * phi: 3N x nT, host or device; num_blocks (may be NULL) receives L. */
int ebem_timemarch_sa(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int datum, double* phi,
                      int* num_blocks, void* stream);

/* ebem_timemarch_sa with the assembly in precision mode prec (EBEM_PREC_*). */
int ebem_timemarch_sa_ex(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int datum, int prec, double* phi,
                         int* num_blocks, void* stream);

/* Displacement u(x, t) at npts points and ntimes times from the density
 * (closed-form inner integrals, the single-point analogue of the assembly).
 * Replaces campoVett = BEMenerg_postProcA_setup(pbParam, domainMesh, density,
 * numPoints, xVal, tVal)
 * (f/BEMenerg_indir/BEMenerg_postProc/BEMenerg_postProcA/BEMenerg_postProcA_setup.m:1).
 * phi: 3N x nT; pts: npts x 3 (row-major); times: host array, each <= tfin
 * (EBEM_ERR_INVALID otherwise; t <= 0 gives zero); u: 3 x npts x ntimes
 * (u[(q*npts + p)*3 + c]); phi/pts/u host or device. */
int ebem_pp_sa(const ebem_mesh* mesh, const ebem_problem* prob, const double* phi, const double* pts, int npts,
               const double* times, int ntimes, double* u, void* stream);

/* Numerical post-processing of the indirect formulation, the reference's
 * method "GPU yy z" (composite Gauss-Hammer rule of n_sub sub-triangles x
 * n_sing nodes on every triangle, n_sub in {1,4,16,64}, n_sing in
 * {1,3,7,12,19}; f/utility/setup/BEMenerg_setupPost.m:15-27), at npts points
 * and ntimes times, arguments and output as ebem_pp_sa.  variant:
 *   EBEM_PP_POINT  kernelSP (f/BEMenerg_indir/BEMenerg_postProc/
 *                  BEMenerg_postProcGPU/CUDAkernels/kernelSP.cu:5-105 with the
 *                  host sum of BEMenerg_postProcGPU_calcSP.m:78-85): entries
 *                  kept when |sum| > 1e-14 before the division by 4 pi rho,
 *                  u = sum_{k<nHat} (M_k - M_{k+1}) phi_k + M_nHat phi_nHat;
 *                  replaces BEMenerg_postProcGPU_setupSP.m:1 (main.m:167).
 *   EBEM_PP_LAYER  kernelLayer (.../CUDAkernels/kernelLayer.cu:5-175):
 *                  entries below 1e-14 after the division zeroed,
 *                  u = sum_{k<=nHat} M_k (phi_k - phi_{k-1});
 *                  replaces BEMenerg_postProcGPU_setupLayer.m:1 (main.m:165).
 * nHat = ceil(t / dt) - 1; u = 0 for t <= 0; times <= tfin.  flags:
 * EBEM_FIX_REFERENCE_DEFECTS reads kernelSP's nodes with stride n_sing; by
 * default it keeps the reference's stride 3 (kernelSP.cu:41), and rules where
 * that read would pass the end of the node table (n_sing = 1, n_sub > 1) are
 * refused with EBEM_ERR_INVALID. */
#define EBEM_PP_POINT 0
#define EBEM_PP_LAYER 1
int ebem_pp_gpu(const ebem_mesh* mesh, const ebem_problem* prob, int n_sub, int n_sing, int variant, int flags,
                const double* phi, const double* pts, int npts, const double* times, int ntimes, double* u,
                void* stream);

/* ------------------------------------------------------------------------
 * Direct formulation (f/BEMenerg_dir, f/BEMenerg_dirPP).
 * Rules: outer Gauss-Hammer n_gh in {3,7,12,19}; inner composite rule
 * (n_sub in {1,4,16,64}, n_sing in {1,3,7,12,19}); DIAG rule n_diag in
 * {16,64,256,1024} (doppioGauss1D).  "FN n_gh n_sub n_sing n_diag" of
 * BEMenerg_setupCore.m:86-110.
 *
 * flags: EBEM_FIX_REFERENCE_DEFECTS evaluates H(t - r/c_P) in the lambda-mu
 * term of kernelK (the reference has H(r - r/c_P), kernelK.cu:414-449),
 * starts the null test's minimum distance at +inf (kernelK.cu:242: 100) and
 * reads kernelG's nodes with stride n_sing (kernelG.cu:51: 3).  Default 0
 * reproduces the reference. */
#define EBEM_FIX_REFERENCE_DEFECTS 1

/* L_V and L_K = min(L_V + 1, nT) (BEMenerg_dir_timeMarchingN.m:10,172). */
int ebem_num_blocks_dir(const ebem_mesh* mesh, const ebem_problem* prob, int* lv, int* lk);

/* Double-layer operator K_lag0..K_{lag0+nlag-1}: nlag x (3N x 3Nv), column
 * major per lag (entry (3t+i, 3s+j): triangle t, vertex s), host or device.
 * The off-singular part of kernelK.cu:14-212 (launched by
 * BEMenerg_dir_timeMarchingN.m:186-206, clamp |x| <= 1e-14, / 4 pi dt) plus,
 * when n_diag > 0, the same-triangle parts of BEMenerg_dir_calcSubBlockSingK.m
 * (BEMenerg_dir_timeMarchingN.m:208-264).  Lags >= L_K stay zero.
 * accumulate = 0 zeroes the output first. */
int ebem_assemble_k(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int n_sub, int n_sing, int n_diag,
                    int lag0, int nlag, int flags, double* K, int accumulate, void* stream);

/* Single-layer operator of the direct formulation, V_lag0..: nlag x (3N x 3N):
 * kernelV.cu off the diagonal (BEMenerg_dir_launchKernelV.m) and the DIAG-rule
 * diagonal blocks of BEMenerg_dir_calcSubBlockDiagV.m
 * (BEMenerg_dir_timeMarchingN.m:94-160).  n_diag > 0 is required. */
int ebem_assemble_v(const ebem_mesh* mesh, const ebem_problem* prob, int n_gh, int n_sub, int n_sing, int n_diag,
                    int lag0, int nlag, double* V, void* stream);

/* DN time marching (BEMenerg_dir_timeMarchingN.m:268-299): beta_V,n =
 * sum_j V_{n-j} gV_j (BEMenerg_dir_calcBetaVgpu.m), then per step the least
 * squares solution of (K_0 + I_Gamma) u_n = beta_V,n + I_Gamma u_{n-1} -
 * sum_{l=1}^{min(n,LK)-1} K_l u_{n-l} (the reference's mldivide of a 3N x 3Nv
 * system), I_Gamma = kron((vertex in triangle) area / 6, eye(3)).
 * V: LV x 3N x 3N; K: LK x 3N x 3Nv; gV: 3N x nT; u: 3Nv x nT. */
int ebem_march_dn(const ebem_mesh* mesh, const ebem_problem* prob, const double* V, int LV, const double* K, int LK,
                  const double* gV, double* u, void* stream);

/* DD time marching (BEMenerg_dir_timeMarchingD.m:272-296): V_0 phi_n =
 * rhs_n / 2 + beta_K,n - sum_l V_l phi_{n-l}, beta_K,n = sum_j K_{n-j} gK_j.
 * rhs: 3N x nT; gK: 3Nv x nT; phi: 3N x nT. */
int ebem_march_dd(const ebem_mesh* mesh, const ebem_problem* prob, const double* V, int LV, const double* K, int LK,
                  const double* rhs, const double* gK, double* phi, void* stream);

/* Direct post-processing u(x, t) = sum_{n=1}^{nHat} G_n a_n - P_n b_n at npts
 * points and ntimes times (BEMenerg_ppN_calc.m:115-124 with a = gV, b = u;
 * BEMenerg_ppD_calc.m:91-99 with a = phi, b = gK), G of kernelG.cu and P of
 * kernelP.cu on the composite rule (n_sub, n_sing), contracted on the device.
 * a: 3N x nT; b: 3Nv x nT; u: ntimes x npts x 3; times host, <= tfin. */
int ebem_pp_dir(const ebem_mesh* mesh, const ebem_problem* prob, int n_sub, int n_sing, int flags, const double* a,
                const double* b, const double* pts, int npts, const double* times, int ntimes, double* u,
                void* stream);

/* The matrices of one (x, t) as the reference builds them (BEMenerg_ppN_calc.m:
 * 80-109): G (3 nHat x 3N) and P (3 nHat x 3Nv) column major, nHat = ceil(t/dt). */
int ebem_pp_dir_matrices(const ebem_mesh* mesh, const ebem_problem* prob, int n_sub, int n_sing, int flags,
                         const double* x, double t, double* G, double* P);

#ifdef __cplusplus
}
#endif

#endif /* EBEM_H */
