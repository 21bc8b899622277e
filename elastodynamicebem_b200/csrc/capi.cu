// C-ABI entry points of libebem (declared in include/ebem.h): argument
// checking, device-resident mesh handles, host/device output staging and the
// thread-local error message.  Every compute step runs as a CUDA kernel; a
// call with no visible CUDA device fails with EBEM_ERR_NODEVICE (there is no
// CPU path).
#include "ebem_internal.h"
#include "ptr_kind.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <mutex>

#ifndef EBEM_STAGE_DEVICE_OUTPUT
#define EBEM_STAGE_DEVICE_OUTPUT 0
#endif

struct ebem_mesh {
    ebem::MeshData d;
    double lo[3], hi[3];    // bounding box of the vertices (host side)
};

namespace ebem {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};
// Bumped by ebem_device_release: state cached under an older generation
// (per-thread library handles, the allocation-free scratch address) is
// abandoned and rebuilt on next use.
std::atomic<unsigned> g_generation[kMaxDevices] = {};
}  // namespace

unsigned device_generation(int dev) {
    return (dev >= 0 && dev < kMaxDevices) ? g_generation[dev].load(std::memory_order_acquire) : 0u;
}

namespace {

// The workspace pool of device dev, created on first use.
cudaError_t workspace_pool(int dev, cudaMemPool_t* pool) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return e;
        unsigned long long keep = kWorkspaceKeep;
        e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return e;
        }
        g_pool[dev] = p;
    }
    *pool = g_pool[dev];
    return cudaSuccess;
}
}  // namespace

cudaError_t ws_malloc(void** p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    cudaMemPool_t pool = nullptr;
    if (e == cudaSuccess) e = workspace_pool(dev, &pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes > 0 ? bytes : 1, pool, s);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
    }
    return e;
}

cudaError_t ws_free(void* p, cudaStream_t s) { return p ? cudaFreeAsync(p, s) : cudaSuccess; }

PhysParams phys_from(const ebem_problem* p) {
    PhysParams P;
    P.rho = p->rho;
    P.velP = std::sqrt((p->lambda + 2 * p->mu) / p->rho);
    P.velS = std::sqrt(p->mu / p->rho);
    P.dt = p->tfin / p->nt;
    P.nT = p->nt;
    P.lam = p->lambda;
    P.mu = p->mu;
    return P;
}

namespace {

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

int check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(EBEM_ERR_NODEVICE, "no CUDA device visible");
    }
    return EBEM_OK;
}

int check_problem(const ebem_problem* p) {
    if (!p) return fail(EBEM_ERR_INVALID, "problem is NULL");
    if (!(p->rho > 0) || !(p->mu > 0) || !(p->lambda + 2 * p->mu > 0))
        return fail(EBEM_ERR_INVALID, "material parameters must give rho > 0, mu > 0, lambda + 2 mu > 0");
    if (!(p->tfin > 0) || p->nt < 1) return fail(EBEM_ERR_INVALID, "need tfin > 0 and nt >= 1");
    return EBEM_OK;
}

// Kind of a caller's buffer relative to the current device (the device the
// call runs on).
PtrKind ptr_kind(const void* p, int* owner = nullptr) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return PtrKind::Host;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (owner) *owner = at.device;
    return classify_pointer((int)at.type, at.device, cur);
}

bool is_device_ptr(const void* p) { return ptr_kind(p) == PtrKind::Device; }

int other_device_error(const void* p) {
    int owner = -1, cur = -1;
    ptr_kind(p, &owner);
    cudaGetDevice(&cur);
    return fail(EBEM_ERR_INVALID, "a buffer in the memory of device " + std::to_string(owner) +
                                      " was passed to a call that runs on device " + std::to_string(cur) +
                                      " (the mesh's device); pass a buffer of that device or a host buffer");
}

// EBEM_OK when p is device memory usable by the current device, else a
// failure naming `what`.
int need_device(const void* p, const char* what) {
    const PtrKind k = ptr_kind(p);
    if (k == PtrKind::Device) return EBEM_OK;
    if (k == PtrKind::OtherDevice) return other_device_error(p);
    return fail(EBEM_ERR_INVALID, std::string(what) + " must be in device memory");
}

// A non-null count is copied to the host and waited for, which a stream
// under capture does not allow: such calls are refused before any work.
int reject_count_under_capture(const long long* nonnull, cudaStream_t s) {
    if (!nonnull) return EBEM_OK;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return fail(EBEM_ERR_INVALID, "the stream's capture status could not be read");
    }
    if (st != cudaStreamCaptureStatusNone)
        return fail(EBEM_ERR_INVALID, "nonnull must be NULL while the stream is being captured (the count is read back "
                                      "to the host and waited for)");
    return EBEM_OK;
}

__global__ void max_vertex_dist_kernel(const double* __restrict__ c, int nv, unsigned long long* out) {
    // max over vertex pairs of |P_a - P_b| (calcNumBlocks.m:8-14); distances
    // are non-negative, so their IEEE bit patterns order like the values
    double best = 0.0;
    long long total = (long long)nv * nv;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        int a = (int)(q / nv), b = (int)(q % nv);
        double v0 = c[3 * a] - c[3 * b], v1 = c[3 * a + 1] - c[3 * b + 1], v2 = c[3 * a + 2] - c[3 * b + 2];
        double d = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        best = fmax(best, d);
    }
    for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

// A host-or-device input array made available on the device.
struct DevIn {
    const double* d = nullptr;
    double* owned = nullptr;
    cudaStream_t st = nullptr;
    int init(const double* p, size_t n, cudaStream_t s) {
        const PtrKind k = ptr_kind(p);
        if (k == PtrKind::Device) { d = p; return EBEM_OK; }
        if (k == PtrKind::OtherDevice) return other_device_error(p);
        st = s;
        if (ws_malloc(&owned, n * sizeof(double), s) != cudaSuccess)
            return fail(EBEM_ERR_NOMEM, "device staging allocation failed");
        EBEM_CUDA_TRY(cudaMemcpyAsync(owned, p, n * sizeof(double), cudaMemcpyHostToDevice, s));
        d = owned;
        return EBEM_OK;
    }
    ~DevIn() { ws_free(owned, st); }
};

// A host-or-device output array: device pointer used directly, host pointer
// staged and copied back by finish().
struct DevOut {
    double* d = nullptr;
    double* host = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr;
    int init(double* p, size_t count, cudaStream_t s) {
        n = count;
        const PtrKind k = ptr_kind(p);
        if (k == PtrKind::Device) { d = p; return EBEM_OK; }
        if (k == PtrKind::OtherDevice) return other_device_error(p);
        host = p;
        st = s;
        if (ws_malloc(&d, n * sizeof(double), s) != cudaSuccess)
            return fail(EBEM_ERR_NOMEM, "device staging allocation failed");
        return EBEM_OK;
    }
    int finish(cudaStream_t s) {
        if (host) {
            EBEM_CUDA_TRY(cudaMemcpyAsync(host, d, n * sizeof(double), cudaMemcpyDeviceToHost, s));
            EBEM_CUDA_TRY(cudaStreamSynchronize(s));
        }
        return EBEM_OK;
    }
    ~DevOut() { if (host) ws_free(d, st); }
};

}  // namespace
}  // namespace ebem

using namespace ebem;

extern "C" {

int ebem_version(void) { return EBEM_VERSION; }

const char* ebem_last_error(void) { return g_last_error.c_str(); }

int ebem_release_workspace(void) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    int prev = -1;
    cudaGetDevice(&prev);
    for (int dev = 0; dev < kMaxDevices; dev++) {
        if (!g_pool[dev]) continue;
        cudaError_t e = cudaSetDevice(dev);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemPoolTrimTo(g_pool[dev], 0);
        if (e != cudaSuccess) {
            if (prev >= 0) cudaSetDevice(prev);
            return fail(EBEM_ERR_CUDA, std::string("workspace release: ") + cudaGetErrorString(e));
        }
    }
    if (prev >= 0) cudaSetDevice(prev);
    return EBEM_OK;
}

int ebem_workspace_info(int device, unsigned long long* reserved, unsigned long long* used) {
    if (device < 0 || device >= kMaxDevices) return fail(EBEM_ERR_INVALID, "device ordinal out of range");
    unsigned long long r = 0, u = 0;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (g_pool[device]) {
        cudaMemPoolGetAttribute(g_pool[device], cudaMemPoolAttrReservedMemCurrent, &r);
        cudaMemPoolGetAttribute(g_pool[device], cudaMemPoolAttrUsedMemCurrent, &u);
        cudaGetLastError();
    }
    if (reserved) *reserved = r;
    if (used) *used = u;
    return EBEM_OK;
}

int ebem_profile_enable(int on) {
    profile_enable(on);
    return EBEM_OK;
}

int ebem_profile_read(double* ms, long long* launches, int reset) {
    if (!ms || !launches) return fail(EBEM_ERR_INVALID, "NULL output");
    profile_read(ms, launches, reset);
    return EBEM_OK;
}

int ebem_device_release(int device) {
    if (device < 0 || device >= kMaxDevices) return fail(EBEM_ERR_INVALID, "device ordinal out of range");
    // first: every cached handle and address of this device becomes stale
    g_generation[device].fetch_add(1, std::memory_order_acq_rel);
    cudaError_t e = cudaSuccess;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (g_pool[device]) {
            DeviceGuard dg(device);
            e = cudaDeviceSynchronize();
            cudaError_t e2 = cudaMemPoolDestroy(g_pool[device]);
            if (e == cudaSuccess) e = e2;
            g_pool[device] = nullptr;
        }
    }
    release_thread_handles(device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(EBEM_ERR_CUDA, std::string("device release: ") + cudaGetErrorString(e));
    }
    return EBEM_OK;
}

int ebem_quad_gh(int n_nodes, int n_sub, double* nodes, double* weights) {
    if (!nodes || !weights) return fail(EBEM_ERR_INVALID, "NULL output");
    int rc = gh_composite(n_nodes, n_sub, nodes, weights);
    if (rc) return fail(rc, "unsupported Gauss-Hammer rule (n_nodes in {1,3,7,12,19,28}, n_sub a square >= 1)");
    return EBEM_OK;
}

int ebem_mesh_create(const double* coords, int n_vertices, const int32_t* tris, int n_triangles, ebem_mesh** out) {
    if (!out) return fail(EBEM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!coords || !tris || n_vertices < 3 || n_triangles < 1)
        return fail(EBEM_ERR_INVALID, "mesh needs >= 3 vertices and >= 1 triangle");
    for (long long k = 0; k < 3LL * n_triangles; k++)
        if (tris[k] < 0 || tris[k] >= n_vertices) return fail(EBEM_ERR_INVALID, "triangle vertex index out of range");
    for (long long k = 0; k < 3LL * n_vertices; k++)
        if (!std::isfinite(coords[k])) return fail(EBEM_ERR_INVALID, "non-finite vertex coordinate");
    for (int t = 0; t < n_triangles; t++) {
        const int32_t* v = tris + 3 * t;
        if (v[0] == v[1] || v[1] == v[2] || v[0] == v[2]) return fail(EBEM_ERR_INVALID, "degenerate triangle (repeated vertex)");
    }
    if (int rc = check_device()) return rc;
    ebem_mesh* m = new ebem_mesh();
    for (int c = 0; c < 3; c++) {
        m->lo[c] = m->hi[c] = coords[c];
        for (int v = 1; v < n_vertices; v++) {
            m->lo[c] = std::min(m->lo[c], coords[3 * v + c]);
            m->hi[c] = std::max(m->hi[c], coords[3 * v + c]);
        }
    }
    cudaGetDevice(&m->d.device);
    m->d.nv = n_vertices;
    m->d.nt = n_triangles;
    auto cleanup = [&](int code, const char* msg) {
        ebem_mesh_destroy(m);
        return fail(code, msg);
    };
    if (cudaMalloc(&m->d.d_coords, sizeof(double) * 3 * (size_t)n_vertices) != cudaSuccess ||
        cudaMalloc(&m->d.d_tris, sizeof(int32_t) * 3 * (size_t)n_triangles) != cudaSuccess ||
        cudaMalloc(&m->d.d_geo, sizeof(TriGeom) * (size_t)n_triangles) != cudaSuccess) {
        cudaGetLastError();
        return cleanup(EBEM_ERR_NOMEM, "device allocation failed");
    }
    if (cudaMemcpy(m->d.d_coords, coords, sizeof(double) * 3 * (size_t)n_vertices, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->d.d_tris, tris, sizeof(int32_t) * 3 * (size_t)n_triangles, cudaMemcpyHostToDevice) != cudaSuccess)
        return cleanup(EBEM_ERR_CUDA, "mesh upload failed");
    if (prep_mesh(m->d, 0) != EBEM_OK) { std::string e = g_last_error; ebem_mesh_destroy(m); return fail(EBEM_ERR_CUDA, e); }
    if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(EBEM_ERR_CUDA, "mesh preparation kernel failed");
    // reject zero-area triangles (the frame would divide by zero)
    std::vector<TriGeom> g(n_triangles);
    if (cudaMemcpy(g.data(), m->d.d_geo, sizeof(TriGeom) * n_triangles, cudaMemcpyDeviceToHost) != cudaSuccess)
        return cleanup(EBEM_ERR_CUDA, "mesh download failed");
    for (int t = 0; t < n_triangles; t++)
        if (!(g[t].area > 0) || !std::isfinite(g[t].area)) return cleanup(EBEM_ERR_INVALID, "zero-area triangle in mesh");
    *out = m;
    return EBEM_OK;
}

int ebem_mesh_destroy(ebem_mesh* m) {
    if (!m) return EBEM_OK;
    DeviceGuard dg(m->d.device);
    if (m->d.d_coords) cudaFree(m->d.d_coords);
    if (m->d.d_tris) cudaFree(m->d.d_tris);
    if (m->d.d_geo) cudaFree(m->d.d_geo);
    for (NodeW* t : m->d.d_node_tables)
        if (t) cudaFree(t);
    for (NodeW* t : m->d.d_comp_tables)
        if (t) cudaFree(t);
    free_direct(m->d);
    delete m;
    return EBEM_OK;
}

int ebem_mesh_info(const ebem_mesh* m, int* nv, int* nt) {
    if (!m) return fail(EBEM_ERR_INVALID, "mesh is NULL");
    if (nv) *nv = m->d.nv;
    if (nt) *nt = m->d.nt;
    return EBEM_OK;
}

int ebem_mesh_derived(const ebem_mesh* m, double* normal, double* area, double* center, double* maxl) {
    if (!m) return fail(EBEM_ERR_INVALID, "mesh is NULL");
    DeviceGuard dg(m->d.device);
    std::vector<TriGeom> g(m->d.nt);
    EBEM_CUDA_TRY(cudaMemcpy(g.data(), m->d.d_geo, sizeof(TriGeom) * m->d.nt, cudaMemcpyDeviceToHost));
    for (int t = 0; t < m->d.nt; t++) {
        for (int c = 0; c < 3; c++) {
            if (normal) normal[3 * t + c] = g[t].n[c];
            if (center) center[3 * t + c] = g[t].ctr[c];
        }
        if (area) area[t] = g[t].area;
        if (maxl) maxl[t] = g[t].maxL;
    }
    return EBEM_OK;
}

int ebem_mesh_cache_info(const ebem_mesh* m, int* rules_cached, long long* device_bytes) {
    if (!m) return fail(EBEM_ERR_INVALID, "mesh is NULL");
    static const int kSlotRule[MeshData::kNodeRules] = {1, 3, 7, 12, 19, 28};
    const MeshData& d = m->d;
    long long bytes = (long long)sizeof(double) * 3 * d.nv + (long long)sizeof(int32_t) * 3 * d.nt +
                      (long long)sizeof(TriGeom) * d.nt;
    int mask = 0;
    for (int k = 0; k < MeshData::kNodeRules; k++)
        if (d.d_node_tables[k]) {
            mask |= 1 << k;
            bytes += 32LL * d.nt * kSlotRule[k];
        }
    for (int k = 0; k < MeshData::kCompRules; k++)
        if (d.d_comp_tables[k])
            bytes += 32LL * d.nt * (d.comp_key[k] / 4096) * (d.comp_key[k] % 4096);
    if (d.d_dir) bytes += (long long)sizeof(DirTri) * d.nt + (long long)sizeof(int32_t) * (d.nv + 1 + 3LL * d.nt);
    if (rules_cached) *rules_cached = mask;
    if (device_bytes) *device_bytes = bytes;
    return EBEM_OK;
}

int ebem_num_blocks(const ebem_mesh* m, const ebem_problem* p, int* num_blocks) {
    if (!m || !num_blocks) return fail(EBEM_ERR_INVALID, "NULL argument");
    if (int rc = check_problem(p)) return rc;
    DeviceGuard dg(m->d.device);
    unsigned long long* d = nullptr;
    EBEM_CUDA_TRY(ws_malloc(&d, sizeof(unsigned long long), 0));
    unsigned long long bits = 0;
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(unsigned long long), 0);
    if (e == cudaSuccess) {
        max_vertex_dist_kernel<<<296, 256>>>(m->d.d_coords, m->d.nv, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost);
    ws_free(d, 0);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, cudaGetErrorString(e));
    double maxD;
    std::memcpy(&maxD, &bits, sizeof(double));
    PhysParams P = phys_from(p);
    long long maxInd = (long long)std::ceil(maxD / (P.velS * P.dt)) + 1;
    *num_blocks = (int)std::min<long long>(p->nt, maxInd);
    return EBEM_OK;
}

static int assemble_impl(const ebem_mesh* m, const ebem_problem* p, int n_gh, int lag0, int nlag, int src0,
                         int nsrc, double* E, long long ld, int accumulate, void* stream, long long* nonnull,
                         int prec = EBEM_PREC_FP64) {
    if (!m || !E) return fail(EBEM_ERR_INVALID, "NULL mesh or output");
    if (int rc = check_problem(p)) return rc;
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19)
        return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    if (src0 < 0 || nsrc < 1 || src0 + nsrc > m->d.nt) return fail(EBEM_ERR_INVALID, "source panel outside the mesh");
    if (ld < 3LL * nsrc) return fail(EBEM_ERR_INVALID, "leading dimension smaller than 3 nsrc");
    if (prec != EBEM_PREC_FP64 && prec != EBEM_PREC_MIXED) return fail(EBEM_ERR_INVALID, "unknown precision mode");
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = reject_count_under_capture(nonnull, s)) return rc;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = map_nodes(md, n_gh, s)) return rc;
    PhysParams P = phys_from(p);
    const size_t n3 = 3 * (size_t)md.nt;
    const size_t lag_elems = (size_t)ld * n3;
    unsigned long long* d_count = nullptr;
    if (nonnull) {
        EBEM_CUDA_TRY(ws_malloc(&d_count, sizeof(unsigned long long), s));
        cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) {
            ws_free(d_count, s);
            return fail(EBEM_ERR_CUDA, std::string("pair counter: ") + cudaGetErrorString(e));
        }
    }
    int rc = EBEM_OK;
    const bool dev_out = is_device_ptr(E);
    // Host outputs are assembled in source-row sub-panels into two compact
    // device buffers (leading dimension 3 x rows) in turn; each is copied into
    // place (a 2D copy into the strided output) on a second stream while the
    // next one is assembled.  Device outputs are written in place unless the
    // library is built with EBEM_STAGE_DEVICE_OUTPUT=1, which stages those of
    // 1 GiB or more the same way: the assembly alone is faster into compact
    // sub-panels (sphere of 1280 triangles, L = 40: 196 ms against 204.5 ms),
    // but with the device-to-device copies running beside it a step took
    // 195 ms in one run and 217 ms in another, against a steady 204-206 ms in
    // place.
    const bool stage = !dev_out || (EBEM_STAGE_DEVICE_OUTPUT && nsrc >= 16 &&
                                    (size_t)ld * n3 * nlag * sizeof(double) >= ((size_t)1 << 30));
    if (!stage) {
        rc = launch_sa_assemble(md, P, n_gh, lag0, nlag, src0, nsrc, E, (size_t)ld, lag_elems, accumulate, d_count, s, 0,
                                prec == EBEM_PREC_MIXED);
    } else {
        if (!dev_out && ld != 3LL * nsrc) {
            ws_free(d_count, s);
            return fail(EBEM_ERR_INVALID, "host output needs ld == 3 nsrc");
        }
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t cols = n3 * (size_t)nlag;                     // columns of all lags
        const size_t per_row = 3 * cols * sizeof(double);          // one source triangle, all lags
        size_t budget = std::min<size_t>(free_b / 2, (size_t)16 << 30) / 2;   // per buffer
        if (dev_out) budget = std::min<size_t>(budget, (size_t)1 << 30);
        int rows = (int)std::max<size_t>(1, std::min<size_t>(budget / per_row, (size_t)(nsrc + 7) / 8));
        rows = std::min(rows, nsrc);
        // sub-panels of `rows` source rows, the remainder halved down to about
        // rows / 8: the copy of the last sub-panel overlaps nothing, so it is
        // kept short (1280 sources: 7 x 160, then 80, 40, 20, 20)
        std::vector<std::pair<int, int>> parts;             // (first row, rows)
        {
            int r0 = 0;
            while (nsrc - r0 > rows) { parts.push_back({r0, rows}); r0 += rows; }
            int rest = nsrc - r0;
            const int tail = std::max(1, rows / 8);
            while (rest > tail) {
                const int nr = (rest + 1) / 2;
                parts.push_back({r0, nr});
                r0 += nr;
                rest -= nr;
            }
            if (rest > 0) parts.push_back({r0, rest});
        }
        double* buf[2] = {nullptr, nullptr};
        cudaStream_t cs = nullptr;
        cudaEvent_t done[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
        // every part has at most `rows` rows; a second buffer exactly when there
        // is a second part
        bool ok = ws_malloc(&buf[0], per_row * rows, s) == cudaSuccess &&
                  (parts.size() < 2 || ws_malloc(&buf[1], per_row * rows, s) == cudaSuccess) &&
                  cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess;
        for (int b = 0; ok && b < 2; b++)
            ok = cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            if (!dev_out) rc = fail(EBEM_ERR_NOMEM, "device staging buffer allocation failed");
        }
        for (int k = 0; ok && rc == EBEM_OK && k < (int)parts.size(); k++) {
            const int r0 = parts[k].first, nr = parts[k].second, b = k & 1;
            const size_t ldb = 3 * (size_t)nr;
            double* hE = E + 3 * (size_t)r0;
            cudaError_t e = cudaSuccess;
            if (k >= 2) e = cudaStreamWaitEvent(s, copied[b], 0);
            if (e == cudaSuccess && accumulate)
                e = cudaMemcpy2DAsync(buf[b], ldb * sizeof(double), hE, (size_t)ld * sizeof(double), ldb * sizeof(double),
                                      cols, cudaMemcpyDefault, s);
            if (e != cudaSuccess) { rc = fail(EBEM_ERR_CUDA, "upload failed"); break; }
            rc = launch_sa_assemble(md, P, n_gh, lag0, nlag, src0 + r0, nr, buf[b], ldb, ldb * n3, accumulate, d_count,
                                    s, 0, prec == EBEM_PREC_MIXED);
            if (rc) break;
            e = cudaEventRecord(done[b], s);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, done[b], 0);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(hE, (size_t)ld * sizeof(double), buf[b], ldb * sizeof(double), ldb * sizeof(double),
                                      cols, cudaMemcpyDefault, cs);
            if (e == cudaSuccess) e = cudaEventRecord(copied[b], cs);
            if (e != cudaSuccess) { rc = fail(EBEM_ERR_CUDA, "download failed"); break; }
        }
        cudaError_t e = cs ? cudaStreamSynchronize(cs) : cudaSuccess;
        cudaError_t e2 = cudaStreamSynchronize(s);
        if (e == cudaSuccess) e = e2;
        for (int b = 0; b < 2; b++) {
            if (done[b]) cudaEventDestroy(done[b]);
            if (copied[b]) cudaEventDestroy(copied[b]);
            ws_free(buf[b], s);          // both streams have finished with it
        }
        if (cs) cudaStreamDestroy(cs);
        if (rc == EBEM_OK && e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, cudaGetErrorString(e));
        // a device output without room for the staging buffers: written in place
        if (!ok && dev_out && rc == EBEM_OK)
            rc = launch_sa_assemble(md, P, n_gh, lag0, nlag, src0, nsrc, E, (size_t)ld, lag_elems, accumulate, d_count, s,
                                    0, prec == EBEM_PREC_MIXED);
    }
    if (d_count) {
        unsigned long long c = 0;
        cudaError_t e = cudaMemcpyAsync(&c, d_count, sizeof(c), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        ws_free(d_count, s);
        if (rc == EBEM_OK && e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, cudaGetErrorString(e));
        *nonnull = (long long)c;
    }
    return rc;
}

int ebem_assemble_sa(const ebem_mesh* m, const ebem_problem* p, int n_gh, int lag0, int nlag, double* E,
                     int accumulate, void* stream, long long* nonnull) {
    if (!m) return fail(EBEM_ERR_INVALID, "mesh is NULL");
    return assemble_impl(m, p, n_gh, lag0, nlag, 0, m->d.nt, E, 3LL * m->d.nt, accumulate, stream, nonnull);
}

int ebem_assemble_ghc(const ebem_mesh* m, const ebem_problem* p, int n_gh, int n_sub, int n_sing, int lag0,
                      int nlag, double* E, int sa_diagonal, void* stream) {
    if (!m || !E) return fail(EBEM_ERR_INVALID, "NULL mesh or output");
    if (int rc = check_problem(p)) return rc;
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19) return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    if ((n_sub != 1 && n_sub != 4 && n_sub != 16 && n_sub != 64) ||
        (n_sing != 1 && n_sing != 3 && n_sing != 7 && n_sing != 12 && n_sing != 19))
        return fail(EBEM_ERR_INVALID, "inner rule: n_sub in {1,4,16,64}, n_sing in {1,3,7,12,19}");
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    PhysParams P = phys_from(p);
    const size_t n3 = 3 * (size_t)md.nt;
    DevOut out;
    if (int rc = out.init(E, n3 * n3 * nlag, s)) return rc;
    if (out.host) EBEM_CUDA_TRY(cudaMemcpyAsync(out.d, E, n3 * n3 * nlag * sizeof(double), cudaMemcpyHostToDevice, s));
    if (int rc = launch_ghc_assemble(md, P, n_gh, n_sub, n_sing, lag0, nlag, out.d, n3, n3 * n3, s)) return rc;
    if (sa_diagonal) {
        if (int rc = map_nodes(md, n_gh, s)) return rc;
        if (int rc = launch_sa_assemble(md, P, n_gh, lag0, nlag, 0, md.nt, out.d, n3, n3 * n3, 0, nullptr, s, 1)) return rc;
    }
    return out.finish(s);
}

int ebem_rhs(const ebem_mesh* m, const ebem_problem* p, int n_gh, int datum, double* rhs, void* stream) {
    if (!m || !rhs) return fail(EBEM_ERR_INVALID, "NULL mesh or output");
    if (int rc = check_problem(p)) return rc;
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19) return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    if (datum < 0 || datum > 8) return fail(EBEM_ERR_INVALID, "unknown datum id (0..8)");
    if (datum == 8 && (m->lo[0] < -1 || m->hi[0] > 1 || m->lo[1] < -1 || m->hi[1] > 1 || m->lo[2] != 0 || m->hi[2] != 0))
        return fail(EBEM_ERR_INVALID, "datum 8 (TEST) is defined on the screen [-1,1]^2 at z = 0");
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = map_nodes(md, n_gh, s)) return rc;
    PhysParams P = phys_from(p);
    DevOut out;
    if (int rc = out.init(rhs, 3 * (size_t)md.nt * P.nT, s)) return rc;
    if (int rc = launch_rhs(md, P, n_gh, datum, out.d, s)) return rc;
    return out.finish(s);
}

int ebem_march(const double* E, int n3, int L, const double* rhs, int nT, double* phi, void* stream) {
    if (!E || !rhs || !phi || n3 < 1 || L < 1 || nT < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_device()) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevIn dE, dr;
    if (int rc = dE.init(E, (size_t)n3 * n3 * L, s)) return rc;
    if (int rc = dr.init(rhs, (size_t)n3 * nT, s)) return rc;
    DevOut out;
    if (int rc = out.init(phi, (size_t)n3 * nT, s)) return rc;
    if (int rc = march_device(dE.d, n3, L, dr.d, nT, out.d, s)) return rc;
    return out.finish(s);
}

int ebem_march_ex(const double* E, int n3, int L, const double* rhs, int nT, double* phi, int factor, void* stream) {
    if (!E || !rhs || !phi || n3 < 1 || L < 1 || nT < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (factor != EBEM_FACTOR_LU && factor != EBEM_FACTOR_CHOLESKY)
        return fail(EBEM_ERR_INVALID, "factor must be EBEM_FACTOR_LU or EBEM_FACTOR_CHOLESKY");
    if (int rc = check_device()) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevIn dE, dr;
    if (int rc = dE.init(E, (size_t)n3 * n3 * L, s)) return rc;
    if (int rc = dr.init(rhs, (size_t)n3 * nT, s)) return rc;
    DevOut out;
    if (int rc = out.init(phi, (size_t)n3 * nT, s)) return rc;
    if (int rc = march_device(dE.d, n3, L, dr.d, nT, out.d, s, factor)) return rc;
    return out.finish(s);
}

struct ebem_banded {
    BandOp op;
    int device = 0;
};

int ebem_banded_assemble(const ebem_mesh* m, const ebem_problem* p, int n_gh, int prec, void* stream,
                         ebem_banded** out) {
    if (!out) return fail(EBEM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!m) return fail(EBEM_ERR_INVALID, "mesh is NULL");
    if (int rc = check_problem(p)) return rc;
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19)
        return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    if (prec != EBEM_PREC_FP64 && prec != EBEM_PREC_MIXED) return fail(EBEM_ERR_INVALID, "unknown precision mode");
    int L = 0;
    if (int rc = ebem_num_blocks(m, p, &L)) return rc;
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = map_nodes(md, n_gh, s)) return rc;
    PhysParams P = phys_from(p);
    ebem_banded* b = new ebem_banded();
    b->device = m->d.device;
    int rc = band_structure(md, P, L, &b->op, s);
    if (!rc) rc = launch_sa_assemble_banded(md, P, n_gh, L, b->op.Eb, b->op.off, b->op.lo, prec == EBEM_PREC_MIXED, s);
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(EBEM_ERR_CUDA, "banded assembly failed");
    if (rc) {
        band_free(&b->op);
        delete b;
        return rc;
    }
    *out = b;
    return EBEM_OK;
}

int ebem_banded_info(const ebem_banded* b, int* n_triangles, int* num_blocks, long long* nonnull, long long* bytes) {
    if (!b) return fail(EBEM_ERR_INVALID, "NULL operator");
    if (n_triangles) *n_triangles = b->op.N;
    if (num_blocks) *num_blocks = b->op.L;
    if (nonnull) *nonnull = b->op.nblocks;
    if (bytes) {
        const long long NN = (long long)b->op.N * b->op.N;
        *bytes = b->op.nblocks * 48 + (NN + 1) * 8 + NN * 4;
    }
    return EBEM_OK;
}

int ebem_banded_to_dense(const ebem_banded* b, int lag0, int nlag, double* E, void* stream) {
    if (!b || !E) return fail(EBEM_ERR_INVALID, "NULL argument");
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    DeviceGuard dg(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n3 = 3 * (size_t)b->op.N;
    DevOut out;
    if (int rc = out.init(E, n3 * n3 * nlag, s)) return rc;
    if (int rc = band_to_dense(b->op, lag0, nlag, out.d, s)) return rc;
    return out.finish(s);
}

int ebem_banded_march(const ebem_banded* b, const double* rhs, int nT, double* phi, void* stream) {
    if (!b || !rhs || !phi || nT < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    DeviceGuard dg(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n3 = 3 * (size_t)b->op.N;
    DevIn dr;
    if (int rc = dr.init(rhs, n3 * nT, s)) return rc;
    DevOut out;
    if (int rc = out.init(phi, n3 * nT, s)) return rc;
    if (int rc = band_march(b->op, dr.d, nT, out.d, s)) return rc;
    return out.finish(s);
}

void ebem_banded_destroy(ebem_banded* b) {
    if (!b) return;
    DeviceGuard dg(b->device);
    band_free(&b->op);
    delete b;
}

struct ebem_lu {
    LuPlan plan;
    int device = 0;
};

int ebem_lu_create(const double* A, int n, void* stream, ebem_lu** out) {
    if (!out) return fail(EBEM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!A || n < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_device()) return rc;
    if (int rc = need_device(A, "the matrix")) return rc;
    ebem_lu* lu = new ebem_lu();
    cudaGetDevice(&lu->device);
    if (int rc = lu_plan_create(A, n, (cudaStream_t)stream, &lu->plan)) {
        lu_plan_destroy(&lu->plan);
        delete lu;
        return rc;
    }
    *out = lu;
    return EBEM_OK;
}

int ebem_lu_solve(ebem_lu* lu, double* b, int nrhs, void* stream) {
    if (!lu || !b || nrhs < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    DeviceGuard dg(lu->device);
    if (int rc = need_device(b, "the right-hand side")) return rc;
    return lu_plan_solve(&lu->plan, b, nrhs, (cudaStream_t)stream);
}

void ebem_lu_destroy(ebem_lu* lu) {
    if (!lu) return;
    DeviceGuard dg(lu->device);
    lu_plan_destroy(&lu->plan);
    delete lu;
}

int ebem_history_gemv(const double* A, int rows, long long K, const double* x, double* y, void* stream) {
    if (!A || !x || !y || rows < 1 || K < 0) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_device()) return rc;
    for (const void* q : {(const void*)A, (const void*)x, (const void*)y})
        if (int rc = need_device(q, "A, x and y")) return rc;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return launch_hist_gemv(A, rows, K, x, y, sms, (cudaStream_t)stream);
}

static int timemarch_impl(const ebem_mesh* m, const ebem_problem* p, int n_gh, int datum, double* phi, int* num_blocks,
                          void* stream, int prec);

int ebem_timemarch_sa(const ebem_mesh* m, const ebem_problem* p, int n_gh, int datum, double* phi, int* num_blocks,
                      void* stream) {
    return timemarch_impl(m, p, n_gh, datum, phi, num_blocks, stream, EBEM_PREC_FP64);
}

int ebem_timemarch_sa_ex(const ebem_mesh* m, const ebem_problem* p, int n_gh, int datum, int prec, double* phi,
                         int* num_blocks, void* stream) {
    return timemarch_impl(m, p, n_gh, datum, phi, num_blocks, stream, prec);
}

static int timemarch_impl(const ebem_mesh* m, const ebem_problem* p, int n_gh, int datum, double* phi, int* num_blocks,
                          void* stream, int prec) {
    if (!m || !phi) return fail(EBEM_ERR_INVALID, "NULL mesh or output");
    if (int rc = check_problem(p)) return rc;
    int L = 0;
    if (int rc = ebem_num_blocks(m, p, &L)) return rc;
    if (num_blocks) *num_blocks = L;
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n3 = 3 * (size_t)m->d.nt;
    double *dE = nullptr, *dr = nullptr;
    if (cudaMalloc(&dE, n3 * n3 * L * sizeof(double)) != cudaSuccess || cudaMalloc(&dr, n3 * p->nt * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        if (dE) cudaFree(dE);
        return fail(EBEM_ERR_NOMEM, "device allocation of E or the right-hand side failed");
    }
    int rc = assemble_impl(m, p, n_gh, 0, L, 0, m->d.nt, dE, 3LL * m->d.nt, 0, stream, nullptr, prec);
    if (!rc) rc = ebem_rhs(m, p, n_gh, datum, dr, stream);
    if (!rc) rc = ebem_march(dE, (int)n3, L, dr, p->nt, phi, stream);
    cudaStreamSynchronize(s);
    cudaFree(dE);
    cudaFree(dr);
    return rc;
}

int ebem_pp_sa(const ebem_mesh* m, const ebem_problem* p, const double* phi, const double* pts, int npts,
               const double* times, int ntimes, double* u, void* stream) {
    if (!m || !phi || !pts || !times || !u || npts < 1 || ntimes < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_problem(p)) return rc;
    if (is_device_ptr(times)) return fail(EBEM_ERR_INVALID, "times must be a host array");
    // u(x, t) uses density column ceil(t / dt) (BEMenerg_postProcA_singlePoint.m:21,58),
    // which exists for t <= tfin; the reference fails past it
    for (int q = 0; q < ntimes; q++)
        if (!(times[q] <= p->tfin * (1 + 1e-12))) return fail(EBEM_ERR_INVALID, "evaluation time beyond tfin");
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    PhysParams P = phys_from(p);
    DevIn dphi, dpts;
    if (int rc = dphi.init(phi, 3 * (size_t)m->d.nt * P.nT, s)) return rc;
    if (int rc = dpts.init(pts, 3 * (size_t)npts, s)) return rc;
    DevOut out;
    if (int rc = out.init(u, 3 * (size_t)npts * ntimes, s)) return rc;
    if (int rc = launch_pp_sa(m->d, P, dphi.d, dpts.d, npts, times, ntimes, out.d, s)) return rc;
    return out.finish(s);
}

int ebem_assemble_sa_panel(const ebem_mesh* m, const ebem_problem* p, int n_gh, int lag0, int nlag, int src0,
                           int nsrc, double* E, long long ld, int accumulate, void* stream, long long* nonnull) {
    return assemble_impl(m, p, n_gh, lag0, nlag, src0, nsrc, E, ld, accumulate, stream, nonnull);
}

int ebem_assemble_sa_ex(const ebem_mesh* m, const ebem_problem* p, int n_gh, int lag0, int nlag, int src0, int nsrc,
                        double* E, long long ld, int accumulate, int prec, void* stream, long long* nonnull) {
    return assemble_impl(m, p, n_gh, lag0, nlag, src0, nsrc, E, ld, accumulate, stream, nonnull, prec);
}

// ---------------------------------------------------------------------------
// direct formulation

static int check_rules(int n_gh, int n_sub, int n_sing, int n_diag) {
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19) return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    if ((n_sub != 1 && n_sub != 4 && n_sub != 16 && n_sub != 64) ||
        (n_sing != 1 && n_sing != 3 && n_sing != 7 && n_sing != 12 && n_sing != 19))
        return fail(EBEM_ERR_INVALID, "inner rule: n_sub in {1,4,16,64}, n_sing in {1,3,7,12,19}");
    if (n_diag != 0 && n_diag != 16 && n_diag != 64 && n_diag != 256 && n_diag != 1024)
        return fail(EBEM_ERR_INVALID, "DIAG rule: n_diag in {16,64,256,1024} (0: none)");
    return EBEM_OK;
}

int ebem_pp_gpu(const ebem_mesh* m, const ebem_problem* p, int n_sub, int n_sing, int variant, int flags,
                const double* phi, const double* pts, int npts, const double* times, int ntimes, double* u,
                void* stream) {
    if (!m || !phi || !pts || !times || !u || npts < 1 || ntimes < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_problem(p)) return rc;
    if (int rc = check_rules(3, n_sub, n_sing, 0)) return rc;
    if (variant != EBEM_PP_POINT && variant != EBEM_PP_LAYER)
        return fail(EBEM_ERR_INVALID, "variant must be EBEM_PP_POINT or EBEM_PP_LAYER");
    if (is_device_ptr(times)) return fail(EBEM_ERR_INVALID, "times must be a host array");
    // the sums read density column ceil(t / dt) (BEMenerg_postProcGPU_calcSP.m:85), which exists for t <= tfin
    for (int q = 0; q < ntimes; q++)
        if (!(times[q] <= p->tfin * (1 + 1e-12))) return fail(EBEM_ERR_INVALID, "evaluation time beyond tfin");
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    PhysParams P = phys_from(p);
    DevIn dphi, dpts;
    if (int rc = dphi.init(phi, 3 * (size_t)m->d.nt * P.nT, s)) return rc;
    if (int rc = dpts.init(pts, 3 * (size_t)npts, s)) return rc;
    DevOut out;
    if (int rc = out.init(u, 3 * (size_t)npts * ntimes, s)) return rc;
    if (int rc = launch_pp_num(m->d, P, n_sub, n_sing, variant == EBEM_PP_LAYER, flags & EBEM_FIX_REFERENCE_DEFECTS,
                               dphi.d, dpts.d, npts, times, ntimes, out.d, s))
        return rc;
    return out.finish(s);
}

int ebem_num_blocks_dir(const ebem_mesh* m, const ebem_problem* p, int* lv, int* lk) {
    int L = 0;
    if (int rc = ebem_num_blocks(m, p, &L)) return rc;
    if (lv) *lv = L;
    if (lk) *lk = std::min(L + 1, p->nt);
    return EBEM_OK;
}

int ebem_assemble_k(const ebem_mesh* m, const ebem_problem* p, int n_gh, int n_sub, int n_sing, int n_diag, int lag0,
                    int nlag, int flags, double* K, int accumulate, void* stream) {
    if (!m || !K) return fail(EBEM_ERR_INVALID, "NULL mesh or output");
    if (int rc = check_problem(p)) return rc;
    if (int rc = check_rules(n_gh, n_sub, n_sing, n_diag)) return rc;
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    int LK = 0;
    if (int rc = ebem_num_blocks_dir(m, p, nullptr, &LK)) return rc;
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = prep_direct(md, s)) return rc;
    PhysParams P = phys_from(p);
    const size_t n = 9 * (size_t)md.nt * md.nv * nlag;
    DevOut out;
    if (int rc = out.init(K, n, s)) return rc;
    if (accumulate) {
        if (out.host) EBEM_CUDA_TRY(cudaMemcpyAsync(out.d, K, n * sizeof(double), cudaMemcpyHostToDevice, s));
    } else {
        EBEM_CUDA_TRY(cudaMemsetAsync(out.d, 0, n * sizeof(double), s));
    }
    if (int rc = launch_k_assemble(md, P, n_gh, n_sub, n_sing, n_diag, lag0, nlag, LK, flags & EBEM_FIX_REFERENCE_DEFECTS,
                                   out.d, s))
        return rc;
    return out.finish(s);
}

int ebem_assemble_v(const ebem_mesh* m, const ebem_problem* p, int n_gh, int n_sub, int n_sing, int n_diag, int lag0,
                    int nlag, double* V, void* stream) {
    if (!m || !V) return fail(EBEM_ERR_INVALID, "NULL mesh or output");
    if (int rc = check_problem(p)) return rc;
    if (int rc = check_rules(n_gh, n_sub, n_sing, n_diag)) return rc;
    if (n_diag == 0) return fail(EBEM_ERR_INVALID, "the direct V operator needs a DIAG rule for its diagonal blocks");
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = prep_direct(md, s)) return rc;
    PhysParams P = phys_from(p);
    const size_t n3 = 3 * (size_t)md.nt;
    DevOut out;
    if (int rc = out.init(V, n3 * n3 * nlag, s)) return rc;
    EBEM_CUDA_TRY(cudaMemsetAsync(out.d, 0, n3 * n3 * nlag * sizeof(double), s));
    if (int rc = launch_ghc_assemble(md, P, n_gh, n_sub, n_sing, lag0, nlag, out.d, n3, n3 * n3, s)) return rc;
    if (int rc = launch_v_diag(md, P, n_gh, n_diag, lag0, nlag, out.d, s)) return rc;
    return out.finish(s);
}

int ebem_march_dn(const ebem_mesh* m, const ebem_problem* p, const double* V, int LV, const double* K, int LK,
                  const double* gV, double* u, void* stream) {
    if (!m || !V || !K || !gV || !u || LV < 1 || LK < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_problem(p)) return rc;
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = prep_direct(md, s)) return rc;
    const size_t R = 3 * (size_t)md.nt, Cn = 3 * (size_t)md.nv;
    DevIn dV, dK, dgv;
    if (int rc = dV.init(V, R * R * LV, s)) return rc;
    if (int rc = dK.init(K, R * Cn * LK, s)) return rc;
    if (int rc = dgv.init(gV, R * p->nt, s)) return rc;
    DevOut out;
    if (int rc = out.init(u, Cn * p->nt, s)) return rc;
    if (int rc = march_dn_device(md, dV.d, LV, dK.d, LK, dgv.d, p->nt, out.d, s)) return rc;
    return out.finish(s);
}

int ebem_march_dd(const ebem_mesh* m, const ebem_problem* p, const double* V, int LV, const double* K, int LK,
                  const double* rhs, const double* gK, double* phi, void* stream) {
    if (!m || !V || !K || !rhs || !gK || !phi || LV < 1 || LK < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_problem(p)) return rc;
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = prep_direct(md, s)) return rc;
    const size_t R = 3 * (size_t)md.nt, Cn = 3 * (size_t)md.nv;
    DevIn dV, dK, dr, dgk;
    if (int rc = dV.init(V, R * R * LV, s)) return rc;
    if (int rc = dK.init(K, R * Cn * LK, s)) return rc;
    if (int rc = dr.init(rhs, R * p->nt, s)) return rc;
    if (int rc = dgk.init(gK, Cn * p->nt, s)) return rc;
    DevOut out;
    if (int rc = out.init(phi, R * p->nt, s)) return rc;
    if (int rc = march_dd_device(md, dV.d, LV, dK.d, LK, dr.d, dgk.d, p->nt, out.d, s)) return rc;
    return out.finish(s);
}

int ebem_pp_dir(const ebem_mesh* m, const ebem_problem* p, int n_sub, int n_sing, int flags, const double* a,
                const double* b, const double* pts, int npts, const double* times, int ntimes, double* u, void* stream) {
    if (!m || !a || !b || !pts || !times || !u || npts < 1 || ntimes < 1) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_problem(p)) return rc;
    if (int rc = check_rules(3, n_sub, n_sing, 0)) return rc;
    if (is_device_ptr(times)) return fail(EBEM_ERR_INVALID, "times must be a host array");
    for (int q = 0; q < ntimes; q++)
        if (!(times[q] <= p->tfin * (1 + 1e-12))) return fail(EBEM_ERR_INVALID, "evaluation time beyond tfin");
    DeviceGuard dg(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = prep_direct(md, s)) return rc;
    PhysParams P = phys_from(p);
    DevIn da, db, dp;
    if (int rc = da.init(a, 3 * (size_t)md.nt * P.nT, s)) return rc;
    if (int rc = db.init(b, 3 * (size_t)md.nv * P.nT, s)) return rc;
    if (int rc = dp.init(pts, 3 * (size_t)npts, s)) return rc;
    DevOut out;
    if (int rc = out.init(u, 3 * (size_t)npts * ntimes, s)) return rc;
    if (int rc = launch_pp_dir(md, P, n_sub, n_sing, flags & EBEM_FIX_REFERENCE_DEFECTS, dp.d, npts, times, ntimes, da.d,
                               db.d, out.d, nullptr, nullptr, 0, s))
        return rc;
    return out.finish(s);
}

int ebem_pp_dir_matrices(const ebem_mesh* m, const ebem_problem* p, int n_sub, int n_sing, int flags, const double* x,
                         double t, double* G, double* Pm) {
    if (!m || !x || !G || !Pm) return fail(EBEM_ERR_INVALID, "bad arguments");
    if (int rc = check_problem(p)) return rc;
    if (int rc = check_rules(3, n_sub, n_sing, 0)) return rc;
    if (!(t > 0)) return EBEM_OK;
    DeviceGuard dg(m->d.device);
    cudaStream_t s = 0;
    MeshData& md = const_cast<MeshData&>(m->d);
    if (int rc = prep_direct(md, s)) return rc;
    PhysParams P = phys_from(p);
    const int nhat = (int)std::ceil(t / P.dt);
    DevIn dx;
    if (int rc = dx.init(x, 3, s)) return rc;
    DevOut oG, oP;
    if (int rc = oG.init(G, 9 * (size_t)nhat * md.nt, s)) return rc;
    if (int rc = oP.init(Pm, 9 * (size_t)nhat * md.nv, s)) return rc;
    EBEM_CUDA_TRY(cudaMemsetAsync(oG.d, 0, 9 * (size_t)nhat * md.nt * sizeof(double), s));
    EBEM_CUDA_TRY(cudaMemsetAsync(oP.d, 0, 9 * (size_t)nhat * md.nv * sizeof(double), s));
    if (int rc = launch_pp_dir(md, P, n_sub, n_sing, flags & EBEM_FIX_REFERENCE_DEFECTS, dx.d, 1, &t, 1, nullptr,
                               nullptr, nullptr, oG.d, oP.d, 1, s))
        return rc;
    if (int rc = oG.finish(s)) return rc;
    return oP.finish(s);
}

// Full semi-analytic assembly that allocates no device memory of its own (for
// callers that may not allocate on the device during the call); see
// ebem_assemble_sa_noalloc in include/ebem.h.
int ebem_assemble_sa_noalloc(const ebem_mesh* m, const ebem_problem* p, int n_gh, int lag0, int nlag, double* E,
                             int accumulate, void* stream, long long* nonnull) {
    if (!m || !E) return fail(EBEM_ERR_INVALID, "NULL mesh or output");
    if (int rc = check_problem(p)) return rc;
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19)
        return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    DeviceGuard dg(m->d.device);
    if (int rc = need_device(E, "the output of the allocation-free assembly")) return rc;
    if (int rc = reject_count_under_capture(nonnull, (cudaStream_t)stream)) return rc;
    PhysParams P = phys_from(p);
    unsigned long long c = 0;
    int rc = launch_sa_assemble_noalloc(m->d, P, n_gh, lag0, nlag, E, accumulate, nonnull != nullptr, &c,
                                        (cudaStream_t)stream);
    if (rc == EBEM_OK && nonnull) *nonnull = (long long)c;
    return rc;
}

// ---------------------------------------------------------------------------
// batched assembly plans

}  // extern "C"

struct ebem_batch {
    int device = 0, n = 0, n_gh = 0, prec = 0;
    std::vector<const ebem_mesh*> meshes;
    std::vector<int> nlag;
    BatchInst* h_insts = nullptr;          // pinned host copy of the table
    BatchInst* d_insts = nullptr;
    unsigned long long* d_next = nullptr;  // work counter, reset inside the graph
    long long total = 0;
    std::vector<PhysParams> params;
    int wpb = 4, chunk = 4;
    // schedule: 0 the persistent launch over all instances, 1 one two-pass
    // assembly per instance (captured in the same way; its graph holds the
    // output pointers, so new outputs mean a new capture)
    int sched = 0;
    std::vector<double*> cap_E;            // outputs of the captured per-instance schedule
    float tuned_ms = -1.0f;
    bool tuned = false;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

// One two-pass assembly per instance (the single-mesh path: level pass and
// whole-sector emission), on the rule table the plan recorded.
int batch_run_twopass(ebem_batch* b, cudaStream_t s) {
    for (int k = 0; k < b->n; k++) {
        const BatchInst& I = b->h_insts[k];
        MeshData m = b->meshes[k]->d;
        m.d_nodes = const_cast<NodeW*>(I.nodes);
        m.nodes_rule = b->n_gh;
        const size_t n3 = 3 * (size_t)I.N;
        if (int rc = launch_sa_twopass(m, b->params[k], b->n_gh, 0, I.nlag, 0, I.N, I.E, n3, n3 * n3, 0, nullptr,
                                       b->prec == EBEM_PREC_MIXED, s))
            return rc;
    }
    return EBEM_OK;
}

int batch_run_direct(ebem_batch* b, int wpb, int chunk, cudaStream_t s) {
    EBEM_CUDA_TRY(cudaMemsetAsync(b->d_next, 0, sizeof(unsigned long long), s));
    return launch_sa_batch(b->d_insts, b->n, b->total, b->n_gh, b->prec == EBEM_PREC_MIXED, wpb, chunk, b->d_next,
                           b->device, s);
}

// Autotuner: time every (warps per block, pairs per grab) candidate once on the
// batch itself and keep the fastest, then capture the launch in a CUDA graph.
// Captures the chosen schedule into b->graph / b->exec (replacing any earlier one).
int batch_capture(ebem_batch* b) {
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    if (!b->cap) EBEM_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    EBEM_CUDA_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    int crc = b->sched == 1 ? batch_run_twopass(b, b->cap) : batch_run_direct(b, b->wpb, b->chunk, b->cap);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (crc) { if (g) cudaGraphDestroy(g); return crc; }
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) return fail(EBEM_ERR_CUDA, std::string("batch graph instantiation: ") + cudaGetErrorString(e));
    b->cap_E.assign(b->n, nullptr);
    for (int k = 0; k < b->n; k++) b->cap_E[k] = b->h_insts[k].E;
    return EBEM_OK;
}

// Autotuner: time every (warps per block, pairs per grab) candidate of the
// persistent launch, and the per-instance two-pass schedule, once each on the
// batch itself; keep the fastest and capture it in a CUDA graph.
int batch_tune_and_capture(ebem_batch* b, cudaStream_t s) {
    std::vector<int> wpbs = {2, 4};
    const int chunks[3] = {1, 4, 16};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    EBEM_CUDA_TRY(cudaEventCreate(&e0));
    EBEM_CUDA_TRY(cudaEventCreate(&e1));
    int rc = batch_run_direct(b, wpbs.back(), 4, s);          // warm-up (module load, caches)
    if (!rc) rc = batch_run_twopass(b, s);
    float best = 1e30f;
    auto timed = [&](auto&& run) -> float {
        float ms = -1.0f;
        cudaEventRecord(e0, s);
        rc = run();
        cudaEventRecord(e1, s);
        if (!rc && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    for (int w : wpbs)
        for (int c : chunks) {
            if (rc) break;
            const float ms = timed([&] { return batch_run_direct(b, w, c, s); });
            if (ms >= 0.0f && ms < best) { best = ms; b->wpb = w; b->chunk = c; b->sched = 0; }
        }
    if (!rc) {
        const float ms = timed([&] { return batch_run_twopass(b, s); });
        if (ms >= 0.0f && ms < best) { best = ms; b->sched = 1; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    b->tuned_ms = best;
    b->tuned = true;
    rc = batch_capture(b);
    if (rc && b->sched == 1) {
        // the per-instance schedule could not be captured: the persistent launch
        cudaGetLastError();
        b->sched = 0;
        rc = batch_capture(b);
    }
    return rc;
}

}  // namespace

extern "C" {

int ebem_batch_destroy(ebem_batch* b) {
    if (!b) return EBEM_OK;
    DeviceGuard dg(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->d_insts) cudaFree(b->d_insts);
    if (b->d_next) cudaFree(b->d_next);
    if (b->h_insts) cudaFreeHost(b->h_insts);
    delete b;
    return EBEM_OK;
}

int ebem_batch_create(const ebem_mesh* const* meshes, const ebem_problem* probs, const int* nlag, int n, int n_gh,
                      int prec, ebem_batch** out) {
    if (!out) return fail(EBEM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!meshes || !probs || n < 1) return fail(EBEM_ERR_INVALID, "need at least one instance");
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19)
        return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    if (prec != EBEM_PREC_FP64 && prec != EBEM_PREC_MIXED) return fail(EBEM_ERR_INVALID, "unknown precision mode");
    for (int k = 0; k < n; k++) {
        if (!meshes[k]) return fail(EBEM_ERR_INVALID, "NULL mesh in the batch");
        if (int rc = check_problem(&probs[k])) return rc;
        if (meshes[k]->d.device != meshes[0]->d.device) return fail(EBEM_ERR_INVALID, "all meshes of a batch must live on one device");
    }
    ebem_batch* b = new ebem_batch();
    b->device = meshes[0]->d.device;
    b->n = n;
    b->n_gh = n_gh;
    b->prec = prec;
    DeviceGuard dg(b->device);
    auto bail = [&](int rc) { ebem_batch_destroy(b); return rc; };
    if (cudaMallocHost(&b->h_insts, sizeof(BatchInst) * n) != cudaSuccess ||
        cudaMalloc(&b->d_insts, sizeof(BatchInst) * n) != cudaSuccess ||
        cudaMalloc(&b->d_next, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        return bail(fail(EBEM_ERR_NOMEM, "batch table allocation failed"));
    }
    long long begin = 0;
    for (int k = 0; k < n; k++) {
        MeshData& md = const_cast<MeshData&>(meshes[k]->d);
        int L = 0;
        if (int rc = ebem_num_blocks(meshes[k], &probs[k], &L)) return bail(rc);
        const int nl = nlag ? nlag[k] : L;
        if (nl < 1) return bail(fail(EBEM_ERR_INVALID, "each instance needs nlag >= 1"));
        if (int rc = map_nodes(md, n_gh, 0)) return bail(rc);
        PhysParams P = phys_from(&probs[k]);
        BatchInst& I = b->h_insts[k];
        I.geo = md.d_geo;
        I.nodes = md.d_nodes;
        I.E = nullptr;
        I.N = md.nt;
        I.nlag = nl;
        I.velP = P.velP;
        I.velS = P.velS;
        I.dt = P.dt;
        I.c4pirho = 4 * kPi * P.rho;
        I.pair_begin = begin;
        begin += (long long)md.nt * md.nt;
        b->meshes.push_back(meshes[k]);
        b->params.push_back(P);
        b->nlag.push_back(nl);
    }
    b->total = begin;
    *out = b;
    return EBEM_OK;
}

int ebem_batch_assemble(ebem_batch* b, double* const* E, void* stream) {
    if (!b || !E) return fail(EBEM_ERR_INVALID, "NULL batch or outputs");
    DeviceGuard dg(b->device);
    for (int k = 0; k < b->n; k++) {
        if (!E[k]) return fail(EBEM_ERR_INVALID, "batch outputs must be device buffers");
        if (int rc = need_device(E[k], "every batch output")) return rc;
        b->h_insts[k].E = E[k];
    }
    cudaStream_t s = (cudaStream_t)stream;
    // the table (output pointers) is read by the kernel at run time, so a new
    // set of outputs needs no new graph
    EBEM_CUDA_TRY(cudaMemcpyAsync(b->d_insts, b->h_insts, sizeof(BatchInst) * b->n, cudaMemcpyHostToDevice, s));
    if (!b->tuned) {
        if (int rc = batch_tune_and_capture(b, s)) return rc;
    } else if (b->sched == 1) {
        bool same = true;
        for (int k = 0; k < b->n; k++) same = same && b->cap_E[k] == E[k];
        if (!same)
            if (int rc = batch_capture(b)) return rc;
    }
    EBEM_CUDA_TRY(cudaGraphLaunch(b->exec, s));
    // the pinned table must not change before this call's copy has run
    EBEM_CUDA_TRY(cudaStreamSynchronize(s));
    return EBEM_OK;
}

int ebem_batch_info(const ebem_batch* b, int* warps_per_block, int* pairs_per_grab, float* tuned_ms,
                    long long* pairs) {
    if (!b) return fail(EBEM_ERR_INVALID, "batch is NULL");
    // 0 and 0: the per-instance schedule was chosen
    if (warps_per_block) *warps_per_block = b->sched == 1 ? 0 : b->wpb;
    if (pairs_per_grab) *pairs_per_grab = b->sched == 1 ? 0 : b->chunk;
    if (tuned_ms) *tuned_ms = b->tuned_ms;
    if (pairs) *pairs = b->total;
    return EBEM_OK;
}

// ---------------------------------------------------------------------------
// learned quadrature selector

static bool all_device(std::initializer_list<const void*> ps) {
    for (const void* q : ps)
        if (!q || !is_device_ptr(q)) return false;
    return true;
}

int ebem_selector_init(float* params, unsigned long long seed) {
    if (!params) return fail(EBEM_ERR_INVALID, "NULL parameters");
    if (is_device_ptr(params)) {
        std::vector<float> h(EBEM_SELECTOR_PARAMS);
        selector_init(h.data(), seed);
        EBEM_CUDA_TRY(cudaMemcpy(params, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
    } else {
        selector_init(params, seed);
    }
    return EBEM_OK;
}

int ebem_sa_pair_blocks(const ebem_mesh* m, const ebem_problem* p, int n_gh, int n_sub, const int* pairs,
                        long long npairs, int nlag, double* out, void* stream) {
    if (!m || npairs < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "mesh, npairs >= 0 and nlag >= 1 required");
    if (npairs == 0) return EBEM_OK;
    if (!all_device({pairs, out})) return fail(EBEM_ERR_INVALID, "device pair and output buffers required");
    if (int rc = check_problem(p)) return rc;
    if (n_gh < 1 || n_sub < 1) return fail(EBEM_ERR_INVALID, "n_gh and n_sub must be >= 1");
    DeviceGuard dg(m->d.device);
    MeshData& d = const_cast<MeshData&>(m->d);
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = map_nodes_composite(d, n_gh, n_sub, s)) return rc;
    return launch_sa_pair_blocks(d, phys_from(p), n_gh * n_sub, reinterpret_cast<const int2*>(pairs), npairs, nlag, out,
                                 s);
}

int ebem_selector_features(const ebem_mesh* m, const ebem_problem* p, const int* samples, long long n, float* feats,
                           void* stream) {
    if (!m || n < 0) return fail(EBEM_ERR_INVALID, "mesh and n >= 0 required");
    if (n == 0) return EBEM_OK;
    if (!all_device({samples, feats})) return fail(EBEM_ERR_INVALID, "device sample and feature buffers required");
    if (int rc = check_problem(p)) return rc;
    DeviceGuard dg(m->d.device);
    return selector_features(m->d, phys_from(p), samples, n, feats, (cudaStream_t)stream);
}

int ebem_selector_sweeps(const ebem_mesh* m, const ebem_problem* p, const int* samples, long long n,
                         unsigned char* flags, void* stream) {
    if (!m || n < 0) return fail(EBEM_ERR_INVALID, "mesh and n >= 0 required");
    if (n == 0) return EBEM_OK;
    if (!all_device({samples, flags})) return fail(EBEM_ERR_INVALID, "device sample and flag buffers required");
    if (int rc = check_problem(p)) return rc;
    DeviceGuard dg(m->d.device);
    return selector_sweeps(m->d, phys_from(p), samples, n, flags, (cudaStream_t)stream);
}

int ebem_selector_labels(const double* blocks, long long n, double tol, double scale, const double* scales,
                         int* labels, void* stream) {
    if (n < 0 || !(tol >= 0) || !(scale >= 0)) return fail(EBEM_ERR_INVALID, "n, tol and scale must be >= 0");
    if (n == 0) return EBEM_OK;
    if (!all_device({blocks, labels}) || (scales && !all_device({scales})))
        return fail(EBEM_ERR_INVALID, "device block, scale and label buffers required");
    if (int rc = check_device()) return rc;
    return selector_labels(blocks, n, tol, scale, scales, labels, (cudaStream_t)stream);
}

int ebem_selector_grad(const float* params, const float* feats, const int* labels, long long n, float* grad,
                       float* loss, void* stream) {
    if (n < 1 || !all_device({params, feats, labels, grad}) || (loss && !is_device_ptr(loss)))
        return fail(EBEM_ERR_INVALID, "device buffers and n >= 1 required");
    if (int rc = check_device()) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = selector_grad(params, feats, labels, n, grad, loss, s)) return rc;
    EBEM_CUDA_TRY(cudaStreamSynchronize(s));
    return EBEM_OK;
}

int ebem_selector_train(float* params, const float* feats, const int* labels, long long n, int epochs, int batch,
                        float lr, unsigned long long seed, float* losses, void* stream) {
    if (n < 1 || epochs < 1 || batch < 1 || !(lr > 0) || !all_device({params, feats, labels}))
        return fail(EBEM_ERR_INVALID, "device buffers, n, epochs, batch >= 1 and lr > 0 required");
    if (int rc = check_device()) return rc;
    return selector_train(params, feats, labels, n, epochs, batch, lr, seed, losses, (cudaStream_t)stream);
}

int ebem_selector_infer(const float* params, const ebem_mesh* m, const ebem_problem* p, float threshold, int lag0,
                        int nlag, unsigned char* cls, long long* counts, void* stream) {
    if (!m || !all_device({params, cls})) return fail(EBEM_ERR_INVALID, "mesh and device buffers required");
    if (int rc = check_problem(p)) return rc;
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    DeviceGuard dg(m->d.device);
    return selector_infer(params, m->d, phys_from(p), threshold, lag0, nlag, cls, counts, (cudaStream_t)stream);
}

int ebem_assemble_sa_selected(const ebem_mesh* m, const ebem_problem* p, const int* rules, int nclass,
                              const unsigned char* cls, int lag0, int nlag, double* E, int prec, void* stream,
                              long long* counts) {
    if (!m || !rules || !all_device({cls, E})) return fail(EBEM_ERR_INVALID, "mesh, rules and device buffers required");
    if (int rc = check_problem(p)) return rc;
    if (nclass < 1 || nclass > 255) return fail(EBEM_ERR_INVALID, "nclass must be in 1..255");
    for (int c = 0; c < nclass; c++)
        if (rules[2 * c] < 1 || rules[2 * c + 1] < 1) return fail(EBEM_ERR_INVALID, "rule sizes must be >= 1");
    if (lag0 < 0 || nlag < 1) return fail(EBEM_ERR_INVALID, "need lag0 >= 0 and nlag >= 1");
    if (prec != EBEM_PREC_FP64 && prec != EBEM_PREC_MIXED) return fail(EBEM_ERR_INVALID, "unknown precision mode");
    DeviceGuard dg(m->d.device);
    return assemble_selected(const_cast<MeshData&>(m->d), phys_from(p), rules, nclass, cls, lag0, nlag, E, prec, counts,
                             (cudaStream_t)stream);
}

}  // extern "C"
