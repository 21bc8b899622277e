// Internal declarations shared by the CUDA translation units of libebem.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ebem.h"
#include "sa_device.cuh"

namespace ebem { struct NodeW; }

namespace ebem {

// Thread-local error message returned by ebem_last_error().
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

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
    // mapped outer nodes cached per rule: (x, y, z, weight) per (triangle, node)
    int nodes_rule = 0;
    NodeW* d_nodes = nullptr;     // nt x nodes_rule
};

// Gauss-Hammer base rules (barycentric nodes, weights summing to 1/2).
int gh_base(int n, double bary[][3], double w[]);
// Composite rule on n_sub congruent sub-triangles, weights scaled by 2/n_sub.
int gh_composite(int n_nodes, int n_sub, double* nodes, double* weights);

// Device preparation of the per-triangle geometry.
int prep_mesh(MeshData& m, cudaStream_t s);
int map_nodes(MeshData& m, int n_gh, cudaStream_t s);

struct PhysParams {
    double rho, velP, velS, dt;
    int nT;
};
PhysParams phys_from(const ebem_problem* p);

// SA assembly of source rows [src0, src0+nsrc) into a device buffer
// (column-major 3 nsrc x 3N per lag, leading dimension ld, lag stride ld_lag).
int launch_sa_assemble(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                       double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count,
                       cudaStream_t s, int diag_only = 0);
int launch_ghc_assemble(const MeshData& m, const PhysParams& P, int n_gh, int n_sub, int n_sing, int lag0, int nlag,
                        double* d_E, size_t ld, size_t ld_lag, cudaStream_t s);

int launch_rhs(const MeshData& m, const PhysParams& P, int n_gh, int datum, double* d_rhs, cudaStream_t s);
int march_device(const double* dE, int n3, int L, const double* drhs, int nT, double* dphi, cudaStream_t s);
int launch_pp_sa(const MeshData& m, const PhysParams& P, const double* d_phi, const double* d_pts, int npts,
                 const double* h_times, int ntimes, double* d_u, cudaStream_t s);

}  // namespace ebem
