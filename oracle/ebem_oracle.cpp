// ORACLE — test infrastructure only (see sa_oracle.hpp).  Exposes a plain C
// ABI that tests/ and bench.py's CPU-baseline leg load with ctypes.
//
// What each entry point restates (paths relative to the reference project
// root; "SA/" = functions/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/):
//   or_gh              f/utility/quadRules/GaussHammer_base.m:19-409,
//                      f/utility/quadRules/GaussHammerComposite.m:1-55
//   or_mesh_derived    f/utility/fileRead/readSpaceMesh.m:93-148
//   or_num_blocks      .../BEMenerg_coreGPU/BEMenerg_coreGPU_calcNumBlocks.m:1-20
//   or_assemble_sa     SA/BEMenerg_coreSA_calcCostantData.m:1-26,
//                      SA/calcoloMatrice/BEMenerg_coreSA_calcMatrixBlock.m:1-90,
//                      SA/calcoloMatrice/BEMenerg_coreSA_calcMatrixSubBlock.m:1-111
//   or_rhs             .../BEMenerg_core_calcTn/BEMenerg_core_calcTnBlock.m:1-63,
//                      .../BEMenerg_core_calcTn/BEMenerg_core_calcNucleoTn.m:196-244
//                      (datum 8 'TEST', :13-132, in test_datum_oracle.cpp)
//   or_march           .../BEMenerg_coreGPU/BEMenerg_coreGPU_timeMarching.m:151-169
//   or_pp_sa           .../BEMenerg_postProc/BEMenerg_postProcA/*.m
//   or_assemble_ghc    .../BEMenerg_coreGPU/CUDAkernels/kernelGHC.cu:5-259
#include "sa_oracle.hpp"

#include <vector>
#include <cstdint>
#include <cstdio>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace oracle;

namespace {

// ---------------------------------------------------------------------------
// Gauss-Hammer base rules: the literal constants of GaussHammer_base.m.  A
// quadrature table is data that must be identical for parity.
struct BaseRule { int n; double b[28][3]; double w[28]; };

void base_rule(int n, BaseRule& r) {
    r.n = n;
    for (int i = 0; i < 28; i++) { r.b[i][0] = r.b[i][1] = r.b[i][2] = 0; r.w[i] = 0; }
    auto set3 = [&](int i, double x, double y, double z) { r.b[i][0] = x; r.b[i][1] = y; r.b[i][2] = z; };
    if (n == 1) {
        set3(0, 1.0 / 3, 1.0 / 3, 1.0 / 3); r.w[0] = 0.5;
    } else if (n == 3) {
        double v1 = 2.0 / 3, v2 = 1.0 / 6, v3 = 1.0 / 6;
        set3(0, v1, v2, v3); set3(1, v3, v1, v2); set3(2, v2, v3, v1);
        r.w[0] = r.w[1] = r.w[2] = 1.0 / 6;
    } else if (n == 7) {
        const double x[7] = {0.1012865073235, 0.7974269853531, 0.1012865073235, 0.4701420641051,
                             0.4701420641051, 0.0597158717898, 0.3333333333333};
        const double y[7] = {0.1012865073235, 0.1012865073235, 0.7974269853531, 0.0597158717898,
                             0.4701420641051, 0.4701420641051, 0.3333333333333};
        for (int i = 0; i < 7; i++) set3(i, x[i], y[i], 1 - x[i] - y[i]);
        for (int i = 0; i < 3; i++) r.w[i] = 0.1259391805448 / 2;
        for (int i = 3; i < 6; i++) r.w[i] = 0.1323941527885 / 2;
        r.w[6] = 0.225 / 2;
    } else if (n == 12) {
        double v1 = 0.873821971016996, v2 = (1 - v1) / 2, v3 = v2;
        set3(0, v1, v2, v3); set3(1, v3, v1, v2); set3(2, v2, v3, v1);
        v1 = 0.501426509658179; v2 = (1 - v1) / 2; v3 = v2;
        set3(3, v1, v2, v3); set3(4, v3, v1, v2); set3(5, v2, v3, v1);
        v1 = 0.636502499121399; v2 = 0.310352451033784; v3 = 1 - v1 - v2;
        set3(6, v1, v2, v3); set3(7, v1, v3, v2); set3(8, v2, v1, v3);
        set3(9, v2, v3, v1); set3(10, v3, v1, v2); set3(11, v3, v2, v1);
        double w1 = 0.050844906370207 / 2, w2 = 0.116786275726379 / 2, w3 = (0.5 - 3 * w1 - 3 * w2) / 6;
        for (int i = 0; i < 3; i++) r.w[i] = w1;
        for (int i = 3; i < 6; i++) r.w[i] = w2;
        for (int i = 6; i < 12; i++) r.w[i] = w3;
    } else if (n == 19) {
        set3(0, 1.0 / 3, 1.0 / 3, 1.0 / 3); r.w[0] = 0.09713579628279610 / 2;
        auto trip = [&](int i0, double a, double b, double w) {
            set3(i0, a, b, b); set3(i0 + 1, b, a, b); set3(i0 + 2, b, b, a);
            r.w[i0] = r.w[i0 + 1] = r.w[i0 + 2] = w;
        };
        trip(1, 0.02063496160252593, 0.48968251919873700, 0.09400410068141950 / 6);
        trip(4, 0.1258208170141290, 0.4370895914929355, 0.2334826230143263 / 6);
        trip(7, 0.6235929287619356, 0.1882035356190322, 0.2389432167816273 / 6);
        trip(10, 0.91054097321109410, 0.04472951339445297, 0.07673302697609430 / 6);
        double v1 = 0.03683841205473626, v2 = 0.74119859878449800, v3 = 1 - v1 - v2;
        set3(13, v1, v2, v3); set3(14, v1, v3, v2); set3(15, v2, v1, v3);
        set3(16, v2, v3, v1); set3(17, v3, v1, v2); set3(18, v3, v2, v1);
        for (int i = 13; i < 19; i++) r.w[i] = 0.2597012362637364 / 12;
    } else if (n == 28) {
        set3(0, 1.0 / 3, 1.0 / 3, 1.0 / 3); r.w[0] = 0.08797730116222190 / 2;
        auto trip = [&](int i0, double a, double b, double w) {
            set3(i0, a, b, b); set3(i0 + 1, b, a, b); set3(i0 + 2, b, b, a);
            r.w[i0] = r.w[i0 + 1] = r.w[i0 + 2] = w;
        };
        trip(1, 0.94802171814342330, 0.02598914092828833, 0.02623293466120857 / 6);
        trip(4, 0.81142499470415460, 0.09428750264792270, 0.1142447159818060 / 6);
        trip(7, 0.01072644996557060, 0.49463677501721470, 0.05656634416839376 / 6);
        trip(10, 0.5853132347709715, 0.2073433826145142, 0.2164790926342230 / 6);
        trip(13, 0.1221843885990187, 0.4389078057004907, 0.2079874161166116 / 6);
        auto six = [&](int i0, double v1, double v2, double w) {
            double v3 = 1 - v1 - v2;
            set3(i0, v1, v2, v3); set3(i0 + 1, v1, v3, v2); set3(i0 + 2, v2, v1, v3);
            set3(i0 + 3, v2, v3, v1); set3(i0 + 4, v3, v1, v2); set3(i0 + 5, v3, v2, v1);
            for (int i = 0; i < 6; i++) r.w[i0 + i] = w;
        };
        six(16, 0, 0.8588702812826364, 0.04417430269980344 / 12);
        six(22, 0.04484167758913055, 0.67793765488259020, 0.2463378925757316 / 12);
    } else {
        r.n = 0;
    }
}

struct Mesh {
    int nv = 0, nt = 0;
    std::vector<double> P;       // nv x 3
    std::vector<int> T;          // nt x 3, 0-based
    std::vector<double> normal, area, center, maxL;
    void vert(int t, double out[3][3]) const {
        for (int v = 0; v < 3; v++) for (int c = 0; c < 3; c++) out[v][c] = P[3 * T[3 * t + v] + c];
    }
};

// readSpaceMesh.m:93-148
void derive(Mesh& m) {
    m.normal.assign(3 * m.nt, 0); m.area.assign(m.nt, 0); m.center.assign(3 * m.nt, 0); m.maxL.assign(m.nt, 0);
    for (int t = 0; t < m.nt; t++) {
        double V[3][3]; m.vert(t, V);
        double vg1[3], vg2[3], vg3[3];
        for (int c = 0; c < 3; c++) { vg1[c] = V[0][c] - V[2][c]; vg2[c] = V[1][c] - V[2][c]; vg3[c] = V[0][c] - V[1][c]; }
        double n[3];
        n[0] = vg1[1] * vg2[2] - vg2[1] * vg1[2];
        n[1] = -vg1[0] * vg2[2] + vg2[0] * vg1[2];
        n[2] = vg1[0] * vg2[1] - vg2[0] * vg1[1];
        double area = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]) / 2;
        m.area[t] = area;
        for (int c = 0; c < 3; c++) m.normal[3 * t + c] = n[c] / (2 * area);
        for (int c = 0; c < 3; c++) m.center[3 * t + c] = (V[0][c] + V[1][c] + V[2][c]) / 3;
        double l1 = std::sqrt(vg3[0] * vg3[0] + vg3[1] * vg3[1] + vg3[2] * vg3[2]);
        double l2 = std::sqrt(vg2[0] * vg2[0] + vg2[1] * vg2[1] + vg2[2] * vg2[2]);
        double l3 = std::sqrt(vg1[0] * vg1[0] + vg1[1] * vg1[1] + vg1[2] * vg1[2]);
        m.maxL[t] = std::max(std::max(l1, l2), l3);
    }
}

Mesh make_mesh(const double* coords, int nv, const int* tris, int nt) {
    Mesh m; m.nv = nv; m.nt = nt;
    m.P.assign(coords, coords + 3 * nv);
    m.T.assign(tris, tris + 3 * nt);
    derive(m);
    return m;
}

struct Params {
    double rho, mu, lambda, velP, velS, dt;
    int nT;
};
Params make_params(double rho, double mu, double lambda, double dt, int nT) {
    Params p; p.rho = rho; p.mu = mu; p.lambda = lambda; p.dt = dt; p.nT = nT;
    p.velP = std::sqrt((lambda + 2 * mu) / rho);       // readInputFile.m:36
    p.velS = std::sqrt(mu / rho);                      // readInputFile.m:40
    return p;
}

// Per-triangle constants (BEMenerg_coreSA_calcCostantData.m): frame, mapped
// outer nodes, area-scaled weights; plus the Euler matrix of the field frame.
struct TriConst {
    real V[3][3];
    real vn[3];
    SdR S;
    M3 C;
    std::vector<double> nodes;   // nGH x 3
    std::vector<double> w;       // nGH
};

extern "C" int or_gh(int nNodes, int nSub, double* nodes, double* w);

// Outer nodes as the reference's SA path takes them: GaussHammerComposite(1, n)
// (BEMenerg_setupCore.m:16), whose node order and barycentric permutation
// differ from the base table (GaussHammerComposite.m:44).
BaseRule composite1(int n) {
    BaseRule R; base_rule(n, R);
    if (R.n == 0) return R;
    double nodes[28 * 3], w[28];
    or_gh(n, 1, nodes, w);
    for (int g = 0; g < n; g++) { for (int c = 0; c < 3; c++) R.b[g][c] = nodes[3 * g + c]; R.w[g] = w[g] / 2.0; }
    return R;
}

std::vector<TriConst> make_consts(const Mesh& m, const BaseRule& R) {
    std::vector<TriConst> tc(m.nt);
    for (int t = 0; t < m.nt; t++) {
        TriConst& k = tc[t];
        double Vd[3][3];
        m.vert(t, Vd);
        for (int v = 0; v < 3; v++) for (int c = 0; c < 3; c++) k.V[v][c] = Vd[v][c];
        for (int c = 0; c < 3; c++) k.vn[c] = m.normal[3 * t + c];
        k.S = calcoloSistemaRiferimento(k.V, k.vn);
        k.C = eulerMatrix(k.S, k.vn);
        k.nodes.resize(3 * R.n); k.w.resize(R.n);
        for (int g = 0; g < R.n; g++) {
            for (int c = 0; c < 3; c++)
                k.nodes[3 * g + c] = R.b[g][0] * Vd[0][c] + R.b[g][1] * Vd[1][c] + R.b[g][2] * Vd[2][c];
            k.w[g] = m.area[t] * (2.0 * R.w[g]);      // GaussHammerComposite(1, n): weights x 2/1
        }
    }
    return tc;
}

// BEMenerg_coreSA_calcMatrixBlock.m:57-61
inline bool sa_nonnull(const Mesh& m, const Params& p, int i, int j, int l) {
    double v[3];
    for (int c = 0; c < 3; c++) v[c] = m.center[3 * j + c] - m.center[3 * i + c];
    double d = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double distMin = d - m.maxL[j] - m.maxL[i];
    double distMax = d + m.maxL[j] + m.maxL[i];
    return ((l - 1) * p.velS * p.dt < distMax) && ((l + 1) * p.velP * p.dt >= distMin);
}

// BEMenerg_coreSA_calcMatrixSubBlock.m:1-111, followed by the clamp of
// BEMenerg_coreSA_calcMatrixBlock.m:77.
M3 sa_subblock(const Params& p, const TriConst& F, const TriConst& Sx, int nGH, int indTemp) {
    M3 ris;
    const double coef[3] = {1, -2, 1};
    const int ist[3] = {indTemp + 1, indTemp, indTemp - 1};
    for (int var = 0; var < 3; var++) {
        if (ist[var] <= 0) continue;
        M3 r[7];
        double currT = ist[var] * p.dt;
        double rP = p.velP * currT, rS = p.velS * currT;
        for (int g = 0; g < nGH; g++) {
            real sp[3] = {Sx.nodes[3 * g], Sx.nodes[3 * g + 1], Sx.nodes[3 * g + 2]};
            Prep pr = preparazioneTriangolo(sp, F.V, F.vn, F.S);
            real rhoP, rhoS;
            int type = classify(pr.zeta, rP, rS, pr.dMIN, rhoP, rhoS);
            if (type == T_NONE) continue;
            R6 t = fieldTriangle(pr.zeta, rP, rhoP, rS, rhoS, pr.children, pr.c, pr.sign_prod, type);
            t.r[2] = rotazioneInversaEulero(F.C, t.r[2]);
            t.r[4] = rotazioneInversaEulero(F.C, t.r[4]);
            t.r[6] = rotazioneInversaEulero(F.C, t.r[6]);
            for (int k = 1; k <= 6; k++) r[k] = r[k] + t.r[k] * Sx.w[g];
        }
        M3 rist = combine(r, p.velP, p.velS, currT);
        ris = ris + coef[var] * rist;
    }
    ris = ris / (4 * PI * p.rho);
    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++)
        if (oracle::fabs(ris.m[a][b]) < 1.0e-14) ris.m[a][b] = 0;
    return ris;
}

// Datum g(x, t) of the Dirichlet problem.  Ids 2.. follow
// BEMenerg_core_calcNucleoTn.m:199-237; ids 0 and 1 are the screen and
// sphere data of the two headline workloads (not in the reference).
void datum(int id, const Params& p, double Tfin, const double x[3], double t, double g[3]) {
    g[0] = g[1] = g[2] = 0;
    switch (id) {
    case 0: g[2] = t * t * t * t * std::exp(-2 * t); break;
    case 1: { double s = (t > 0) ? std::sin(2 * PI * t) : 0.0; for (int c = 0; c < 3; c++) g[c] = x[c] * s; } break;
    case 2: g[2] = 0.5 * t; break;
    case 3: { double f = (t < PI / 2) ? std::pow(std::sin(t), 5) : 1.0; g[2] = f * (x[0] * x[0]); } break;
    case 4: case 5: {
        double h = (id == 4) ? 1.0 : 3.0;
        double velP = p.velP;
        int hat_k = (int)std::ceil((velP * Tfin) / (2 * h)) - 1;
        double s = 0;
        for (int k = 0; k <= hat_k; k++) {
            double a1 = velP * t - 2 * h * k - (h - x[2]);
            double a2 = velP * t - 2 * h * (k + 1) + (h - x[2]);
            double term = a1 * (a1 > 0) - a2 * (a2 > 0);
            s += ((k % 2) ? -1.0 : 1.0) * term;
        }
        g[2] = s;
    } break;
    case 6: { double u = x[0] - 2 + p.velP * t - 0.475; g[0] = -std::exp(-20 * u * u); } break;
    case 7: { double u = x[2] + 1 - p.velP * t; g[2] = -std::exp(-20 * u * u); } break;
    default: break;
    }
}

// LU with partial pivoting (row interchanges), column-major n x n.
bool lu_factor(std::vector<double>& A, int n, std::vector<int>& piv) {
    piv.resize(n);
    for (int k = 0; k < n; k++) {
        int p = k; double best = std::fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; i++) { double v = std::fabs(A[(size_t)k * n + i]); if (v > best) { best = v; p = i; } }
        piv[k] = p;
        if (best == 0) return false;
        if (p != k) for (int j = 0; j < n; j++) std::swap(A[(size_t)j * n + k], A[(size_t)j * n + p]);
        double d = A[(size_t)k * n + k];
        for (int i = k + 1; i < n; i++) A[(size_t)k * n + i] /= d;
        for (int j = k + 1; j < n; j++) {
            double akj = A[(size_t)j * n + k];
            if (akj == 0) continue;
            double* colj = &A[(size_t)j * n];
            const double* colk = &A[(size_t)k * n];
            for (int i = k + 1; i < n; i++) colj[i] -= colk[i] * akj;
        }
    }
    return true;
}

void lu_solve(const std::vector<double>& A, int n, const std::vector<int>& piv, double* b) {
    for (int k = 0; k < n; k++) if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (int j = 0; j < n; j++) { double bj = b[j]; if (bj != 0) for (int i = j + 1; i < n; i++) b[i] -= A[(size_t)j * n + i] * bj; }
    for (int j = n - 1; j >= 0; j--) { b[j] /= A[(size_t)j * n + j]; double bj = b[j]; for (int i = 0; i < j; i++) b[i] -= A[(size_t)j * n + i] * bj; }
}

int set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
#else
    (void)nthreads; return 1;
#endif
}

// kernelGHC.cu:204-259 (nucleo), with the reference's expression shapes.
void nucleo(double nu[3][3], const double x[3], double r, double t, double cP, double cS) {
    double r3 = std::pow(r, 3), r5 = std::pow(r, 5);
    double HP = (t - (r / cP) > 0), HS = (t - (r / cS) > 0);
    double tail = ((cP * cP * t * t - r * r) / (cP * cP) * HP - (cS * cS * t * t - r * r) / (cS * cS) * HS);
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
        double xx = x[i] * x[j];
        if (i == j) {
            nu[i][j] = ((xx) / r3) * (1 / (cP * cP)) * HP
                       + ((1 / r) - (xx / r3)) * (1 / (cS * cS)) * HS
                       - 0.5 * ((1 / r3) - 3 * (xx / r5)) * tail;
        } else {
            nu[i][j] = ((xx) / r3) * (1 / (cP * cP)) * HP
                       + (-(xx / r3)) * (1 / (cS * cS)) * HS
                       - 0.5 * (-3 * (xx / r5)) * tail;
        }
    }
}

}  // namespace

extern "C" {

int or_gh(int nNodes, int nSub, double* nodes, double* w) {
    BaseRule R; base_rule(nNodes, R);
    if (R.n == 0) return -1;
    int nDiv = (int)std::lround(std::sqrt((double)nSub));
    if (nDiv * nDiv != nSub || nSub < 1) return -2;
    double fl = 1.0 / nDiv;
    int n = 0;
    for (int i = 1; i <= nDiv; i++) {
        double zMin = (i - 1) * fl, zMax = i * fl;
        int nTr = 2 * (nDiv - i) + 1;
        double xv[3] = {1 - zMin, 1 - zMin, 1 - zMin - fl};
        double yv[3] = {0 - fl, 0, 0};
        double zv[3] = {0, 0, 0};
        for (int j = 1; j <= nTr; j++) {
            if (j % 2 == 1) {
                double nx[3] = {xv[1], xv[2], xv[2]}, ny[3] = {yv[1], yv[2], yv[2] + fl};
                for (int q = 0; q < 3; q++) { xv[q] = nx[q]; yv[q] = ny[q]; }
                zv[0] = zMin; zv[1] = zMax; zv[2] = zMin;
            } else {
                double nx[3] = {xv[1], xv[2], xv[2] - fl}, ny[3] = {yv[1], yv[2], yv[2]};
                for (int q = 0; q < 3; q++) { xv[q] = nx[q]; yv[q] = ny[q]; }
                zv[0] = zMax; zv[1] = zMin; zv[2] = zMax;
            }
            for (int g = 0; g < nNodes; g++) {
                double* o = nodes + 3 * ((size_t)n * nNodes + g);
                o[0] = R.b[g][0] * xv[0] + R.b[g][1] * xv[1] + R.b[g][2] * xv[2];
                o[1] = R.b[g][0] * yv[0] + R.b[g][1] * yv[1] + R.b[g][2] * yv[2];
                o[2] = R.b[g][0] * zv[0] + R.b[g][1] * zv[1] + R.b[g][2] * zv[2];
            }
            n++;
        }
    }
    for (int g = 0; g < nNodes; g++) w[g] = (2.0 / nSub) * R.w[g];
    return 0;
}

int or_mesh_derived(const double* coords, int nv, const int* tris, int nt,
                    double* normal, double* area, double* center, double* maxL) {
    Mesh m = make_mesh(coords, nv, tris, nt);
    for (int i = 0; i < 3 * nt; i++) { normal[i] = m.normal[i]; center[i] = m.center[i]; }
    for (int i = 0; i < nt; i++) { area[i] = m.area[i]; maxL[i] = m.maxL[i]; }
    return 0;
}

int or_num_blocks(const double* coords, int nv, double velS, double dt, int nT) {
    double maxD = 0;
    for (int a = 0; a < nv; a++) for (int b = 0; b < nv; b++) {
        double v[3] = {coords[3 * a] - coords[3 * b], coords[3 * a + 1] - coords[3 * b + 1], coords[3 * a + 2] - coords[3 * b + 2]};
        double d = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (d > maxD) maxD = d;
    }
    int maxIndTemp = (int)std::ceil(maxD / (velS * dt)) + 1;
    return std::min(nT, maxIndTemp);
}

// Dense SA assembly of lags [lag0, lag0+nlag): E is column-major
// 3N x 3N x nlag (row = 3*source + comp, col = 3*field + comp).  Returns the
// number of non-null pair-lags.
long long or_assemble_sa(const double* coords, int nv, const int* tris, int nt,
                         double rho, double mu, double lambda, double dt, int nT,
                         int nGH, int lag0, int nlag, double* E, int nthreads) {
    BaseRule R = composite1(nGH);
    if (R.n == 0) return -1;
    Mesh m = make_mesh(coords, nv, tris, nt);
    Params p = make_params(rho, mu, lambda, dt, nT);
    std::vector<TriConst> tc = make_consts(m, R);
    set_threads(nthreads);
    const size_t n3 = 3 * (size_t)nt;
    long long nonnull = 0;
    for (int q = 0; q < nlag; q++) {
        int l = lag0 + q;
        double* El = E + (size_t)q * n3 * n3;
        #pragma omp parallel for schedule(dynamic, 16) reduction(+ : nonnull)
        for (long long ind = 0; ind < (long long)nt * nt; ind++) {
            int i = (int)(ind % nt), j = (int)(ind / nt);   // ind2sub: source fastest
            M3 b;
            if (sa_nonnull(m, p, i, j, l)) {
                nonnull++;
                b = sa_subblock(p, tc[j], tc[i], nGH, l);
            }
            for (int c = 0; c < 3; c++) for (int r = 0; r < 3; r++)
                El[(3 * (size_t)j + c) * n3 + 3 * (size_t)i + r] = b.m[r][c];
        }
    }
    return nonnull;
}

// Selected (source, field, lag) blocks; out is npairs x 9, column-major 3x3.
int or_assemble_sa_pairs(const double* coords, int nv, const int* tris, int nt,
                         double rho, double mu, double lambda, double dt, int nT, int nGH,
                         int npairs, const int* src, const int* fld, const int* lag, double* out, int nthreads) {
    BaseRule R = composite1(nGH);
    if (R.n == 0) return -1;
    Mesh m = make_mesh(coords, nv, tris, nt);
    Params p = make_params(rho, mu, lambda, dt, nT);
    std::vector<TriConst> tc = make_consts(m, R);
    set_threads(nthreads);
    #pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < npairs; q++) {
        M3 b;
        if (sa_nonnull(m, p, src[q], fld[q], lag[q])) b = sa_subblock(p, tc[fld[q]], tc[src[q]], nGH, lag[q]);
        for (int c = 0; c < 3; c++) for (int r = 0; r < 3; r++) out[9 * (size_t)q + 3 * c + r] = b.m[r][c];
    }
    return 0;
}

int or_tn_test(double x1, double x2, double t0, double t1, double rho, double mu, double lambda, int nang, int nsplit,
               int nrad, double* out);

// Right-hand side b_n, n = 0..nT-1, column-major 3N x nT.  Datum 8 is the
// reference's 'TEST' case, whose value is computed for the pair of instants
// at once (BEMenerg_core_calcNucleoTn(pbParam, puntoT, t0, t1)).
int or_rhs(const double* coords, int nv, const int* tris, int nt,
           double rho, double mu, double lambda, double dt, int nT, int nGH, int datum_id, double* rhs) {
    BaseRule R = composite1(nGH);
    if (R.n == 0) return -1;
    Mesh m = make_mesh(coords, nv, tris, nt);
    Params p = make_params(rho, mu, lambda, dt, nT);
    std::vector<TriConst> tc = make_consts(m, R);
    double Tfin = dt * nT;
    for (int n = 0; n < nT; n++) {
        double tInz = dt * n, tFin = dt * (n + 1);
        for (int t = 0; t < nt; t++) {
            double ris[3] = {0, 0, 0};
            for (int g = 0; g < nGH; g++) {
                const double* x = &tc[t].nodes[3 * g];
                double g1[3], g0[3];
                if (datum_id == 8) {
                    if (or_tn_test(x[0], x[1], tInz, tFin, rho, mu, lambda, 24, 4, 24, g1)) return -1;
                    g0[0] = g0[1] = g0[2] = 0;
                } else {
                    datum(datum_id, p, Tfin, x, tFin, g1);
                    datum(datum_id, p, Tfin, x, tInz, g0);
                }
                for (int c = 0; c < 3; c++) ris[c] = ris[c] + (g1[c] - g0[c]) * tc[t].w[g];
            }
            for (int c = 0; c < 3; c++) {
                if (std::fabs(ris[c]) < 1.0e-14) ris[c] = 0;
                rhs[(size_t)n * 3 * nt + 3 * t + c] = ris[c];
            }
        }
    }
    return 0;
}

// Time marching with LU of E_0: phi_n = E_0^{-1}(b_n - sum_{m=1}^{min(n,L-1)} E_m phi_{n-m}).
int or_march(const double* E, int n3, int L, const double* rhs, int nT, double* phi) {
    std::vector<double> A(E, E + (size_t)n3 * n3);
    std::vector<int> piv;
    if (!lu_factor(A, n3, piv)) return -1;
    std::vector<double> b(n3);
    for (int n = 0; n < nT; n++) {
        for (int i = 0; i < n3; i++) b[i] = rhs[(size_t)n * n3 + i];
        int endInd = std::min(n + 1, L);
        for (int mm = 1; mm < endInd; mm++) {
            const double* Em = E + (size_t)mm * n3 * n3;
            const double* ph = phi + (size_t)(n - mm) * n3;
            for (int j = 0; j < n3; j++) {
                double pj = ph[j];
                if (pj == 0) continue;
                const double* col = Em + (size_t)j * n3;
                for (int i = 0; i < n3; i++) b[i] -= col[i] * pj;
            }
        }
        lu_solve(A, n3, piv, b.data());
        for (int i = 0; i < n3; i++) phi[(size_t)n * n3 + i] = b[i];
    }
    return 0;
}

// The same marching with the LU factorisation, the history sums and the
// solves carried out in `real` (binary128 in the quad build; identical to
// or_march's arithmetic order otherwise), the inputs being the double
// blocks and right-hand side: the exact marching of the given data, used to
// pin the time-marched density of the benchmark configurations.
int or_march_exact(const double* E, int n3, int L, const double* rhs, int nT, double* phi) {
    std::vector<real> A(E, E + (size_t)n3 * n3);
    std::vector<int> piv(n3);
    for (int k = 0; k < n3; k++) {                       // column-major, partial pivoting
        int p = k;
        real best = oracle::fabs(A[(size_t)k * n3 + k]);
        for (int i = k + 1; i < n3; i++) {
            real v = oracle::fabs(A[(size_t)k * n3 + i]);
            if (v > best) { best = v; p = i; }
        }
        if (best == 0) return -1;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n3; j++) std::swap(A[(size_t)j * n3 + k], A[(size_t)j * n3 + p]);
        const real d = A[(size_t)k * n3 + k];
        for (int i = k + 1; i < n3; i++) A[(size_t)k * n3 + i] /= d;
        for (int j = k + 1; j < n3; j++) {
            const real f = A[(size_t)j * n3 + k];
            if (f == 0) continue;
            for (int i = k + 1; i < n3; i++) A[(size_t)j * n3 + i] -= A[(size_t)k * n3 + i] * f;
        }
    }
    std::vector<real> ph((size_t)n3 * nT), b(n3);
    for (int n = 0; n < nT; n++) {
        for (int i = 0; i < n3; i++) b[i] = rhs[(size_t)n * n3 + i];
        const int endInd = std::min(n + 1, L);
        for (int mm = 1; mm < endInd; mm++) {
            const double* Em = E + (size_t)mm * n3 * n3;
            const real* pp = ph.data() + (size_t)(n - mm) * n3;
            for (int j = 0; j < n3; j++) {
                const real pj = pp[j];
                if (pj == 0) continue;
                const double* col = Em + (size_t)j * n3;
                for (int i = 0; i < n3; i++) b[i] -= real(col[i]) * pj;
            }
        }
        for (int k = 0; k < n3; k++) std::swap(b[k], b[piv[k]]);
        for (int k = 0; k < n3; k++)                     // L y = P b (unit lower)
            for (int i = k + 1; i < n3; i++) b[i] -= A[(size_t)k * n3 + i] * b[k];
        for (int k = n3 - 1; k >= 0; k--) {              // U x = y
            b[k] /= A[(size_t)k * n3 + k];
            for (int i = 0; i < k; i++) b[i] -= A[(size_t)k * n3 + i] * b[k];
        }
        for (int i = 0; i < n3; i++) ph[(size_t)n * n3 + i] = b[i];
    }
    for (size_t i = 0; i < ph.size(); i++) phi[i] = (double)ph[i];
    return 0;
}

// Closed-form single-instant block of BEMenerg_postProcA_calcMatrixBlock.m.
static M3 pp_block(const Params& p, const TriConst& F, const double x[3], double tau) {
    M3 ris;
    double rP = p.velP * tau, rS = p.velS * tau;
    real sp[3] = {x[0], x[1], x[2]};
    Prep pr = preparazioneTriangolo(sp, F.V, F.vn, F.S);
    real rhoP, rhoS;
    int type = classify(pr.zeta, rP, rS, pr.dMIN, rhoP, rhoS);
    if (type == T_NONE) return ris;
    R6 t = fieldTriangle(pr.zeta, rP, rhoP, rS, rhoS, pr.children, pr.c, pr.sign_prod, type);
    t.r[2] = rotazioneInversaEulero(F.C, t.r[2]);
    t.r[4] = rotazioneInversaEulero(F.C, t.r[4]);
    t.r[6] = rotazioneInversaEulero(F.C, t.r[6]);
    ris = combine(t.r, p.velP, p.velS, tau);
    ris = ris / (4 * PI * p.rho);
    return ris;
}

// u(x, t) at npts points x ntimes times; u is 3 x npts x ntimes (column-major).
int or_pp_sa(const double* coords, int nv, const int* tris, int nt,
             double rho, double mu, double lambda, double dt, int nT,
             const double* phi, const double* pts, int npts, const double* times, int ntimes,
             double* u, int nthreads) {
    BaseRule R; base_rule(1, R);
    Mesh m = make_mesh(coords, nv, tris, nt);
    Params p = make_params(rho, mu, lambda, dt, nT);
    std::vector<TriConst> tc = make_consts(m, R);
    set_threads(nthreads);
    const size_t n3 = 3 * (size_t)nt;
    #pragma omp parallel for schedule(dynamic, 1)
    for (long long q = 0; q < (long long)npts * ntimes; q++) {
        int ix = (int)(q % npts), it = (int)(q / npts);
        double t = times[it];
        const double* x = pts + 3 * ix;
        real uu[3] = {0, 0, 0};
        if (t > 0) {
            int nHat = (int)std::ceil(t / p.dt) - 1;
            std::vector<M3> cur(nt), nxt(nt);
            for (int j = 0; j < nt; j++) {
                cur[j] = pp_block(p, tc[j], x, t);
                for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) if (oracle::fabs(cur[j].m[a][b]) < 1.0e-14) cur[j].m[a][b] = 0;
            }
            for (int k = 1; k <= nHat; k++) {
                double diffT = t - (k * p.dt);
                const double* al = phi + (size_t)(k - 1) * n3;
                for (int j = 0; j < nt; j++) {
                    nxt[j] = pp_block(p, tc[j], x, diffT);
                    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) if (oracle::fabs(nxt[j].m[a][b]) < 1.0e-14) nxt[j].m[a][b] = 0;
                }
                for (int j = 0; j < nt; j++)
                    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++)
                        uu[a] += (cur[j].m[a][b] - nxt[j].m[a][b]) * al[3 * j + b];
                std::swap(cur, nxt);
            }
            const double* al = phi + (size_t)nHat * n3;
            for (int j = 0; j < nt; j++)
                for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) uu[a] += cur[j].m[a][b] * al[3 * j + b];
        }
        for (int a = 0; a < 3; a++) u[3 * (size_t)q + a] = (double)uu[a];
    }
    return 0;
}

// kernelGHC.cu:5-169 restated on the CPU: numerical inner composite rule,
// off-diagonal blocks only, the null test of kernelGHC.cu:171-201, the
// per-thread accumulation and the shared-memory tree reduction reproduced in
// the reference's order.  E (column-major 3N x 3N x nlag) is accumulated into.
int or_assemble_ghc(const double* coords, int nv, const int* tris, int nt,
                    double rho, double mu, double lambda, double dt, int nT,
                    int nGH, int nSub, int nSing, int lag0, int nlag, double* E, int nthreads) {
    std::vector<double> ghn(3 * nGH), ghw(nGH), gcn(3 * (size_t)nSub * nSing), gcw(nSing);
    if (or_gh(nGH, 1, ghn.data(), ghw.data()) != 0) return -1;
    if (or_gh(nSing, nSub, gcn.data(), gcw.data()) != 0) return -1;
    Mesh m = make_mesh(coords, nv, tris, nt);
    Params p = make_params(rho, mu, lambda, dt, nT);
    set_threads(nthreads);
    const double c4 = 4 * PI * rho;
    const size_t n3 = 3 * (size_t)nt;
    const int bx = nSub, by = nSing, nthr = bx * by;
    for (int q = 0; q < nlag; q++) {
        int z = lag0 + q;
        double* El = E + (size_t)q * n3 * n3;
        #pragma omp parallel for schedule(dynamic, 16)
        for (long long ind = 0; ind < (long long)nt * nt; ind++) {
            int bxI = (int)(ind % nt), byI = (int)(ind / nt);   // blockIdx.x = source, blockIdx.y = field
            if (bxI == byI) continue;
            double VS[3][3], VF[3][3]; m.vert(bxI, VS); m.vert(byI, VF);
            double distMax = 0;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                double v[3] = {VS[i][0] - VF[j][0], VS[i][1] - VF[j][1], VS[i][2] - VF[j][2]};
                double d = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                if (d > distMax) distMax = d;
            }
            if ((z - 1) * p.velS * dt > distMax) continue;
            std::vector<double> sm((size_t)nthr * 9, 0.0);
            for (int tx = 0; tx < bx; tx++) for (int ty = 0; ty < by; ty++) {
                double* acc = &sm[(size_t)(tx * by + ty) * 9];
                double pesoInt = gcw[ty] * m.area[byI];
                const double* nd = &gcn[3 * (size_t)(tx * by + ty)];
                double yI[3];
                for (int c = 0; c < 3; c++) yI[c] = nd[0] * VF[0][c] + nd[1] * VF[1][c] + nd[2] * VF[2][c];
                for (int l = 0; l < nGH; l++) {
                    double pesoExt = ghw[l] * m.area[bxI];
                    const double* ne = &ghn[3 * l];
                    double xE[3];
                    for (int c = 0; c < 3; c++) xE[c] = ne[0] * VS[0][c] + ne[1] * VS[1][c] + ne[2] * VS[2][c];
                    double pt[3] = {yI[0] - xE[0], yI[1] - xE[1], yI[2] - xE[2]};
                    double pn = std::sqrt(pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2]);
                    const double cn[3] = {1, -2, 1}, ctm[3] = {-1, 0, 1};
                    for (int k = 0; k < 3; k++) {
                        double ist = dt * (z + ctm[k]);
                        if (ist < 0) continue;
                        double nu[3][3];
                        nucleo(nu, pt, pn, ist, p.velP, p.velS);
                        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
                            acc[3 * i + j] += pesoExt * pesoInt * cn[k] * nu[i][j];
                    }
                }
            }
            // reduction: y to a power of two, then y halving, then x halving
            int yDim = 1; while (yDim * 2 <= by) yDim *= 2;
            for (int tx = 0; tx < bx; tx++) for (int ty = 0; ty < by; ty++)
                if (ty + yDim < by) for (int e = 0; e < 9; e++)
                    sm[(size_t)(tx * by + ty) * 9 + e] += sm[(size_t)(tx * by + ty + yDim) * 9 + e];
            for (yDim /= 2; yDim > 0; yDim /= 2)
                for (int tx = 0; tx < bx; tx++) for (int ty = 0; ty < yDim; ty++)
                    for (int e = 0; e < 9; e++) sm[(size_t)(tx * by + ty) * 9 + e] += sm[(size_t)(tx * by + ty + yDim) * 9 + e];
            for (int xDim = bx / 2; xDim > 0; xDim /= 2)
                for (int tx = 0; tx < xDim; tx++) for (int ty = 0; ty < by; ty++)
                    for (int e = 0; e < 9; e++) sm[(size_t)(tx * by + ty) * 9 + e] += sm[(size_t)((tx + xDim) * by + ty) * 9 + e];
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                double v = sm[3 * i + j];
                if (std::fabs(v) > 1.0e-14)
                    El[(3 * (size_t)byI + j) * n3 + 3 * (size_t)bxI + i] += v / c4;
            }
        }
    }
    return 0;
}

// The reference's numerical post-processing "GPU yy z" restated on the CPU:
// kernelSP.cu:5-121 with the host sum of BEMenerg_postProcGPU_calcSP.m:21-85
// (variant 0) and kernelLayer.cu:5-170 with BEMenerg_postProcGPU_calcLayer.m
// (variant 1), per (point, time).  stride: node index stride*subregion + l
// (kernelSP.cu:41 has 3; kernelLayer n_sing).  phi column-major 3N x nT;
// u is 3 x npts x ntimes (column-major).
int or_pp_gpu(const double* coords, int nv, const int* tris, int nt, double rho, double mu, double lambda, double dt,
              int nT, const double* phi, const double* pts, int npts, const double* times, int ntimes, int nSub,
              int nSing, int variant, int stride, double* u, int nthreads) {
    std::vector<double> gcn(3 * (size_t)nSub * nSing), gcw(nSing);
    if (or_gh(nSing, nSub, gcn.data(), gcw.data()) != 0) return -1;
    if ((nSub - 1) * stride + nSing > nSub * nSing) return -2;
    Mesh m = make_mesh(coords, nv, tris, nt);
    Params p = make_params(rho, mu, lambda, dt, nT);
    set_threads(nthreads);
    const double c4 = 4 * PI * rho;
    const size_t n3 = 3 * (size_t)nt;
    #pragma omp parallel for schedule(dynamic, 1)
    for (long long q = 0; q < (long long)npts * ntimes; q++) {
        const int ix = (int)(q % npts), it = (int)(q / npts);
        const double t = times[it];
        const double* x = pts + 3 * ix;
        double uu[3] = {0, 0, 0};
        if (t > 0) {
            int nHat = (int)std::ceil(t / dt) - 1;
            const int numIst = nHat + 1;
            // matrixTotal [3 numIst x 3N] (variant 0) or the per-instant blocks (variant 1)
            std::vector<double> Mt((size_t)3 * numIst * n3, 0.0);
            for (int k = 0; k < numIst; k++) {
                volatile double kd = k * dt;
                const double tau = t - kd;
                for (int mm = 0; mm < nt; mm++) {
                    double dv[3] = {x[0] - m.center[3 * mm], x[1] - m.center[3 * mm + 1], x[2] - m.center[3 * mm + 2]};
                    double distMin = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]) - m.maxL[mm];
                    if (tau * p.velP < distMin) continue;
                    double V[3][3]; m.vert(mm, V);
                    double blk[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                    for (int sub = 0; sub < nSub; sub++) for (int l = 0; l < nSing; l++) {
                        const double* nd = &gcn[3 * (size_t)(stride * sub + l)];
                        double y[3];
                        for (int c = 0; c < 3; c++) y[c] = nd[0] * V[0][c] + nd[1] * V[1][c] + nd[2] * V[2][c];
                        double pt[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
                        double pn = std::sqrt(pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2]);
                        double nu[3][3];
                        nucleo(nu, pt, pn, tau, p.velP, p.velS);
                        double wt = gcw[l] * m.area[mm];
                        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) blk[i][j] += wt * nu[i][j];
                    }
                    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                        double v;
                        if (variant == 0) v = (std::fabs(blk[i][j]) > 1.0e-14) ? blk[i][j] / c4 : 0.0;
                        else { v = blk[i][j] / c4; if (std::fabs(v) < 1.0e-14) v = 0.0; }
                        Mt[(3 * (size_t)mm + j) * 3 * numIst + 3 * k + i] = v;     // row 3k+i, column 3mm+j
                    }
                }
            }
            auto M = [&](int k, int i, size_t col) { return Mt[col * 3 * numIst + 3 * k + i]; };
            if (variant == 0) {
                for (int k = 0; k < nHat; k++)
                    for (size_t col = 0; col < n3; col++) {
                        double d = phi[(size_t)k * n3 + col];
                        for (int i = 0; i < 3; i++) uu[i] += (M(k, i, col) - M(k + 1, i, col)) * d;
                    }
                for (size_t col = 0; col < n3; col++)
                    for (int i = 0; i < 3; i++) uu[i] += M(nHat, i, col) * phi[(size_t)nHat * n3 + col];
            } else {
                for (int k = 0; k < numIst; k++)
                    for (size_t col = 0; col < n3; col++) {
                        double d = phi[(size_t)k * n3 + col] - (k > 0 ? phi[(size_t)(k - 1) * n3 + col] : 0.0);
                        for (int i = 0; i < 3; i++) uu[i] += M(k, i, col) * d;
                    }
            }
        }
        for (int a = 0; a < 3; a++) u[3 * (size_t)q + a] = uu[a];
    }
    return 0;
}

// Null-test census: number of non-null pair-lags over lags [0, L).
long long or_count_nonnull(const double* coords, int nv, const int* tris, int nt,
                           double rho, double mu, double lambda, double dt, int nT, int L) {
    Mesh m = make_mesh(coords, nv, tris, nt);
    Params p = make_params(rho, mu, lambda, dt, nT);
    long long c = 0;
    for (int l = 0; l < L; l++)
        for (int j = 0; j < nt; j++) for (int i = 0; i < nt; i++) c += sa_nonnull(m, p, i, j, l);
    return c;
}

}  // extern "C"

extern "C" {

// The six closed-form kernel integrals ris1..ris6 of one field triangle j
// seen from a point x at time t (BEMenerg_coreSA_calcMatrixSubBlock.m:88-97
// without the outer weight), rotated back to global axes.  out: 6 x 9
// (row-major 3x3 each).  Returns the case id (0 none, 1 SP_SP, 2 SP_P, 3 P).
int or_field_integrals(const double* coords, int nv, const int* tris, int nt, double velP, double velS,
                       int j, const double* x, double t, double* out) {
    Mesh m = make_mesh(coords, nv, tris, nt);
    BaseRule R; base_rule(1, R);
    std::vector<TriConst> tc = make_consts(m, R);
    const TriConst& F = tc[j];
    real sp[3] = {x[0], x[1], x[2]};
    Prep pr = preparazioneTriangolo(sp, F.V, F.vn, F.S);
    real rhoP, rhoS;
    double rP = velP * t, rS = velS * t;
    int type = classify(pr.zeta, rP, rS, pr.dMIN, rhoP, rhoS);
    for (int k = 0; k < 54; k++) out[k] = 0;
    if (type == T_NONE) return 0;
    R6 r = fieldTriangle(pr.zeta, rP, rhoP, rS, rhoS, pr.children, pr.c, pr.sign_prod, type);
    r.r[2] = rotazioneInversaEulero(F.C, r.r[2]);
    r.r[4] = rotazioneInversaEulero(F.C, r.r[4]);
    r.r[6] = rotazioneInversaEulero(F.C, r.r[6]);
    for (int k = 1; k <= 6; k++)
        for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) out[9 * (k - 1) + 3 * a + b] = r.r[k].m[a][b];
    return type;
}

}  // extern "C"
