// ORACLE — test infrastructure only.  CPU restatement of the direct
// (displacement/traction) formulation: the double-layer operator K_l with its
// P1 basis, the singular (same-triangle) parts of K_l and the diagonal blocks
// of V_l on Duffy-type "DIAG" rules, and the direct post-processing operators.
// Loaded with ctypes by tests/ only; nothing in the library links it.
//
// What each entry point restates (paths relative to the reference project
// root; "DIR/" = functions/BEMenerg_dir/, "PP/" = functions/BEMenerg_dirPP/):
//   or_p1_coeffs     DIR/BEMenerg_dir_calcCostantData.m:17-21 (matCoeff, vetCoeff);
//                    PP/BEMenerg_pp_calcCostantData.m:7-12 (unit-normal variant)
//   or_doppio_gauss  functions/utility/quadRules/doppioGauss1D.m:1-43,
//                    functions/utility/quadRules/Gauss1D.m (Gauss-Legendre)
//   or_assemble_k    DIR/CUDAkernels/kernelK.cu:14-460 (thread/reduction order kept)
//   or_k_sing        DIR/BEMenerg_dir_calcSubBlockSingK.m:1-41,
//                    DIR/BEMenerg_dir_calcKIntgSing.m:1-175
//   or_v_diag        DIR/BEMenerg_dir_calcSubBlockDiagV.m:1-118
//   or_pp_dir_g      PP/CUDAkernels/kernelG.cu:10-113
//   or_pp_dir_p      PP/CUDAkernels/kernelP.cu:12-150
//
// Reference defects kept for parity, each behind `fix` (0 = reproduce):
//   kernelK.cu:414,420,426,437,443,449  H(r - r/c_P) instead of H(t - r/c_P)
//                                        in the lambda-mu term of nucleoKRj
//   kernelK.cu:242                       distMin starts at 100, not +inf
//   kernelG.cu:51                        node stride 3 instead of n_sing
#include <cmath>
#include <vector>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" int or_gh(int nNodes, int nSub, double* nodes, double* w);
extern "C" int or_mesh_derived(const double* coords, int nv, const int* tris, int nt, double* normal, double* area,
                               double* center, double* maxL);

namespace {

constexpr double PI = 3.14159265358979323846;

struct DMesh {
    int nv = 0, nt = 0;
    const double* X = nullptr;
    const int* T = nullptr;
    std::vector<double> normal, area, center, maxL;
    std::vector<double> M, v;      // phi_k(y) = v[k] + M[k][:] . y, k = 0..2, per triangle
    double maxLen = 0;
    void vert(int t, double V[3][3]) const {
        for (int a = 0; a < 3; a++)
            for (int c = 0; c < 3; c++) V[a][c] = X[3 * T[3 * t + a] + c];
    }
    int local(int t, int s) const {   // 1..3 if vertex s belongs to triangle t, else 0
        for (int k = 0; k < 3; k++)
            if (T[3 * t + k] == s) return k + 1;
        return 0;
    }
};

void cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// M = A B^-1 with B = [l21, l31, n] (columns), A = [-1 -1 0; 1 0 0; 0 1 0]:
// the rows of B^-1 are (l31 x n, n x l21, l21 x l31) / det(B).  Then
// v = e1 - M V1, so phi_k is the barycentric coordinate of vertex k.
void p1_coeffs(const double V[3][3], const double n[3], double M[9], double v[3]) {
    double l21[3], l31[3];
    for (int c = 0; c < 3; c++) { l21[c] = V[1][c] - V[0][c]; l31[c] = V[2][c] - V[0][c]; }
    double r0[3], r1[3], r2[3];
    cross3(l31, n, r0);
    cross3(n, l21, r1);
    cross3(l21, l31, r2);
    double det = dot3(l21, r0);
    for (int c = 0; c < 3; c++) { r0[c] /= det; r1[c] /= det; }
    for (int c = 0; c < 3; c++) {
        M[c] = -r0[c] - r1[c];
        M[3 + c] = r0[c];
        M[6 + c] = r1[c];
    }
    for (int k = 0; k < 3; k++) v[k] = (k == 0 ? 1.0 : 0.0) - (M[3 * k] * V[0][0] + M[3 * k + 1] * V[0][1] + M[3 * k + 2] * V[0][2]);
}

DMesh make(const double* X, int nv, const int* T, int nt, bool unit_normal) {
    DMesh m;
    m.nv = nv; m.nt = nt; m.X = X; m.T = T;
    m.normal.resize(3 * (size_t)nt); m.area.resize(nt); m.center.resize(3 * (size_t)nt); m.maxL.resize(nt);
    or_mesh_derived(X, nv, T, nt, m.normal.data(), m.area.data(), m.center.data(), m.maxL.data());
    m.M.resize(9 * (size_t)nt); m.v.resize(3 * (size_t)nt);
    for (int t = 0; t < nt; t++) {
        double V[3][3];
        m.vert(t, V);
        double n[3];
        if (unit_normal) {
            for (int c = 0; c < 3; c++) n[c] = m.normal[3 * t + c];
        } else {
            double l21[3], l31[3];
            for (int c = 0; c < 3; c++) { l21[c] = V[1][c] - V[0][c]; l31[c] = V[2][c] - V[0][c]; }
            cross3(l21, l31, n);
        }
        p1_coeffs(V, n, &m.M[9 * (size_t)t], &m.v[3 * (size_t)t]);
        if (m.maxL[t] > m.maxLen) m.maxLen = m.maxL[t];
    }
    return m;
}

double phi(const DMesh& m, int t, int k /*1..3*/, const double y[3]) {
    const double* M = &m.M[9 * (size_t)t + 3 * (k - 1)];
    return m.v[3 * (size_t)t + k - 1] + M[0] * y[0] + M[1] * y[1] + M[2] * y[2];
}

int levi(int a, int b, int c) {   // Levi-Civita symbol, 0-based indices
    if (a == b || b == c || a == c) return 0;
    return ((a + 1) % 3 == b) ? 1 : -1;
}

struct Mat { double lam, mu, rho, cP, cS; };

// Time factors of the direct kernels at (r, t).
struct TF {
    double HP, HS;      // Heaviside of the fronts
    double RP, RS;      // (t - r/c) H
    double SP, SS;      // (t - r/c)^2 (t + 2 r/c) / 6 H
};
TF tfac(double r, double t, const Mat& p) {
    TF f;
    double aP = t - r / p.cP, aS = t - r / p.cS;
    f.HP = aP > 0 ? 1.0 : 0.0;
    f.HS = aS > 0 ? 1.0 : 0.0;
    f.RP = aP * f.HP;
    f.RS = aS * f.HS;
    f.SP = aP * aP * (t + 2 * r / p.cP) / 6 * f.HP;
    f.SS = aS * aS * (t + 2 * r / p.cS) / 6 * f.HS;
    return f;
}

// Double-layer kernel of kernelK.cu (nucleoKL + nucleoKT + nucleoKR) for the
// P1 basis function k of the field triangle: x = outer - inner node, n the
// field normal, vms = n x grad(phi_k), phik = phi_k(inner node).  with_xn
// adds the (x.n) terms (false for the coplanar singular part,
// BEMenerg_dir_calcKIntgSing.m), bad_front reproduces H(r - r/c_P).
void kernel_k(double out[3][3], const double x[3], double r, const double n[3], double t, const double vms[3],
              double phik, const Mat& p, bool with_xn, bool bad_front) {
    TF f = tfac(r, t, p);
    const double a1 = p.lam / (p.lam + p.mu), a2 = p.mu / (p.lam + p.mu);
    const double c1 = p.lam * p.mu / (p.rho * (p.lam + p.mu)), c2 = 2 * p.mu / p.rho;
    const double r2 = r * r, r3 = r2 * r, r5 = r3 * r2;
    const double xn = dot3(x, n);
    const double D = f.RP - f.RS, DT = f.HP / p.cP - f.HS / p.cS;
    const double RPl = bad_front ? (t - r / p.cP) * ((r - r / p.cP) > 0 ? 1.0 : 0.0) : f.RP;
    const double Dl = f.RS / (p.cS * p.cS) - RPl / (p.cP * p.cP);
    const double Dd = f.RS / (p.cS * p.cS) - f.RP / (p.cP * p.cP);
    const double Hh = f.SS - f.SP;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            const double dik = (i == k) ? 1.0 : 0.0;
            double kl = (a1 * x[i] * n[k] + a2 * x[k] * n[i]) / r3 * D;
            double kt = (a1 * x[i] * n[k] + a2 * x[k] * n[i]) / r2 * DT;
            if (with_xn) {
                kl += dik * xn / r3 * f.RS;
                kt += dik * xn / r2 * f.HS / p.cS;
            }
            double kr = 0.0;
            for (int j = 0; j < 3; j++) {
                double s = c1 * levi(j, k, i) / r * Dl;
                double h = 0.0, d = 0.0;
                for (int q = 0; q < 3; q++) {
                    const double e = levi(j, i, q);
                    if (e == 0) continue;
                    h += e * (3 * x[q] * x[k] / r5 - ((q == k) ? 1.0 : 0.0) / r3);
                    d += e * (x[q] * x[k] / r3);
                }
                kr += vms[j] * (s + c2 * h * Hh + c2 * d * Dd);
            }
            out[i][k] = -kr + phik * (kl + kt);
        }
}

// Lame kernel twice integrated in time (kernelGHC.cu:204-259 / calcSubBlockDiagV.m:9-59).
void kernel_v(double nu[3][3], const double x[3], double r, double t, double cP, double cS) {
    const double HP = (t - r / cP) > 0 ? 1.0 : 0.0, HS = (t - r / cS) > 0 ? 1.0 : 0.0;
    const double r3 = r * r * r, r5 = r3 * r * r;
    const double tail = (cP * cP * t * t - r * r) / (cP * cP) * HP - (cS * cS * t * t - r * r) / (cS * cS) * HS;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const double xx = x[i] * x[j], d = (i == j) ? 1.0 : 0.0;
            nu[i][j] = (xx / r3) * (1 / (cP * cP)) * HP + (d / r - xx / r3) * (1 / (cS * cS)) * HS -
                       0.5 * (d / r3 - 3 * (xx / r5)) * tail;
        }
}

// Traction kernel of kernelP.cu (nucleo) times phi: x = source - node.
void kernel_p(double nu[3][3], const double x[3], const double n[3], double r, double t, double phik, const Mat& p) {
    TF f = tfac(r, t, p);
    const double xn = dot3(x, n);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r7 = r5 * r2;
    const double lam = p.lam, mu = p.mu;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const double d = (i == j) ? 1.0 : 0.0;
            const double xinj = x[i] * n[j], xjni = x[j] * n[i], xx = x[j] * x[i];
            double v = (lam * xinj / r2 + 2 * mu * xx / r4 * xn) * (f.HP / (p.cP * p.cP * p.cP)) +
                       mu * (xjni / r2 + (d / r2 - 2 * xx / r4) * xn) * (f.HS / (p.cS * p.cS * p.cS)) +
                       ((lam - 2 * mu) * xinj / r3 - 2 * mu * xjni / r3 - 2 * mu * (d / r3 - 6 * xx / r5) * xn) *
                           (f.RP / (p.cP * p.cP)) +
                       mu * (2 * xinj / r3 + 3 * xjni / r3 + 3 * (d / r3 - 4 * xx / r5) * xn) * (f.RS / (p.cS * p.cS)) -
                       6 * mu * (xinj / r5 + xjni / r5 + (d / r5 - 5 * xx / r7) * xn) * (f.SP - f.SS);
            nu[i][j] = v * phik;
        }
}

// Tree reduction of per-thread 3x3 partial sums in the order of the reference
// kernels: y to a power of two, y halving, then x halving.
void reduce_xy(std::vector<double>& sm, int bx, int by) {
    int yDim = 1;
    while (yDim * 2 <= by) yDim *= 2;
    for (int tx = 0; tx < bx; tx++)
        for (int ty = 0; ty < by; ty++)
            if (ty + yDim < by)
                for (int e = 0; e < 9; e++) sm[(size_t)(tx * by + ty) * 9 + e] += sm[(size_t)(tx * by + ty + yDim) * 9 + e];
    for (yDim /= 2; yDim > 0; yDim /= 2)
        for (int tx = 0; tx < bx; tx++)
            for (int ty = 0; ty < yDim; ty++)
                for (int e = 0; e < 9; e++) sm[(size_t)(tx * by + ty) * 9 + e] += sm[(size_t)(tx * by + ty + yDim) * 9 + e];
    for (int xDim = bx / 2; xDim > 0; xDim /= 2)
        for (int tx = 0; tx < xDim; tx++)
            for (int ty = 0; ty < by; ty++)
                for (int e = 0; e < 9; e++) sm[(size_t)(tx * by + ty) * 9 + e] += sm[(size_t)((tx + xDim) * by + ty) * 9 + e];
}

void set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

}  // namespace

extern "C" {

int or_p1_coeffs(const double* coords, int nv, const int* tris, int nt, int unit_normal, double* M, double* v) {
    DMesh m = make(coords, nv, tris, nt, unit_normal != 0);
    std::memcpy(M, m.M.data(), sizeof(double) * 9 * (size_t)nt);
    std::memcpy(v, m.v.data(), sizeof(double) * 3 * (size_t)nt);
    return 0;
}

// doppioGauss1D(n): n = n1^2 nodes, n1-point Gauss-Legendre on (0, 1) in
// both directions of the collapsed square; node k = i + n1 j has barycentric
// coordinates ((1-x_j)(1-x_i), x_j (1-x_i), x_i) and weight 2 w_i w_j (1-x_i).
// The Gauss-Legendre nodes come from Newton's iteration on P_n1 (the values
// of the reference's eigenvalue routine to rounding), ascending.
int or_doppio_gauss(int n, double* nodes, double* w) {
    int n1 = (int)std::lround(std::sqrt((double)n));
    if (n1 < 1 || n1 * n1 != n) return -1;
    std::vector<double> x(n1), wt(n1);
    for (int i = 0; i < n1; i++) {
        double z = std::cos(PI * (i + 0.75) / (n1 + 0.5)), pp = 1;
        for (int it = 0; it < 100; it++) {
            double p0 = 1, p1 = z;
            for (int k = 2; k <= n1; k++) { double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
            if (n1 == 1) { p1 = z; p0 = 1; }
            pp = n1 * (z * p1 - p0) / (z * z - 1);
            double dz = p1 / pp;
            z -= dz;
            if (std::fabs(dz) < 1e-17) break;
        }
        double p0 = 1, p1 = z;
        for (int k = 2; k <= n1; k++) { double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
        pp = n1 * (z * p1 - p0) / (z * z - 1);
        x[n1 - 1 - i] = z;
        wt[n1 - 1 - i] = 2 / ((1 - z * z) * pp * pp);
    }
    if (n1 == 1) { x[0] = 0; wt[0] = 2; }
    for (int i = 0; i < n1; i++) { x[i] = 0.5 + x[i] / 2; wt[i] = wt[i] / 2; }
    for (int j = 0; j < n1; j++)
        for (int i = 0; i < n1; i++) {
            int k = i + n1 * j;
            nodes[3 * k] = (1 - x[j]) * (1 - x[i]);
            nodes[3 * k + 1] = x[j] * (1 - x[i]);
            nodes[3 * k + 2] = x[i];
            w[k] = 2 * wt[j] * (wt[i] * (1 - x[i]));
        }
    return 0;
}

// K_l off the singular (same-triangle) part, kernelK.cu: K is L x (3N) x
// (3 Nv) column-major per lag (entry (3x+i, 3s+j) of lag q at
// q 9 N Nv + 3N (3s+j) + 3x+i), accumulated (+=) where |value| > 1e-14,
// divided by 4 pi dt.  Rule: outer GH n_gh, inner composite (n_sub, n_sing).
int or_assemble_k(const double* coords, int nv, const int* tris, int nt, double rho, double mu, double lambda,
                  double dt, int n_gh, int n_sub, int n_sing, int lag0, int nlag, int nblocks, int fix, double* K,
                  int nthreads) {
    std::vector<double> ghn(3 * n_gh), ghw(n_gh), gcn(3 * (size_t)n_sub * n_sing), gcw(n_sing);
    if (or_gh(n_gh, 1, ghn.data(), ghw.data()) != 0) return -1;
    if (or_gh(n_sing, n_sub, gcn.data(), gcw.data()) != 0) return -1;
    DMesh m = make(coords, nv, tris, nt, false);
    Mat p{lambda, mu, rho, std::sqrt((lambda + 2 * mu) / rho), std::sqrt(mu / rho)};
    set_threads(nthreads);
    const size_t R = 3 * (size_t)nt, C = 3 * (size_t)nv;
    const int bx = n_sub, by = n_sing;
    for (int q = 0; q < nlag; q++) {
        const int z = lag0 + q;
        if (z >= nblocks) continue;
        double* Kl = K + (size_t)q * R * C;
#pragma omp parallel for schedule(dynamic, 16)
        for (long long ind = 0; ind < (long long)nt * nv; ind++) {
            const int x = (int)(ind % nt), s = (int)(ind / nt);
            double VS[3][3];
            m.vert(x, VS);
            // isBlockNull (kernelK.cu:234-262)
            double distMax = 0, distMin = fix ? 1e300 : 100.0;
            for (int a = 0; a < 3; a++) {
                double dv[3] = {VS[a][0] - coords[3 * s], VS[a][1] - coords[3 * s + 1], VS[a][2] - coords[3 * s + 2]};
                double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                if (d > distMax) distMax = d;
                if (d < distMin) distMin = d;
            }
            if (((z - 2) * p.cS * dt > distMax + m.maxLen) || ((z + 1) * p.cP * dt < distMin - 2 * m.maxLen)) continue;
            std::vector<double> sm((size_t)bx * by * 9, 0.0);
            for (int tx = 0; tx < bx; tx++)
                for (int ty = 0; ty < by; ty++) {
                    double* acc = &sm[(size_t)(tx * by + ty) * 9];
                    for (int fm = 0; fm < nt; fm++) {
                        if (fm == x) continue;
                        const int k = m.local(fm, s);
                        if (k == 0) continue;
                        const double* n = &m.normal[3 * (size_t)fm];
                        double VF[3][3];
                        m.vert(fm, VF);
                        const double pesoInt = gcw[ty] * m.area[fm];
                        const double* nd = &gcn[3 * (size_t)(tx * by + ty)];
                        double y[3];
                        for (int c = 0; c < 3; c++) y[c] = nd[0] * VF[0][c] + nd[1] * VF[1][c] + nd[2] * VF[2][c];
                        double gradk[3] = {m.M[9 * (size_t)fm + 3 * (k - 1)], m.M[9 * (size_t)fm + 3 * (k - 1) + 1],
                                           m.M[9 * (size_t)fm + 3 * (k - 1) + 2]};
                        double vms[3];
                        cross3(n, gradk, vms);
                        const double phik = phi(m, fm, k, y);
                        for (int l = 0; l < n_gh; l++) {
                            const double pesoExt = ghw[l] * m.area[x];
                            const double* ne = &ghn[3 * l];
                            double xo[3], pt[3];
                            for (int c = 0; c < 3; c++) xo[c] = ne[0] * VS[0][c] + ne[1] * VS[1][c] + ne[2] * VS[2][c];
                            for (int c = 0; c < 3; c++) pt[c] = xo[c] - y[c];
                            const double r = std::sqrt(pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2]);
                            const int cN[4] = {-1, 3, -3, 1}, cT[4] = {-2, -1, 0, 1};
                            for (int kk = 0; kk < 4; kk++) {
                                const double t = dt * (z + cT[kk]);
                                if (t <= 0) continue;
                                double T[3][3];
                                kernel_k(T, pt, r, n, t, vms, phik, p, true, !fix);
                                for (int i = 0; i < 3; i++)
                                    for (int j = 0; j < 3; j++) acc[3 * i + j] += pesoExt * pesoInt * cN[kk] * T[i][j];
                            }
                        }
                    }
                }
            reduce_xy(sm, bx, by);
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    const double v = sm[3 * i + j];
                    if (std::fabs(v) > 1.0e-14) Kl[(3 * (size_t)s + j) * R + 3 * (size_t)x + i] += v / (4 * PI * dt);
                }
        }
    }
    return 0;
}

// Singular parts of K_l (calcSubBlockSingK.m + calcKIntgSing.m): for each
// triangle x and each of its vertices, the same-triangle integral on the DIAG
// rule (n_diag nodes on each of the three children (V_c, V_c', node) of every
// outer node), added to the (3x, 3 vertex) block.  No clamp, / (4 pi dt).
int or_k_sing(const double* coords, int nv, const int* tris, int nt, double rho, double mu, double lambda, double dt,
              int n_gh, int n_diag, int lag0, int nlag, double* K, int nthreads) {
    std::vector<double> ghn(3 * n_gh), ghw(n_gh), dn(3 * (size_t)n_diag), dw(n_diag);
    if (or_gh(n_gh, 1, ghn.data(), ghw.data()) != 0) return -1;
    if (or_doppio_gauss(n_diag, dn.data(), dw.data()) != 0) return -1;
    DMesh m = make(coords, nv, tris, nt, false);
    Mat p{lambda, mu, rho, std::sqrt((lambda + 2 * mu) / rho), std::sqrt(mu / rho)};
    set_threads(nthreads);
    const size_t R = 3 * (size_t)nt, C = 3 * (size_t)nv;
    for (int q = 0; q < nlag; q++) {
        const int z = lag0 + q;
        double* Kl = K + (size_t)q * R * C;
#pragma omp parallel for schedule(dynamic, 4)
        for (int x = 0; x < nt; x++) {
            if (z >= (int)std::ceil(m.maxL[x] / (p.cS * dt)) + 2) continue;
            double V[3][3];
            m.vert(x, V);
            const double* n = &m.normal[3 * (size_t)x];
            for (int kv = 1; kv <= 3; kv++) {
                const double* gk = &m.M[9 * (size_t)x + 3 * (kv - 1)];
                double vms[3];
                cross3(n, gk, vms);
                double blk[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                const int cT[4] = {-2, -1, 0, 1}, cN[4] = {-1, 3, -3, 1};
                for (int kk = 0; kk < 4; kk++) {
                    const int ist = z + cT[kk];
                    if (ist <= 0) continue;
                    const double t = ist * dt;
                    double tot[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                    for (int l = 0; l < n_gh; l++) {
                        double xo[3];
                        const double* ne = &ghn[3 * l];
                        for (int c = 0; c < 3; c++) xo[c] = ne[0] * V[0][c] + ne[1] * V[1][c] + ne[2] * V[2][c];
                        const double pesoExt = m.area[x] * ghw[l];
                        double in[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                        for (int ch = 0; ch < 3; ch++) {
                            const int a = ch, b = (ch + 2) % 3;     // children (V1,V3,x), (V2,V1,x), (V3,V2,x)
                            double ea[3], eb[3], cr[3];
                            for (int c = 0; c < 3; c++) { ea[c] = V[a][c] - xo[c]; eb[c] = V[b][c] - xo[c]; }
                            cross3(ea, eb, cr);
                            const double ac = std::sqrt(dot3(cr, cr)) / 2;
                            for (int d = 0; d < n_diag; d++) {
                                const double* bd = &dn[3 * (size_t)d];
                                double y[3];
                                for (int c = 0; c < 3; c++) y[c] = bd[0] * V[a][c] + bd[1] * V[b][c] + bd[2] * xo[c];
                                const double pesoInt = dw[d] * ac;
                                double R3[3] = {xo[0] - y[0], xo[1] - y[1], xo[2] - y[2]};
                                const double r = std::sqrt(dot3(R3, R3));
                                double T[3][3];
                                kernel_k(T, R3, r, n, t, vms, phi(m, x, kv, y), p, false, false);
                                for (int i = 0; i < 3; i++)
                                    for (int j = 0; j < 3; j++) in[i][j] += pesoInt * T[i][j];
                            }
                        }
                        for (int i = 0; i < 3; i++)
                            for (int j = 0; j < 3; j++) tot[i][j] += pesoExt * in[i][j];
                    }
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) blk[i][j] += cN[kk] * tot[i][j];
                }
                const int s = tris[3 * x + kv - 1];
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) Kl[(3 * (size_t)s + j) * R + 3 * (size_t)x + i] += blk[i][j] / (4 * PI * dt);
            }
        }
    }
    return 0;
}

// Diagonal blocks of V_l on the DIAG rule (calcSubBlockDiagV.m): written
// (not accumulated) into V (L x 3N x 3N column-major per lag).
int or_v_diag(const double* coords, int nv, const int* tris, int nt, double rho, double mu, double lambda, double dt,
              int n_gh, int n_diag, int lag0, int nlag, double* Vout, int nthreads) {
    std::vector<double> ghn(3 * n_gh), ghw(n_gh), dn(3 * (size_t)n_diag), dw(n_diag);
    if (or_gh(n_gh, 1, ghn.data(), ghw.data()) != 0) return -1;
    if (or_doppio_gauss(n_diag, dn.data(), dw.data()) != 0) return -1;
    DMesh m = make(coords, nv, tris, nt, false);
    const double cP = std::sqrt((lambda + 2 * mu) / rho), cS = std::sqrt(mu / rho);
    set_threads(nthreads);
    const size_t R = 3 * (size_t)nt;
    for (int q = 0; q < nlag; q++) {
        const int z = lag0 + q;
        double* Vl = Vout + (size_t)q * R * R;
#pragma omp parallel for schedule(dynamic, 4)
        for (int x = 0; x < nt; x++) {
            double V[3][3];
            m.vert(x, V);
            double ris[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            const int ist3[3] = {z + 1, z, z - 1};
            const double coef[3] = {1, -2, 1};
            for (int k = 0; k < 3; k++) {
                if (ist3[k] <= 0) continue;
                const double t = ist3[k] * dt;
                double tot[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                for (int l = 0; l < n_gh; l++) {
                    double xo[3];
                    const double* ne = &ghn[3 * l];
                    for (int c = 0; c < 3; c++) xo[c] = ne[0] * V[0][c] + ne[1] * V[1][c] + ne[2] * V[2][c];
                    double in[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                    for (int ch = 0; ch < 3; ch++) {
                        const int a = ch, b = (ch + 2) % 3;
                        double ea[3], eb[3], cr[3];
                        for (int c = 0; c < 3; c++) { ea[c] = V[a][c] - xo[c]; eb[c] = V[b][c] - xo[c]; }
                        cross3(ea, eb, cr);
                        const double ac = std::sqrt(dot3(cr, cr)) / 2;
                        for (int d = 0; d < n_diag; d++) {
                            const double* bd = &dn[3 * (size_t)d];
                            double y[3];
                            for (int c = 0; c < 3; c++) y[c] = bd[0] * V[a][c] + bd[1] * V[b][c] + bd[2] * xo[c];
                            double X3[3] = {y[0] - xo[0], y[1] - xo[1], y[2] - xo[2]};
                            double nu[3][3];
                            kernel_v(nu, X3, std::sqrt(dot3(X3, X3)), t, cP, cS);
                            for (int i = 0; i < 3; i++)
                                for (int j = 0; j < 3; j++) in[i][j] += dw[d] * ac * nu[i][j];
                        }
                    }
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) tot[i][j] += m.area[x] * ghw[l] * in[i][j];
                }
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) ris[i][j] += coef[k] * tot[i][j];
            }
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) Vl[(3 * (size_t)x + j) * R + 3 * (size_t)x + i] = ris[i][j] / (4 * PI * rho);
        }
    }
    return 0;
}

// Direct post-processing single-layer matrix of kernelG.cu at one point x and
// time t: G is (3 nHat) x (3N) column-major, nHat = ceil(t / dt) time slices,
// slice y combines G(t - y dt) - G(t - (y+1) dt).  Rule: composite
// (n_sub, n_sing); `fix` = 0 keeps the node stride 3 of kernelG.cu:51.
int or_pp_dir_g(const double* coords, int nv, const int* tris, int nt, double rho, double mu, double lambda,
                double dt, int n_sub, int n_sing, const double* xsrc, double t, int fix, double* G) {
    std::vector<double> pn(3 * (size_t)n_sub * n_sing), pw(n_sing);
    if (or_gh(n_sing, n_sub, pn.data(), pw.data()) != 0) return -1;
    if (!fix && 3 * (n_sub - 1) + n_sing > n_sub * n_sing) return -1;   // the reference would read out of bounds
    DMesh m = make(coords, nv, tris, nt, true);
    const double cP = std::sqrt((lambda + 2 * mu) / rho), cS = std::sqrt(mu / rho);
    const int nHat = (int)std::ceil(t / dt);
    if (t <= 0 || nHat <= 0) return 0;
    const size_t R = 3 * (size_t)nHat;
    const int stride = fix ? n_sing : 3;
    for (int x = 0; x < nt; x++) {
        double V[3][3];
        m.vert(x, V);
        for (int yb = 0; yb < nHat; yb++) {
            std::vector<double> sm((size_t)n_sub * 9, 0.0);
            for (int tx = 0; tx < n_sub; tx++) {
                double* acc = &sm[(size_t)tx * 9];
                const double cT[2] = {-1, 0}, cN[2] = {1, -1};
                for (int k = 0; k < 2; k++) {
                    const double tc = t - (yb + 1 + cT[k]) * dt;
                    if (tc <= 0) continue;
                    for (int l = 0; l < n_sing; l++) {
                        const double* nd = &pn[3 * (size_t)(stride * tx + l)];
                        double y[3];
                        for (int c = 0; c < 3; c++) y[c] = nd[0] * V[0][c] + nd[1] * V[1][c] + nd[2] * V[2][c];
                        const double w = pw[l] * m.area[x];
                        double pt[3] = {y[0] - xsrc[0], y[1] - xsrc[1], y[2] - xsrc[2]};
                        double nu[3][3];
                        kernel_v(nu, pt, std::sqrt(dot3(pt, pt)), tc, cP, cS);
                        for (int i = 0; i < 3; i++)
                            for (int j = 0; j < 3; j++) acc[3 * i + j] += cN[k] * w * nu[i][j];
                    }
                }
            }
            for (int xd = n_sub / 2; xd > 0; xd /= 2)
                for (int tx = 0; tx < xd; tx++)
                    for (int e = 0; e < 9; e++) sm[(size_t)tx * 9 + e] += sm[(size_t)(tx + xd) * 9 + e];
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    const double v = sm[3 * i + j];
                    if (std::fabs(v) > 1.0e-14) G[(3 * (size_t)x + j) * R + 3 * (size_t)yb + i] += v / (4 * PI * rho);
                }
        }
    }
    return 0;
}

// Direct post-processing double-layer matrix of kernelP.cu: P is (3 nHat) x
// (3 Nv), slice y combines P(t - y dt) - 2 P(t - (y+1) dt) + P(t - (y+2) dt),
// divided by 4 pi rho dt.
int or_pp_dir_p(const double* coords, int nv, const int* tris, int nt, double rho, double mu, double lambda,
                double dt, int n_sub, int n_sing, const double* xsrc, double t, double* P) {
    std::vector<double> pn(3 * (size_t)n_sub * n_sing), pw(n_sing);
    if (or_gh(n_sing, n_sub, pn.data(), pw.data()) != 0) return -1;
    DMesh m = make(coords, nv, tris, nt, true);
    Mat p{lambda, mu, rho, std::sqrt((lambda + 2 * mu) / rho), std::sqrt(mu / rho)};
    const int nHat = (int)std::ceil(t / dt);
    if (t <= 0 || nHat <= 0) return 0;
    const size_t R = 3 * (size_t)nHat;
    for (int s = 0; s < nv; s++)
        for (int yb = 0; yb < nHat; yb++) {
            std::vector<double> sm((size_t)n_sub * 9, 0.0);
            for (int tx = 0; tx < n_sub; tx++) {
                double* acc = &sm[(size_t)tx * 9];
                const double cT[3] = {-1, 0, 1}, cN[3] = {1, -2, 1};
                for (int k = 0; k < 3; k++) {
                    const double tc = t - (yb + 1 + cT[k]) * dt;
                    if (tc <= 0) continue;
                    for (int fm = 0; fm < nt; fm++) {
                        const int kv = m.local(fm, s);
                        if (kv == 0) continue;
                        const double* n = &m.normal[3 * (size_t)fm];
                        double V[3][3];
                        m.vert(fm, V);
                        for (int l = 0; l < n_sing; l++) {
                            const double* nd = &pn[3 * (size_t)(n_sing * tx + l)];
                            double y[3];
                            for (int c = 0; c < 3; c++) y[c] = nd[0] * V[0][c] + nd[1] * V[1][c] + nd[2] * V[2][c];
                            const double w = pw[l] * m.area[fm];
                            double pt[3] = {xsrc[0] - y[0], xsrc[1] - y[1], xsrc[2] - y[2]};
                            double nu[3][3];
                            kernel_p(nu, pt, n, std::sqrt(dot3(pt, pt)), tc, phi(m, fm, kv, y), p);
                            for (int i = 0; i < 3; i++)
                                for (int j = 0; j < 3; j++) acc[3 * i + j] += cN[k] * w * nu[i][j];
                        }
                    }
                }
            }
            for (int xd = n_sub / 2; xd > 0; xd /= 2)
                for (int tx = 0; tx < xd; tx++)
                    for (int e = 0; e < 9; e++) sm[(size_t)tx * 9 + e] += sm[(size_t)(tx + xd) * 9 + e];
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    const double v = sm[3 * i + j];
                    if (std::fabs(v) > 1.0e-14) P[(3 * (size_t)s + j) * R + 3 * (size_t)yb + i] += v / (4 * PI * rho * dt);
                }
        }
    return 0;
}

}  // extern "C"
