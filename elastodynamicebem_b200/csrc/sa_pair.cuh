// Per-pair algebra of the semi-analytic assembly shared by the CUDA kernels
// (and compilable as host code): the per-triangle preparation, the
// projection of an outer node on the field plane, the case split, the null
// test and the combined kernel integral F(t_k) of one (source, field) pair.
//
// Reference ("SA/" = functions/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/):
//   frame            SA/calcoloMatrice/operazioniGeometriche/calcoloSistemaRiferimento.m
//   Euler matrix     SA/calcoloMatrice/operazioniGeometriche/rotazioneInversaEulero.m:23-176
//   projection       SA/calcoloMatrice/operazioniGeometriche/preparazioneTriangolo.m:1-115
//   edge distance    SA/calcoloMatrice/operazioniGeometriche/calcoloDistanzaTriangolo.m
//   children         SA/calcoloMatrice/BEMenerg_coreSA_calcIntgInt_fieldTriangle.m:13-84
//   case split       SA/calcoloMatrice/BEMenerg_coreSA_calcMatrixSubBlock.m:58-81
//   null test        SA/calcoloMatrice/BEMenerg_coreSA_calcMatrixBlock.m:57-61
#pragma once

#include "sa_device.cuh"
#include "sa_edge.cuh"

// 1: child integrals in the edge variable (stable; default); 0: the
// reference's closed-form region formulas (for comparison)
#ifndef EBEM_SA_FORM
#define EBEM_SA_FORM 1
#endif

namespace ebem {

// Mapped outer node and its area-scaled weight.
#ifdef __CUDACC__
struct __align__(32) NodeW { double x, y, z, w; };
#else
struct alignas(32) NodeW { double x, y, z, w; };
#endif

EBEM_DI void euler_matrix(const double e1[3], const double n[3], double C[9]) {
    // rotazioneInversaEulero.m:23-91; X = e1, Z = n, canonical e1 = x, e3 = z
    const double* X = e1;
    const double* Z = n;
    double cz0 = -Z[1], cz1 = Z[0];          // cross(e3, Z) = (-Z2, Z1, 0)
    double ncz = sqrt(cz0 * cz0 + cz1 * cz1);
    double phi, omega, psi;
    if (ncz < 1.0e-10) {
        phi = acos_c(X[0]);
        if (X[1] < -1.0e-10) phi = 2 * kPi - phi;          // cross(e1, X) . e3 = X2
        omega = (Z[2] < 0) ? kPi : 0.0;
        psi = 0.0;
    } else {
        double l0 = cz0 / ncz, l1 = cz1 / ncz;              // l_nodi (third component 0)
        phi = acos_c(l0);
        if (l1 < -1.0e-10) phi = 2 * kPi - phi;
        omega = acos_c(Z[2]);
        psi = acos_c(l0 * X[0] + l1 * X[1]);
        // cross(l, X) . Z
        double cx = l1 * X[2], cy = -l0 * X[2], cw = l0 * X[1] - l1 * X[0];
        if (cx * Z[0] + cy * Z[1] + cw * Z[2] < -1.0e-10) psi = 2 * kPi - psi;
    }
    double cps, sps, co, so, cf, sf;
    sincos(psi, &sps, &cps);
    sincos(omega, &so, &co);
    sincos(phi, &sf, &cf);
    // C = A_psi * A_omega * A_phi
    double Ap[9] = {cps, sps, 0, -sps, cps, 0, 0, 0, 1};
    double Ao[9] = {1, 0, 0, 0, co, so, 0, -so, co};
    double Af[9] = {cf, sf, 0, -sf, cf, 0, 0, 0, 1};
    double T[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            T[3 * r + c] = Ap[3 * r] * Ao[c] + Ap[3 * r + 1] * Ao[3 + c] + Ap[3 * r + 2] * Ao[6 + c];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            double v = T[3 * r] * Af[c] + T[3 * r + 1] * Af[3 + c] + T[3 * r + 2] * Af[6 + c];
            C[3 * r + c] = (fabs(v) < 1.0e-14) ? 0.0 : v;
        }
}


// Per-triangle geometry of one triangle with vertices V (prep stage):
// readSpaceMesh.m:93-139 (normal, area, centroid, longest edge),
// calcoloSistemaRiferimento.m (frame) and the Euler matrix.
EBEM_DI void tri_geom(const double V[3][3], TriGeom& g) {
    double vg1[3], vg2[3], vg3[3];
    for (int c = 0; c < 3; c++) { vg1[c] = V[0][c] - V[2][c]; vg2[c] = V[1][c] - V[2][c]; vg3[c] = V[0][c] - V[1][c]; }
    double nn[3];
    nn[0] = vg1[1] * vg2[2] - vg2[1] * vg1[2];
    nn[1] = -vg1[0] * vg2[2] + vg2[0] * vg1[2];
    nn[2] = vg1[0] * vg2[1] - vg2[0] * vg1[1];
    double area = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]) / 2;
    g.area = area;
    for (int c = 0; c < 3; c++) g.n[c] = nn[c] / (2 * area);
    for (int c = 0; c < 3; c++) g.ctr[c] = (V[0][c] + V[1][c] + V[2][c]) / 3;
    double l1 = sqrt(vg3[0] * vg3[0] + vg3[1] * vg3[1] + vg3[2] * vg3[2]);
    double l2 = sqrt(vg2[0] * vg2[0] + vg2[1] * vg2[1] + vg2[2] * vg2[2]);
    double l3 = sqrt(vg1[0] * vg1[0] + vg1[1] * vg1[1] + vg1[2] * vg1[2]);
    g.maxL = fmax(fmax(l1, l2), l3);
    for (int c = 0; c < 3; c++) g.P1[c] = V[0][c];
    double a[3] = {V[1][0] - V[0][0], V[1][1] - V[0][1], V[1][2] - V[0][2]};
    g.L1 = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int c = 0; c < 3; c++) g.e1[c] = a[c] / g.L1;
    double b[3] = {V[2][0] - V[0][0], V[2][1] - V[0][1], V[2][2] - V[0][2]};
    g.L3 = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    double e3[3];
    for (int c = 0; c < 3; c++) e3[c] = b[c] / g.L3;
    g.cd = e3[0] * g.e1[0] + e3[1] * g.e1[1] + e3[2] * g.e1[2];
    g.sd = sin(acos_c(g.cd));
    double e2[3] = {g.n[1] * g.e1[2] - g.n[2] * g.e1[1], g.n[2] * g.e1[0] - g.n[0] * g.e1[2],
                    g.n[0] * g.e1[1] - g.n[1] * g.e1[0]};
    double ne2 = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    for (int c = 0; c < 3; c++) g.e2[c] = e2[c] / ne2;
    euler_matrix(g.e1, g.n, g.C);
    g.pad = 0.0;
}

// Node-level geometry: the projection of preparazioneTriangolo.m — the field
// triangle in the plane frame centred at the projected node, the signed
// doubled areas of the three children, zeta, the side of the node and d_min.
struct NodeGeo {
    double zeta, sigma, dMIN;
    double tri[3][2];
    double c[3];
};

EBEM_DI double edge_distance(const double tri[3][2]) {
    // calcoloDistanzaTriangolo.m:1-52 (min over the three sides, NaN skipped)
    double D[3];
#pragma unroll
    for (int k = 0; k < 3; k++) D[k] = sqrt(tri[k][0] * tri[k][0] + tri[k][1] * tri[k][1]);
    const int pa[3] = {0, 1, 0}, pb[3] = {1, 2, 2};
    double best = INFINITY;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double* P1 = tri[pa[i]];
        const double* P2 = tri[pb[i]];
        double d1 = D[pa[i]], d2 = D[pb[i]];
        double vx = P2[0] - P1[0], vy = P2[1] - P1[1];
        double L = sqrt(vx * vx + vy * vy);
        double d;
        if (-(P1[0] * vx + P1[1] * vy) < -1.0e-6) d = d1;
        else if (-(P2[0] * (-vx) + P2[1] * (-vy)) < -1.0e-6) d = d2;
        else {
            double ca = (-P1[0] / d1) * (vx / L) + (-P1[1] / d1) * (vy / L);
            d = d1 * sqrt_c(1 - ca * ca);
        }
        if (d < best) best = d;          // NaN compares false: skipped as MATLAB min does
    }
    return (best == INFINITY) ? 0.0 : best;
}

EBEM_DI void node_geo(NodeGeo& G, const NodeW& sp, const TriGeom& F) {
    double ds0 = sp.x - F.P1[0], ds1 = sp.y - F.P1[1], ds2 = sp.z - F.P1[2];
    double param_s = F.n[0] * ds0 + F.n[1] * ds1 + F.n[2] * ds2;
    double pp0 = sp.x - param_s * F.n[0], pp1 = sp.y - param_s * F.n[1], pp2 = sp.z - param_s * F.n[2];
    double sp_ = (sp.x - pp0) * F.n[0] + (sp.y - pp1) * F.n[1] + (sp.z - pp2) * F.n[2];
    if (fabs(sp_) <= 1.0e-6) sp_ = 0.0;
    G.sigma = sgn(sp_);
    G.zeta = fabs(param_s);
    if (G.zeta < 1.0e-6) G.zeta = 0.0;
    double df0 = F.P1[0] - pp0, df1 = F.P1[1] - pp1, df2 = F.P1[2] - pp2;
    double (*tri)[2] = G.tri;
    tri[0][0] = df0 * F.e1[0] + df1 * F.e1[1] + df2 * F.e1[2];
    tri[0][1] = df0 * F.e2[0] + df1 * F.e2[1] + df2 * F.e2[2];
    tri[1][0] = tri[0][0] + F.L1;
    tri[1][1] = tri[0][1];
    tri[2][0] = tri[0][0] + F.L3 * F.cd;
    tri[2][1] = tri[0][1] + F.L3 * F.sd;
    double* c = G.c;
    c[0] = (tri[0][0] * tri[1][1]) - (tri[0][1] * tri[1][0]);
    c[1] = (tri[1][0] * tri[2][1]) - (tri[1][1] * tri[2][0]);
    c[2] = (tri[2][0] * tri[0][1]) - (tri[2][1] * tri[0][0]);
    double Ad = (tri[1][0] - tri[0][0]) * (tri[2][1] - tri[0][1]);
    double eta2 = c[2] / Ad, eta3 = c[0] / Ad, eta1 = 1 - eta2 - eta3;
    bool inside = (-1.0e-6 <= eta1) && (-1.0e-6 <= eta2) && (-1.0e-6 <= eta3) && (eta1 <= 1) && (eta2 <= 1) &&
                  (eta3 <= 1);
    G.dMIN = inside ? 0.0 : edge_distance(tri);
}

// Child k = (O, P_k, P_k+1) of a projected node, oriented counter-clockwise
// (fieldTriangle.m:22-33); false when the child is degenerate (|c| < 1e-6).
EBEM_DI bool node_child(ChildGeo& g, const NodeGeo& G, int k) {
    const int k1 = (k == 2) ? 0 : k + 1;
    double C = G.c[k];
    if (fabs(C) < 1.0e-06) return false;
    double v1x = G.tri[k][0], v1y = G.tri[k][1], v2x = G.tri[k1][0], v2y = G.tri[k1][1];
    if (C < 0) { double tx = v1x, ty = v1y; v1x = v2x; v1y = v2y; v2x = tx; v2y = ty; }
    child_geo(g, v1x, v1y, v2x, v2y, sgn(C));
    return true;
}

EBEM_DI bool node_child_e(ChildE& g, const NodeGeo& G, int k) {
    const int k1 = (k == 2) ? 0 : k + 1;
    double C = G.c[k];
    if (fabs(C) < 1.0e-06) return false;
    double v1x = G.tri[k][0], v1y = G.tri[k][1], v2x = G.tri[k1][0], v2y = G.tri[k1][1];
    if (C < 0) { double tx = v1x, ty = v1y; v1x = v2x; v1y = v2y; v2x = tx; v2y = ty; }
    child_geo_e(g, v1x, v1y, v2x, v2y, sgn(C));
    return true;
}

// rho_P / rho_S and the case split (BEMenerg_coreSA_calcMatrixSubBlock.m:58-81)
EBEM_DI int classify(double zeta, double rP, double rS, double dMIN, double& rhoP, double& rhoS) {
    if (zeta == 0) { rhoP = rP; rhoS = rS; }
    else if (zeta < rS) { rhoP = sqrt(rP * rP - zeta * zeta); rhoS = sqrt(rS * rS - zeta * zeta); }
    else if (rS < zeta && zeta < rP) { rhoP = sqrt(rP * rP - zeta * zeta); rhoS = -1.0; }
    else { rhoP = -1.0; rhoS = -1.0; }
    if (dMIN < rhoS) return T_SP_SP;
    if (0 < rhoS && rhoS <= dMIN && dMIN < rhoP) return T_SP_P;
    if (rhoS <= 0 && dMIN < rhoP) return T_P;
    return T_NONE;
}

// Null test of BEMenerg_coreSA_calcMatrixBlock.m:57-61.
EBEM_DI bool lag_nonnull(int l, double velP, double velS, double dt, double distMin, double distMax) {
    return ((l - 1) * velS * dt < distMax) && ((l + 1) * velP * dt >= distMin);
}

// The non-null lags of the pair (source S, field F) within [lag0, lag0 + nlag):
// the null test is monotone in the lag, so they form one band [*llo, *lhi]
// (*llo = -1 when empty).
EBEM_DI void pair_band(const TriGeom& F, const TriGeom& S, double velP, double velS, double dt, int lag0, int nlag,
                       int* llo, int* lhi) {
    const double v0 = F.ctr[0] - S.ctr[0], v1 = F.ctr[1] - S.ctr[1], v2 = F.ctr[2] - S.ctr[2];
    const double d = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    const double distMin = d - F.maxL - S.maxL;
    const double distMax = d + F.maxL + S.maxL;
    *llo = -1;
    *lhi = -2;
    for (int q = 0; q < nlag; q++) {
        const int l = lag0 + q;
        if (lag_nonnull(l, velP, velS, dt, distMin, distMax)) {
            if (*llo < 0) *llo = l;
            *lhi = l;
        }
    }
}

// F(t_k) for one pair: sum over the outer nodes of the source triangle of the
// weighted closed-form inner integrals, combined (calcMatrixSubBlock.m:101-104)
// and rotated back to global axes; 6 symmetric entries (11,12,13,22,23,33).
EBEM_DI void level_value(double Fk[6], int k, double velP, double velS, double dt, const TriGeom& F,
                         const NodeW* __restrict__ nodes, int n_gh) {
    const double t = k * dt;
    LevelCtx L;
    L.t2 = t * t;
    L.RP = velP * t;
    L.RS = velS * t;
    double vp2 = velP * velP, vs2 = velS * velS, den = (velP * velS) * (velP * velS);
    L.k1 = 1.0 / vp2;
    L.k5 = (vp2 + vs2) / den;
    L.k6 = (vp2 - vs2) / den;
    double S = 0.0, T[6] = {0, 0, 0, 0, 0, 0};
    for (int g = 0; g < n_gh; g++) {
        NodeW sp = nodes[g];
        NodeGeo G;
        node_geo(G, sp, F);
        double rhoP, rhoS;
        int type = classify(G.zeta, L.RP, L.RS, G.dMIN, rhoP, rhoS);
        if (type == T_NONE) continue;
        double s = 0.0, tt[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 1
        for (int c = 0; c < 3; c++) {
#if EBEM_SA_FORM == 1
            ChildE cg;
            if (!node_child_e(cg, G, c)) continue;
            child_level_e(s, tt, cg, L, G.zeta, G.sigma, rhoP, rhoS, type);
#else
            ChildGeo cg;
            if (!node_child(cg, G, c)) continue;
            child_level(s, tt, cg, L, G.zeta, G.sigma, rhoP, rhoS, type);
#endif
        }
        S += sp.w * s;
#pragma unroll
        for (int e = 0; e < 6; e++) T[e] += sp.w * tt[e];
    }
    // local tensor (child-frame order 11,12,22,13,23,33) -> full symmetric
    double M[3][3] = {{T[0], T[1], T[3]}, {T[1], T[2], T[4]}, {T[3], T[4], T[5]}};
    const double* C = F.C;
    // R = C^T M C
    double MC[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) MC[r][c] = M[r][0] * C[c] + M[r][1] * C[3 + c] + M[r][2] * C[6 + c];
    double R[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = r; c < 3; c++) R[r][c] = C[r] * MC[0][c] + C[3 + r] * MC[1][c] + C[6 + r] * MC[2][c];
    Fk[0] = 0.5 * (S + R[0][0]);
    Fk[1] = 0.5 * R[0][1];
    Fk[2] = 0.5 * R[0][2];
    Fk[3] = 0.5 * (S + R[1][1]);
    Fk[4] = 0.5 * R[1][2];
    Fk[5] = 0.5 * (S + R[2][2]);
}


}  // namespace ebem
