// Closed-form inner integrals of the semi-analytic (SA) energetic BEM
// assembly, device side, FP64.
//
// The mathematics is that of the reference's MATLAB SA path (paths relative to
// the reference project root, "SA/" = functions/BEMenerg_indir/BEMenerg_core/
// BEMenerg_coreSA/calcoloMatrice/, "AI/" = functions/BEMenerg_analiticIntg/):
// the field triangle seen from the projection O of an outer node is split into
// three children (O, P_k, P_k+1); each child is cut by the P- and S-front
// circles into up to nine regions (SA/BEMenerg_coreSA_calcIntgInt_childTriangle.m),
// each integrated in closed form (AI/BEMenerg_analiticIntg_{CC,SC_P,SC_SP,TC,
// TR_P,TR_SP}.m with the G coefficients of AI/coefficientiG/*.m).
//
// Representation chosen for the GPU (not the reference's): every region
// integral is a scalar multiple of the identity plus a combination
// sum_m beta_m B_m of the six child matrices B_1..B_6 of
// AI/coefficientiB/BEMenerg_coreSA_coeffB.m.  Because the final kernel
// combination (SA/BEMenerg_coreSA_calcMatrixSubBlock.m:101-104) and all the
// rotations are linear, a child carries just 7 scalars (S, beta_1..beta_6)
// with the combination weights already applied; the 3x3 tensor is formed once
// per child, rotated back by theta0, and the field-triangle Euler rotation
// (SA/operazioniGeometriche/rotazioneInversaEulero.m) is applied once per
// (pair, time level) instead of three times per (pair, node, instant).
#pragma once

#include <math.h>

#ifndef EBEM_NOINLINE_MATH
#define EBEM_NOINLINE_MATH 1
#endif
#ifndef EBEM_NOINLINE_REGIONS
#define EBEM_NOINLINE_REGIONS 0
#endif
#ifndef EBEM_UNIFORM_SLOTS
#define EBEM_UNIFORM_SLOTS 1
#endif

#ifdef __CUDACC__
#include <cuda_runtime.h>
#define EBEM_DI __device__ __forceinline__
#define EBEM_HDI __host__ __device__ inline
// One out-of-line copy of each transcendental and of each region routine
// keeps the kernel's instruction footprint inside the instruction caches
// (fully inlined, the kernel stalls on instruction fetch).
#if EBEM_NOINLINE_MATH
#define EBEM_MFN static __device__ __noinline__
#else
#define EBEM_MFN __device__ __forceinline__
#endif
#if EBEM_NOINLINE_REGIONS
#define EBEM_RFN static __device__ __noinline__
#else
#define EBEM_RFN __device__ __forceinline__
#endif
#else
// host compilation of the same device algebra (used to emulate the kernels'
// arithmetic on the CPU when investigating a numerical difference)
#define EBEM_DI inline
#define EBEM_HDI inline
#define EBEM_MFN inline
#define EBEM_RFN inline
#endif

namespace ebem {

constexpr double kPi = 3.141592653589793238462643383279502884;

EBEM_MFN double m_sin(double x) { return sin(x); }
EBEM_MFN double m_cos(double x) { return cos(x); }
EBEM_MFN void m_sincos(double x, double* s, double* c) { sincos(x, s, c); }
EBEM_MFN double m_log(double x) { return log(x); }
EBEM_MFN double m_exp(double x) { return exp(x); }
EBEM_MFN double m_acos(double x) { return acos(x); }
EBEM_MFN double m_asin(double x) { return asin(x); }
EBEM_MFN double m_atan2(double y, double x) { return atan2(y, x); }

enum : int { T_NONE = 0, T_SP_SP = 1, T_SP_P = 2, T_P = 3 };

EBEM_HDI double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
EBEM_DI double acos_c(double x) { return m_acos(fmin(1.0, fmax(-1.0, x))); }
EBEM_DI double asin_c(double x) { return m_asin(fmin(1.0, fmax(-1.0, x))); }
EBEM_DI double sqrt_c(double x) { return x > 0.0 ? sqrt(x) : 0.0; }

// Per field triangle data produced by the preparation kernel.
struct TriGeom {
    double P1[3];          // first vertex
    double e1[3], e2[3];   // in-plane frame (calcoloSistemaRiferimento.m)
    double n[3];           // unit normal (readSpaceMesh.m:114-122)
    double L1, L3, cd, sd; // |P2-P1|, |P3-P1|, cos/sin of the angle at P1
    double C[9];           // Euler matrix, row-major (rotazioneInversaEulero.m:160-176)
    double ctr[3];         // centroid
    double maxL;           // longest edge
    double area;
    double pad;
};

// Time-level constants shared by every node and child.
struct LevelCtx {
    double t2;                  // t^2
    double RP, RS;              // c_P t, c_S t
    double k1, k5, k6;          // 1/c_P^2, (c_P^2+c_S^2)/(c_P c_S)^2, (c_P^2-c_S^2)/(c_P c_S)^2
};

// Child triangle data that does not depend on the time level
// (SA/operazioniGeometriche/calcoloDatiTriangolo.m and the theta0 rotation of
// SA/BEMenerg_coreSA_calcIntgInt_fieldTriangle.m:37-59).
struct ChildGeo {
    double a, bm, F;                 // |V1|, a*vt_x, a*m_sin(beta)
    double alpha, beta, gamma;
    double ca, cb, cg, sa, sb, sg;   // cos/sin of alpha, beta, gamma
    double ct, st;                   // cos/sin of the back-rotation angle theta0
    double sgnC;                     // sign of the child's signed area; 0 = skipped
};

struct Acc7 { double S, b[6]; };

EBEM_DI void acc_zero(Acc7& A) {
    A.S = 0.0;
#pragma unroll
    for (int m = 0; m < 6; m++) A.b[m] = 0.0;
}

// Phi(1..5) of the region integrals (identical in AI/BEMenerg_analiticIntg_CC.m:79-83,
// _SC_P.m:31-35, _SC_SP.m:85-89, coefficientiG/*_TC.m:35-39).
struct Phi { double p1, p2, p3, p4, p5; };

EBEM_DI Phi phi_all(double T1t, double T2t, double gamma, double cos_gamma) {
    Phi P;
    double sh = m_sin(T1t / 2);
    P.p1 = 2 * m_sin(T2t / 2) * sh;
    P.p2 = 2 * m_sin(gamma - (T2t / 2)) * sh;
    double s1 = m_sin(T1t);
    P.p3 = 0.5 * (T1t - (m_cos(T2t) * s1));
    P.p4 = -0.5 * (-(s1 * m_cos(gamma - T2t)) + (T1t * cos_gamma));
    P.p5 = 0.5 * (T1t - (m_cos(2 * gamma - T2t) * s1));
    return P;
}

// Regions whose radial integrals separate (annulus "CC" and P-disc sector
// "SC_P"): ris1 = T1t I1, ris2 = I2 B_1 + I3 B_2 + T1t I4 B_3, ris3 = T1t I4,
// ris4 = I5 B_1 + I6 B_2 + T1t I7 B_3 with B_1 = Phi5 B4 + Phi4 B5 + Phi3 B6,
// B_2 = Phi2 B2 + Phi1 B3, B_3 = B1 (AI/BEMenerg_analiticIntg_CC.m:85-102).
EBEM_DI void add_sep_P(Acc7& A, const LevelCtx& L, double T1t, const Phi& P, bool full,
                                          double I1, double I2, double I3, double I4, double I5, double I6, double I7) {
    A.S += L.k1 * (T1t * I1) - L.t2 * (T1t * I4);
    double X = -L.k1 * I2 + 3 * L.t2 * I5;
    A.b[3] += X * P.p5; A.b[4] += X * P.p4; A.b[5] += X * P.p3;
    if (full) {
        double Y = -L.k1 * I3 + 3 * L.t2 * I6;
        double Z = T1t * (-L.k1 * I4 + 3 * L.t2 * I7);
        A.b[0] += Z; A.b[1] += Y * P.p2; A.b[2] += Y * P.p1;
    }
}

// AI/BEMenerg_analiticIntg_CC.m:1-93 — annulus between the S and P fronts.
EBEM_RFN void reg_CC(Acc7& A, const LevelCtx& L, const ChildGeo& g, double zeta,
                                       double rhoS, double rhoP, double TH1, double TH2) {
    const double RS = L.RS, RP = L.RP;
    double T1t = TH2 - TH1, T2t = TH2 + TH1;
    Phi P = phi_all(T1t, T2t, g.gamma, g.cg);
    if (zeta > 1.0e-6) {
        double I1 = RP - RS;
        double I2 = RP - RS + (zeta * zeta * (1 / RP - 1 / RS));
        double I3 = m_log((rhoP + RP) / (rhoS + RS)) - (rhoP / RP) + (rhoS / RS);
        double I4 = -(1 / RP) + (1 / RS);
        double iRP3 = 1 / (RP * RP * RP), iRS3 = 1 / (RS * RS * RS);
        double I5 = I4 + (zeta * zeta / 3) * (iRP3 - iRS3);
        double q1 = rhoP / RP, q2 = rhoS / RS;
        double I6 = (1 / (3 * zeta * zeta)) * (q1 * q1 * q1 - q2 * q2 * q2);
        double I7 = (-1.0 / 3) * (iRP3 - iRS3);
        add_sep_P(A, L, T1t, P, true, I1, I2, I3, I4, I5, I6, I7);
    } else {
        double I1 = RP - RS;
        double I4 = -(1 / RP) + (1 / RS);
        add_sep_P(A, L, T1t, P, false, I1, I1, 0.0, I4, I4, 0.0, 0.0);
    }
}

// AI/BEMenerg_analiticIntg_SC_P.m:1-54 — sector of the P disc (zeta > 0 always
// reaches here: the P-only case needs the S sphere to miss the plane).
EBEM_RFN void reg_SC_P(Acc7& A, const LevelCtx& L, const ChildGeo& g, double zeta,
                                         double rhoP, double TH1, double TH2) {
    const double RP = L.RP;
    double T1t = TH2 - TH1, T2t = TH2 + TH1;
    Phi P = phi_all(T1t, T2t, g.gamma, g.cg);
    double I1 = RP - zeta;
    double I2 = RP + (zeta * zeta / RP) - (2 * zeta);
    double I3 = m_log((rhoP + RP) / zeta) - (rhoP / RP);
    double I4 = -(1 / RP) + (1 / zeta);
    double I5 = -(1 / RP) + (zeta * zeta / (3 * RP * RP * RP)) + (2 / (3 * zeta));
    double q1 = rhoP / RP;
    double I6 = (1 / (3 * zeta * zeta)) * (q1 * q1 * q1);
    double I7 = -(1 / (3 * RP * RP * RP)) + (1 / (3 * zeta * zeta * zeta));
    add_sep_P(A, L, T1t, P, true, I1, I2, I3, I4, I5, I6, I7);
}

// AI/BEMenerg_analiticIntg_SC_SP.m:1-75 — sector of the S disc (P&S terms).
EBEM_RFN void reg_SC_SP(Acc7& A, const LevelCtx& L, const ChildGeo& g, double zeta,
                                          double rhoS, double TH1, double TH2) {
    const double RS = L.RS;
    double T1t = TH2 - TH1, T2t = TH2 + TH1;
    Phi P = phi_all(T1t, T2t, g.gamma, g.cg);
    if (zeta > 1.0e-6) {
        double I1 = RS - zeta;
        double I2 = RS + (zeta * zeta / RS) - (2 * zeta);
        double I3 = m_log((rhoS + RS) / zeta) - (rhoS / RS);
        double I4 = -(1 / RS) + (1 / zeta);
        A.S += L.k5 * (T1t * I1);
        double X = L.k6 * I2, Y = L.k6 * I3;
        A.b[0] += L.k6 * (T1t * I4);
        A.b[1] += Y * P.p2; A.b[2] += Y * P.p1;
        A.b[3] += X * P.p5; A.b[4] += X * P.p4; A.b[5] += X * P.p3;
    } else {
        A.S += L.k5 * (T1t * RS);
        double X = L.k6 * RS;
        A.b[3] += X * P.p5; A.b[4] += X * P.p4; A.b[5] += X * P.p3;
    }
}

// G coefficients of the "triangle minus circle" region,
// AI/coefficientiG/BEMenerg_analiticIntg_coeffG_TC.m:1-182.  G[k] = G(k).
EBEM_RFN void coeffG_TC(double G[20], double zeta, double RS, double rhoS,
                                          double TH1, double TH2, const ChildGeo& g) {
    const double sin_beta = g.sb, sin_alpha = g.sa;
    const double cos_alpha = g.ca, cos_beta = g.cb, cos_gamma = g.cg;
    const double alpha = g.alpha, beta = g.beta, gamma = g.gamma;
    double T1t = TH2 - TH1, T2t = TH2 + TH1;
    const double F = g.F;
    Phi P = phi_all(T1t, T2t, gamma, cos_gamma);
    double s1b, c1b, s2b, c2b;
    m_sincos(TH1 + beta, &s1b, &c1b);
    m_sincos(TH2 + beta, &s2b, &c2b);
    if (zeta > 1.0e-6) {
        double R1 = F / s1b, R2 = F / s2b;
        double FR1 = zeta / R1, FR2 = zeta / R2;
        double ADD = zeta * zeta + F * F;
        double g1 = sqrt(1 + FR1 * FR1);
        double g2 = sqrt(1 + FR2 * FR2);
        double g3 = 0.5 * (m_log((g1 + c1b) * (g2 - c2b)) - m_log((g1 - c1b) * (g2 + c2b)));
        double iF1 = 1 / FR1, iF2 = 1 / FR2;
        double g4 = m_log(iF1 + sqrt(1 + iF1 * iF1));
        double g5 = m_log(iF2 + sqrt(1 + iF2 * iF2));
        double sq = sqrt(ADD);
        double g7 = kPi - acos_c((-zeta * c2b) / sq) - acos_c((zeta * c1b) / sq);
        double g8 = F * F / ADD;
        double Lg = (rhoS / RS) - m_log((rhoS + RS) / zeta);
        double cgm1 = m_cos(gamma - TH1), cgm2 = m_cos(gamma - TH2);
        double cth1 = m_cos(TH1), cth2 = m_cos(TH2);
        double cag1 = m_cos(alpha - gamma + TH1), cag2 = m_cos(alpha - gamma + TH2);
        double cta1 = m_cos(TH1 + alpha), cta2 = m_cos(TH2 + alpha);
        double ctb1 = m_cos(TH1 - beta), ctb2 = m_cos(TH2 - beta);
        G[1] = -(RS * T1t) + (zeta * g7) + (F * g3);
        G[4] = (1 / RS * T1t) - (1 / zeta * g7);
        G[5] = cgm2 * g5 - cgm1 * g4 - cos_alpha * g3 + Lg * (cgm2 - cgm1);
        G[6] = -cth2 * g5 + cth1 * g4 - cos_beta * g3 - Lg * (cth2 - cth1);
        double Q = (RS * RS + zeta * zeta) / RS;
        G[7] = zeta * g7 - Q * P.p5 + F * (-g1 * cag1 + g2 * cag2 + g3 * (sin_alpha * sin_alpha));
        G[8] = -zeta * cos_gamma * g7 - Q * P.p4 + F * (-sin_alpha * sin_beta * g3 + g1 * cta1 - g2 * cta2);
        G[9] = zeta * g7 - Q * P.p3 + F * ((sin_beta * sin_beta) * g3 + g1 * ctb1 - g2 * ctb2);
        double iz2 = 1 / (3 * zeta * zeta);
        G[14] = 1 / (3 * RS * RS * RS) * T1t + iz2 * (F / ADD * (c1b / g1 - c2b / g2) - 1 / zeta * g7);
        double rs3 = rhoS * rhoS * rhoS;
        double pre = -rs3 / (3 * zeta * zeta * RS * RS * RS);
        G[15] = pre * P.p2 + iz2 * ((sin_alpha * s2b - g8 * cos_alpha * c2b) / g2
                                    + (-sin_alpha * s1b + g8 * cos_alpha * c1b) / g1);
        G[16] = pre * P.p1 + iz2 * ((sin_beta * s1b + g8 * cos_beta * c1b) / g1
                                    + (-sin_beta * s2b - g8 * cos_beta * c2b) / g2);
        double K = ((1 / RS) - (zeta * zeta / (3 * RS * RS * RS)));
        double s1b2 = s1b * s1b, s2b2 = s2b * s2b;
        G[17] = 1.0 / 3 * (-s2b2 * cag2 + g8 * (cos_alpha * cos_alpha) * c2b) / (F * g2)
              - 1.0 / 3 * (-s1b2 * cag1 + g8 * (cos_alpha * cos_alpha) * c1b) / (F * g1)
              - g7 / (3 * zeta) + K * P.p5;
        G[18] = 1.0 / 3 * (s2b2 * cta2 + g8 * (cos_alpha * cos_beta * c2b)) / (F * g2)
              - 1.0 / 3 * (s1b2 * cta1 + g8 * (cos_alpha * cos_beta * c1b)) / (F * g1)
              + g7 / (3 * zeta) * cos_gamma + K * P.p4;
        G[19] = 1.0 / 3 * (s2b2 * ctb2 + g8 * ((cos_beta * cos_beta) * c2b)) / (F * g2)
              - 1.0 / 3 * (s1b2 * ctb1 + g8 * ((cos_beta * cos_beta) * c1b)) / (F * g1)
              - g7 / (3 * zeta) + K * P.p3;
    } else {
        double g_3 = 0.5 * (m_log((1 + c1b) * (1 - c2b)) - m_log((1 - c1b) * (1 + c2b)));
        double cag1 = m_cos(alpha - gamma + TH1), cag2 = m_cos(alpha - gamma + TH2);
        double cta1 = m_cos(TH1 + alpha), cta2 = m_cos(TH2 + alpha);
        double ctb1 = m_cos(TH1 - beta), ctb2 = m_cos(TH2 - beta);
        double s1b2 = s1b * s1b, s2b2 = s2b * s2b;
        G[1] = (F * g_3) - (RS * T1t);
        G[4] = 1 / F * (c2b - c1b) + 1 / RS * T1t;
        G[7] = -RS * P.p5 + F * (cag2 - cag1 + (sin_alpha * sin_alpha) * g_3);
        G[8] = -RS * P.p4 + F * (cta1 - cta2 - sin_alpha * sin_beta * g_3);
        G[9] = -RS * P.p3 + F * (ctb1 - ctb2 + (sin_beta * sin_beta) * g_3);
        double cab = (cos_alpha * cos_beta) + m_cos(alpha + beta);
        G[17] = 1 / (3 * F) * (((1 + cos_alpha * cos_alpha) * c2b - s2b2 * cag2)
                               - ((1 + cos_alpha * cos_alpha) * c1b - s1b2 * cag1)) + 1 / RS * P.p5;
        G[18] = 1 / (3 * F) * ((c2b * cab + s2b2 * cta2) - (c1b * cab + s1b2 * cta1)) + 1 / RS * P.p4;
        G[19] = 1 / (3 * F) * (((1 + cos_beta * cos_beta) * c2b + s2b2 * ctb2)
                               - ((1 + cos_beta * cos_beta) * c1b + s1b2 * ctb1)) + 1 / RS * P.p3;
        G[5] = G[6] = G[14] = G[15] = G[16] = 0.0;
    }
}

// AI/coefficientiG/BEMenerg_analiticIntg_coeffG_TR_P.m:1-120 and
// _TR_SP.m:1-111 (the TR_SP set is G(1), G(4..9) of the same expressions;
// with_p4 selects whether G(14..19) are needed).
EBEM_RFN void coeffG_TR(double G[20], double zeta, double TH1, double TH2,
                                          const ChildGeo& g, bool with_r4) {
    const double sin_beta = g.sb, sin_alpha = g.sa;
    const double cos_alpha = g.ca, cos_beta = g.cb, cos_gamma = g.cg;
    const double alpha = g.alpha, beta = g.beta, gamma = g.gamma;
    double T1t = TH2 - TH1, T2t = TH2 + TH1;
    const double F = g.F;
    double s1b, c1b, s2b, c2b;
    m_sincos(TH1 + beta, &s1b, &c1b);
    m_sincos(TH2 + beta, &s2b, &c2b);
    double cag1 = m_cos(alpha - gamma + TH1), cag2 = m_cos(alpha - gamma + TH2);
    double cta1 = m_cos(TH1 + alpha), cta2 = m_cos(TH2 + alpha);
    double ctb1 = m_cos(TH1 - beta), ctb2 = m_cos(TH2 - beta);
    if (with_r4 || zeta > 1.0e-6) {   // TR_P has no coplanar branch
        double p3 = 0.5 * (T1t - (m_cos(T2t) * m_sin(T1t)));
        double p4 = -0.5 * (-(m_sin(T1t) * m_cos(gamma - T2t)) + (T1t * cos_gamma));
        double p5 = 0.5 * (T1t - (m_cos(2 * gamma - T2t) * m_sin(T1t)));
        double R1 = F / s1b, R2 = F / s2b;
        double FR1 = zeta / R1, FR2 = zeta / R2;
        double ADD = zeta * zeta + F * F;
        double g1 = sqrt(1 + FR1 * FR1);
        double g2 = sqrt(1 + FR2 * FR2);
        double g3 = 0.5 * (m_log((g1 + c1b) * (g2 - c2b)) - m_log((g1 - c1b) * (g2 + c2b)));
        double iF1 = 1 / FR1, iF2 = 1 / FR2;
        double g4 = m_log(iF1 + sqrt(1 + iF1 * iF1));
        double g5 = m_log(iF2 + sqrt(1 + iF2 * iF2));
        double sq = sqrt(ADD);
        double g7 = kPi - acos_c((-zeta * c2b) / sq) - acos_c((zeta * c1b) / sq);
        G[1] = (zeta * (-T1t + g7)) + (F * g3);
        G[4] = 1 / zeta * (T1t - g7);
        G[5] = m_cos(gamma - TH2) * g5 - m_cos(gamma - TH1) * g4 - cos_alpha * g3;
        G[6] = -m_cos(TH2) * g5 + m_cos(TH1) * g4 - cos_beta * g3;
        G[7] = zeta * (g7 - 2 * p5) + F * (-g1 * cag1 + g2 * cag2 + g3 * (sin_alpha * sin_alpha));
        G[8] = -zeta * ((cos_gamma * g7) + 2 * p4) + F * (-sin_alpha * sin_beta * g3 + g1 * cta1 - g2 * cta2);
        G[9] = zeta * (g7 - 2 * p3) + F * ((sin_beta * sin_beta) * g3 + g1 * ctb1 - g2 * ctb2);
        if (with_r4) {
            double g8 = F * F / ADD;
            double iz2 = 1 / (3 * zeta * zeta);
            double s1b2 = s1b * s1b, s2b2 = s2b * s2b;
            G[14] = iz2 * (1 / zeta * (T1t - g7) + (F / ADD * (c1b / g1 - c2b / g2)));
            G[15] = iz2 * ((sin_alpha * s2b - g8 * cos_alpha * c2b) / g2 + (-sin_alpha * s1b + g8 * cos_alpha * c1b) / g1);
            G[16] = iz2 * ((sin_beta * s1b + g8 * cos_beta * c1b) / g1 + (-sin_beta * s2b - g8 * cos_beta * c2b) / g2);
            G[17] = (1 / (3 * F) * ((-s2b2 * cag2 + g8 * (cos_alpha * cos_alpha) * c2b) / g2
                                    - (-s1b2 * cag1 + g8 * (cos_alpha * cos_alpha) * c1b) / g1))
                  - (1 / (3 * zeta) * (g7 - 2 * p5));
            G[18] = (1 / (3 * F) * ((s2b2 * cta2 + g8 * (cos_alpha * cos_beta * c2b)) / g2
                                    - (s1b2 * cta1 + g8 * (cos_alpha * cos_beta * c1b)) / g1))
                  + (1 / (3 * zeta) * ((g7 * cos_gamma) + 2 * p4));
            G[19] = (1 / (3 * F) * ((s2b2 * ctb2 + g8 * ((cos_beta * cos_beta) * c2b)) / g2
                                    - (s1b2 * ctb1 + g8 * ((cos_beta * cos_beta) * c1b)) / g1))
                  - (1 / (3 * zeta) * (g7 - 2 * p3));
        }
    } else {
        // coplanar branch of _TR_SP.m:210-229 (TR_P never sees zeta = 0)
        double g_3 = 0.5 * (m_log((1 + c1b) * (1 - c2b)) - m_log((1 - c1b) * (1 + c2b)));
        G[1] = F * g_3;
        G[4] = G[5] = G[6] = 0.0;
        G[7] = F * (-cag1 + cag2 + (sin_alpha * sin_alpha) * g_3);
        G[8] = F * (-(sin_alpha * sin_beta * g_3) + cta1 - cta2);
        G[9] = F * ((sin_beta * sin_beta) * g_3 + ctb1 - ctb2);
    }
}

// AI/BEMenerg_analiticIntg_TC.m:1-50 — triangle minus the S disc (P terms).
EBEM_RFN void reg_TC(Acc7& A, const LevelCtx& L, const ChildGeo& g, double zeta,
                                       double rhoS, double TH1, double TH2) {
    double G[20];
    bool full = zeta > 1.0e-6;
    coeffG_TC(G, full ? zeta : 0.0, L.RS, rhoS, TH1, TH2, g);
    A.S += L.k1 * G[1] - L.t2 * G[4];
    if (full) {
#pragma unroll
        for (int m = 0; m < 3; m++) A.b[m] += -L.k1 * G[4 + m] + 3 * L.t2 * G[14 + m];
    }
#pragma unroll
    for (int m = 3; m < 6; m++) A.b[m] += -L.k1 * G[4 + m] + 3 * L.t2 * G[14 + m];
}

// AI/BEMenerg_analiticIntg_TR_P.m:1-28 — plain triangle piece inside the P
// disc (P terms; zeta > 0 here).
EBEM_RFN void reg_TR_P(Acc7& A, const LevelCtx& L, const ChildGeo& g, double zeta,
                                         double TH1, double TH2) {
    double G[20];
    coeffG_TR(G, zeta, TH1, TH2, g, true);
    A.S += L.k1 * G[1] - L.t2 * G[4];
#pragma unroll
    for (int m = 0; m < 6; m++) A.b[m] += -L.k1 * G[4 + m] + 3 * L.t2 * G[14 + m];
}

// AI/BEMenerg_analiticIntg_TR_SP.m:1-40 — plain triangle piece inside the S
// disc (P&S terms).
EBEM_RFN void reg_TR_SP(Acc7& A, const LevelCtx& L, const ChildGeo& g, double zeta,
                                          double TH1, double TH2) {
    double G[20];
    bool full = zeta > 1.0e-6;
    coeffG_TR(G, full ? zeta : 0.0, TH1, TH2, g, false);
    A.S += L.k5 * G[1];
    if (full) {
#pragma unroll
        for (int m = 0; m < 3; m++) A.b[m] += L.k6 * G[4 + m];
    }
#pragma unroll
    for (int m = 3; m < 6; m++) A.b[m] += L.k6 * G[4 + m];
}

// One child triangle at one time level: the region decomposition of
// SA/BEMenerg_coreSA_calcIntgInt_childTriangle.m:27-234.  Accumulates into
// `out` the child's scalar part and its tensor part rotated back by theta0
// and signed (fieldTriangle.m:57-84); tensor entries in T[0..5] =
// (11, 12, 22, 13, 23, 33).
EBEM_DI void child_level(double& Sout, double T[6], const ChildGeo& g, const LevelCtx& L,
                                            double zeta, double sigma, double rhoP, double rhoS, int type) {
    const double a = g.a;
    double DeltaP = g.bm * g.bm - (a * a - rhoP * rhoP);
    double DeltaS = g.bm * g.bm - (a * a - rhoS * rhoS);
    double rP = g.F / rhoP;
    double rS = g.F / rhoS;
    if (type == T_P) { rS = 0.0; DeltaS = 0.0; }
    const double beta = g.beta, gamma = g.gamma;
    double TH1, TH2, TH3, TH4, TH5, TH6;
    if (DeltaP <= 1.0e-06) {
        TH1 = 0.0; TH2 = TH3 = TH4 = TH5 = TH6 = gamma;
    } else if (DeltaS <= 1.0e-06) {
        double as = asin_c(rP);
        double O1 = as - beta, O2 = kPi - as - beta;
        double t1 = fmin(O1, O2), t2 = fmax(O1, O2);
        TH1 = 0.0;
        TH2 = fmin(fmax(0.0, t1), gamma);
        TH3 = TH4 = TH5 = fmax(0.0, fmin(t2, gamma));
        TH6 = gamma;
    } else {
        double asP = asin_c(rP), asS = asin_c(rS);
        double O1 = asP - beta, O2 = kPi - asP - beta;
        double O3 = asS - beta, O4 = kPi - asS - beta;
        double t1 = fmin(O1, O2), t2 = fmax(O1, O2);
        double t3 = fmin(O3, O4), t4 = fmax(O3, O4);
        TH1 = 0.0;
        TH2 = fmin(fmax(0.0, t1), gamma);
        TH3 = fmin(fmax(0.0, t3), gamma);
        TH4 = fmax(0.0, fmin(t4, gamma));
        TH5 = fmax(0.0, fmin(t2, gamma));
        TH6 = gamma;
    }
    Acc7 A;
    acc_zero(A);
    const bool spsp = (type == T_SP_SP);
    if (TH1 < TH2) {
        if (spsp) reg_SC_SP(A, L, g, zeta, rhoS, TH1, TH2);
        if (type == T_P) reg_SC_P(A, L, g, zeta, rhoP, TH1, TH2);
        else reg_CC(A, L, g, zeta, rhoS, rhoP, TH1, TH2);
    }
    if (TH2 < TH3) {
        if (spsp) reg_SC_SP(A, L, g, zeta, rhoS, TH2, TH3);
        if (type == T_P) reg_TR_P(A, L, g, zeta, TH2, TH5);
        else reg_TC(A, L, g, zeta, rhoS, TH2, TH3);
    }
    if (TH3 < TH4) {
        if (spsp) reg_TR_SP(A, L, g, zeta, TH3, TH4);
    }
    if (TH4 < TH5) {
        if (spsp) reg_SC_SP(A, L, g, zeta, rhoS, TH4, TH5);
        reg_TC(A, L, g, zeta, rhoS, TH4, TH5);
    }
    if (TH5 < TH6) {
        if (spsp) reg_SC_SP(A, L, g, zeta, rhoS, TH5, TH6);
        if (type == T_P) reg_SC_P(A, L, g, zeta, rhoP, TH5, TH6);
        else reg_CC(A, L, g, zeta, rhoS, rhoP, TH5, TH6);
    }
    // tensor sum_m beta_m B_m in the child frame (coeffB.m:20-43 with
    // A1 = (1,0,0), A2 = (cos g, sin g, 0), A3 = (0, 0, -sigma))
    const double sg = g.sg, cg = g.cg;
    const double* b = A.b;
    double isg = 1.0 / sg;
    double t11 = (b[3] + 2 * cg * b[4] + cg * cg * b[5]) * (isg * isg);
    double t12 = (b[4] + cg * b[5]) * isg;
    double t22 = b[5];
    double zs = zeta * sigma;
    double t13 = -zs * (b[1] + cg * b[2]) * isg;
    double t23 = -zs * b[2];
    double t33 = zs * zs * b[0];
    // back-rotation A T A^T, A = [c s 0; -s c 0; 0 0 1]
    const double c = g.ct, s = g.st;
    double cc = c * c, ss = s * s, cs = c * s;
    double w = g.sgnC;
    Sout += w * A.S;
    T[0] += w * (cc * t11 + 2 * cs * t12 + ss * t22);
    T[1] += w * (-cs * t11 + (cc - ss) * t12 + cs * t22);
    T[2] += w * (ss * t11 - 2 * cs * t12 + cc * t22);
    T[3] += w * (c * t13 + s * t23);
    T[4] += w * (-s * t13 + c * t23);
    T[5] += w * t33;
}

// The child data of calcoloDatiTriangolo.m:1-39 for a child (O, V1, V2)
// already oriented counter-clockwise, plus the theta0 back-rotation of
// fieldTriangle.m:37-59.  The reference obtains the angles from the law of
// cosines and acos, which loses about half the digits on thin children (an
// angle of 1e-3 comes out with a relative error near 1e-10 and the region
// formulas amplify it through their 1/F terms).  The same angles are computed
// here from the cross and dot products of the edge vectors with atan2, and
// F = a m_sin(beta) = 2 area / |V2 - V1| directly: identical quantities, full
// precision.
EBEM_DI void child_geo(ChildGeo& g, double v1x, double v1y, double v2x, double v2y, double sgnC) {
    double a = sqrt(v1x * v1x + v1y * v1y);
    double b = sqrt(v2x * v2x + v2y * v2y);
    double dx = v2x - v1x, dy = v2y - v1y;
    double c = sqrt(dx * dx + dy * dy);
    double cr = v1x * v2y - v1y * v2x;            // twice the child's area (> 0)
    double dg = v1x * v2x + v1y * v2y;            // V1 . V2          (angle at O)
    double db = -(v1x * dx + v1y * dy);           // (-V1) . (V2-V1)  (angle at V1)
    double da = v2x * dx + v2y * dy;              // (-V2) . (V1-V2)  (angle at V2)
    g.a = a;
    g.gamma = m_atan2(cr, dg);
    g.beta = m_atan2(cr, db);
    g.alpha = m_atan2(cr, da);
    double iab = 1.0 / (a * b), iac = 1.0 / (a * c), ibc = 1.0 / (b * c);
    g.cg = dg * iab; g.sg = cr * iab;
    g.cb = db * iac; g.sb = cr * iac;
    g.ca = da * ibc; g.sa = cr * ibc;
    g.F = cr / c;
    // Bmezzi = a * vt_x = a (b m_cos(gamma) - a) / c = -a m_cos(beta)
    g.bm = -db / c;
    // back-rotation by theta0 = -m_atan2(v1y, v1x) (mod 2 pi): cos = v1x/a, sin = -v1y/a
    g.ct = v1x / a;
    g.st = -v1y / a;
    g.sgnC = sgnC;
}

}  // namespace ebem
