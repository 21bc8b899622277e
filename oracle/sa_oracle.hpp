// ORACLE — test infrastructure only.  Nothing in the product library links or
// calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load the oracle, and only as the checker.
//
// CPU restatement, in C++, of the reference's semi-analytic ("SA") assembly of
// the energetic space-time BEM blocks E_l: outer Gauss-Hammer quadrature on the
// source triangle, closed-form inner integrals on the field triangle, separate
// P- and S-wave fronts.  Each routine follows one MATLAB function of the
// reference (paths relative to the reference project root; "f/" abbreviates
// "functions/", "SA/" abbreviates
// "f/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/calcoloMatrice/") and keeps
// its evaluation order, thresholds and branch structure, so that the oracle's
// numbers are the reference's numbers up to libm rounding.
//
// MATLAB semantics reproduced explicitly:
//  * sign(0) = 0;
//  * acos/asin/sqrt of arguments that leave the real domain by rounding return
//    complex values in MATLAB, and the reference keeps only the real part
//    (SA/operazioniGeometriche/rotazioneInversaEulero.m:66); the real part of
//    acos(1+d) is acos(1), so arguments are clamped to the real domain;
//  * min() ignores NaN.
//
// The scalar type is `real` so that the same source compiles once with double
// (the oracle) and once with an operation-counting type (the flop census).
#pragma once

#include <cmath>
#include <cstring>
#include <algorithm>

#if defined(ORACLE_QUAD)
// quad precision (binary128) evaluation of the same formulas on the same
// double inputs: the arbiter for "the exact value of the reference's formulas"
#include <quadmath.h>
namespace oracle {
typedef __float128 real;
inline real sqrt(real x) { return sqrtq(x); }
inline real sin(real x) { return sinq(x); }
inline real cos(real x) { return cosq(x); }
inline real log(real x) { return logq(x); }
inline real acos(real x) { return acosq(x); }
inline real asin(real x) { return asinq(x); }
inline real atan2(real y, real x) { return atan2q(y, x); }
inline real fabs(real x) { return fabsq(x); }
}
#elif !defined(ORACLE_REAL)
namespace oracle { typedef double real; }
#else
namespace oracle { typedef ORACLE_REAL real; }
#endif

namespace oracle {

using std::sqrt; using std::sin; using std::cos; using std::log;
using std::acos; using std::asin; using std::atan2; using std::fabs;

static const double PI = 3.141592653589793238462643383279502884;

inline real sgn(const real& x) { return x > 0 ? real(1) : (x < 0 ? real(-1) : real(0)); }
inline real acos_r(const real& x) { return x >= 1 ? acos(real(1)) : (x <= -1 ? acos(real(-1)) : acos(x)); }
inline real asin_r(const real& x) { return x >= 1 ? asin(real(1)) : (x <= -1 ? asin(real(-1)) : asin(x)); }
inline real sqrt_r(const real& x) { return x > 0 ? sqrt(x) : real(0); }
inline real rmin(const real& a, const real& b) { return (a < b) ? a : b; }
inline real rmax(const real& a, const real& b) { return (a > b) ? a : b; }

struct M3 {
    real m[3][3];
    M3() { for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) m[i][j] = real(0); }
    static M3 eye(const real& s) { M3 r; r.m[0][0] = s; r.m[1][1] = s; r.m[2][2] = s; return r; }
};
inline M3 operator+(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r.m[i][j] = a.m[i][j] + b.m[i][j]; return r; }
inline M3 operator-(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r.m[i][j] = a.m[i][j] - b.m[i][j]; return r; }
inline M3 operator*(const real& s, const M3& a) { M3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r.m[i][j] = s * a.m[i][j]; return r; }
inline M3 operator*(const M3& a, const real& s) { M3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r.m[i][j] = a.m[i][j] * s; return r; }
inline M3 operator/(const M3& a, const real& s) { M3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r.m[i][j] = a.m[i][j] / s; return r; }
inline M3 matmul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
        r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}
inline M3 transpose(const M3& a) { M3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r.m[i][j] = a.m[j][i]; return r; }
// u' * v for row vectors u, v (outer product)
inline M3 outer(const real u[3], const real v[3]) { M3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r.m[i][j] = u[i] * v[j]; return r; }

inline real dot3(const real a[3], const real b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross3(const real a[3], const real b[3], real r[3]) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

// --------------------------------------------------------------------------
// SA/operazioniGeometriche/calcoloSistemaRiferimento.m:1-45
struct SdR { real L1, e1[3], L3, e3[3], cos_d, delta, sin_d, e2[3]; };

inline SdR calcoloSistemaRiferimento(const real T3[3][3], const real vnF[3]) {
    SdR s;
    real vl1[3] = {T3[1][0] - T3[0][0], T3[1][1] - T3[0][1], T3[1][2] - T3[0][2]};
    s.L1 = sqrt(vl1[0] * vl1[0] + vl1[1] * vl1[1] + vl1[2] * vl1[2]);
    for (int c = 0; c < 3; c++) s.e1[c] = vl1[c] / s.L1;
    real vl3[3] = {T3[2][0] - T3[0][0], T3[2][1] - T3[0][1], T3[2][2] - T3[0][2]};
    s.L3 = sqrt(vl3[0] * vl3[0] + vl3[1] * vl3[1] + vl3[2] * vl3[2]);
    for (int c = 0; c < 3; c++) s.e3[c] = vl3[c] / s.L3;
    s.cos_d = dot3(s.e3, s.e1);
    s.delta = acos_r(s.cos_d);
    s.sin_d = sin(s.delta);
    real e2[3];
    cross3(vnF, s.e1, e2);
    real n2 = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    for (int c = 0; c < 3; c++) s.e2[c] = e2[c] / n2;
    return s;
}

// SA/operazioniGeometriche/calcoloDistanzaTriangolo.m:1-52
inline real calcoloDistanzaTriangolo(const real tri2D[3][2]) {
    real D[3];
    for (int k = 0; k < 3; k++) D[k] = sqrt(tri2D[k][0] * tri2D[k][0] + tri2D[k][1] * tri2D[k][1]);
    const int pa[3] = {0, 1, 0}, pb[3] = {1, 2, 2};
    real best = real(0); bool have = false;
    for (int i = 0; i < 3; i++) {
        const real* P1 = tri2D[pa[i]];
        const real* P2 = tri2D[pb[i]];
        real d1 = D[pa[i]], d2 = D[pb[i]];
        real vL[2] = {P2[0] - P1[0], P2[1] - P1[1]};
        real L = sqrt(vL[0] * vL[0] + vL[1] * vL[1]);
        real d;
        if (-(P1[0] * vL[0] + P1[1] * vL[1]) < -1.0e-6) {
            d = d1;
        } else if (-(P2[0] * (-vL[0]) + P2[1] * (-vL[1])) < -1.0e-6) {
            d = d2;
        } else {
            real cosang = (-P1[0] / d1) * (vL[0] / L) + (-P1[1] / d1) * (vL[1] / L);
            real sinang = sqrt_r(1 - cosang * cosang);
            d = d1 * sinang;
        }
        if (d != d) continue;                 // MATLAB min() omits NaN
        if (!have || d < best) { best = d; have = true; }
    }
    return best;
}

// SA/operazioniGeometriche/preparazioneTriangolo.m:1-115
struct Prep { real zeta, children[3][3][2], dMIN, c[3], sign_prod; };

inline Prep preparazioneTriangolo(const real sp[3], const real T3[3][3], const real vnF[3], const SdR& S) {
    Prep p;
    real dsp[3] = {sp[0] - T3[0][0], sp[1] - T3[0][1], sp[2] - T3[0][2]};
    real param_s = dot3(vnF, dsp);
    real sp_plane[3];
    for (int c = 0; c < 3; c++) sp_plane[c] = sp[c] - param_s * vnF[c];
    real dd[3] = {sp[0] - sp_plane[0], sp[1] - sp_plane[1], sp[2] - sp_plane[2]};
    real sign_prod = dot3(dd, vnF);
    if (fabs(sign_prod) <= 1.0e-6) sign_prod = real(0);
    p.sign_prod = sgn(sign_prod);
    p.zeta = fabs(param_s);
    if (p.zeta < 1.0e-6) p.zeta = real(0);

    real diff[3] = {T3[0][0] - sp_plane[0], T3[0][1] - sp_plane[1], T3[0][2] - sp_plane[2]};
    real tri2D[3][2];
    tri2D[0][0] = dot3(diff, S.e1);
    tri2D[0][1] = dot3(diff, S.e2);
    tri2D[1][0] = tri2D[0][0] + S.L1;
    tri2D[1][1] = tri2D[0][1] + real(0);
    tri2D[2][0] = tri2D[0][0] + S.L3 * S.cos_d;
    tri2D[2][1] = tri2D[0][1] + S.L3 * S.sin_d;

    for (int k = 0; k < 3; k++) { p.children[k][0][0] = real(0); p.children[k][0][1] = real(0); }
    for (int d = 0; d < 2; d++) {
        p.children[0][1][d] = tri2D[0][d]; p.children[0][2][d] = tri2D[1][d];
        p.children[1][1][d] = tri2D[1][d]; p.children[1][2][d] = tri2D[2][d];
        p.children[2][1][d] = tri2D[2][d]; p.children[2][2][d] = tri2D[0][d];
    }
    p.c[0] = (tri2D[0][0] * tri2D[1][1]) - (tri2D[0][1] * tri2D[1][0]);
    p.c[1] = (tri2D[1][0] * tri2D[2][1]) - (tri2D[1][1] * tri2D[2][0]);
    p.c[2] = (tri2D[2][0] * tri2D[0][1]) - (tri2D[2][1] * tri2D[0][0]);

    real A_doppia = (tri2D[1][0] - tri2D[0][0]) * (tri2D[2][1] - tri2D[0][1]);
    real eta2 = p.c[2] / A_doppia;
    real eta3 = p.c[0] / A_doppia;
    real eta1 = 1 - eta2 - eta3;
    bool inside = (-1.0e-6 <= eta1) && (-1.0e-6 <= eta2) && (-1.0e-6 <= eta3) &&
                  (eta1 <= 1) && (eta2 <= 1) && (eta3 <= 1);
    p.dMIN = inside ? real(0) : calcoloDistanzaTriangolo(tri2D);
    return p;
}

// SA/operazioniGeometriche/calcoloDatiTriangolo.m:1-39
struct Info { real a, b, c, cos_alpha, cos_beta, cos_gamma, sin_alpha, sin_beta, sin_gamma, alpha, beta, gamma; };

inline Info calcoloDatiTriangolo(const real v[3][2], real tri2D[3][2]) {
    Info f;
    real dx, dy;
    dx = v[1][0] - v[0][0]; dy = v[1][1] - v[0][1]; f.a = sqrt(dx * dx + dy * dy);
    dx = v[2][0] - v[0][0]; dy = v[2][1] - v[0][1]; f.b = sqrt(dx * dx + dy * dy);
    dx = v[2][0] - v[1][0]; dy = v[2][1] - v[1][1]; f.c = sqrt(dx * dx + dy * dy);
    f.cos_alpha = (f.b * f.b + f.c * f.c - f.a * f.a) / (2 * f.b * f.c);
    f.cos_beta  = (f.a * f.a + f.c * f.c - f.b * f.b) / (2 * f.a * f.c);
    f.cos_gamma = (f.a * f.a + f.b * f.b - f.c * f.c) / (2 * f.a * f.b);
    f.sin_alpha = sqrt_r(1 - f.cos_alpha * f.cos_alpha);
    f.sin_beta  = sqrt_r(1 - f.cos_beta * f.cos_beta);
    f.sin_gamma = sqrt_r(1 - f.cos_gamma * f.cos_gamma);
    f.alpha = acos_r(f.cos_alpha);
    f.beta  = acos_r(f.cos_beta);
    f.gamma = acos_r(f.cos_gamma);
    tri2D[0][0] = real(0); tri2D[0][1] = real(0);
    tri2D[1][0] = f.a; tri2D[1][1] = real(0);
    tri2D[2][0] = f.b * f.cos_gamma; tri2D[2][1] = f.b * f.sin_gamma;
    return f;
}

// f/BEMenerg_analiticIntg/coefficientiB/BEMenerg_coreSA_coeffB.m:1-45
struct Bset { M3 B[6]; };

inline Bset coeffB(const real& zeta, const Info& f, const real& sign_prod) {
    real A1[3] = {real(1), real(0), real(0)};
    real A2[3] = {f.cos_gamma, f.sin_gamma, real(0)};
    real A3[3] = {real(0), real(0), -sign_prod};
    Bset b;
    b.B[0] = (zeta * zeta) * outer(A3, A3);
    b.B[1] = (zeta * (outer(A1, A3) + outer(A3, A1))) / f.sin_gamma;
    b.B[2] = (zeta * (outer(A2, A3) + outer(A3, A2))) / f.sin_gamma;
    b.B[3] = outer(A1, A1) / (f.sin_gamma * f.sin_gamma);
    b.B[4] = (outer(A1, A2) + outer(A2, A1)) / (f.sin_gamma * f.sin_gamma);
    b.B[5] = outer(A2, A2) / (f.sin_gamma * f.sin_gamma);
    return b;
}

struct Phi5 { real p[6]; };   // p[1..5] as in the reference's Phi(1..5)

inline Phi5 phiAll(const real& T1t, const real& T2t, const real& gamma, const real& cos_gamma) {
    Phi5 P;
    P.p[0] = real(0);
    P.p[1] = 2 * sin(T2t / 2) * sin(T1t / 2);
    P.p[2] = 2 * sin(gamma - (T2t / 2)) * sin(T1t / 2);
    P.p[3] = real(0.5) * (T1t - (cos(T2t) * sin(T1t)));
    P.p[4] = real(-0.5) * (-(sin(T1t) * cos(gamma - T2t)) + (T1t * cos_gamma));
    P.p[5] = real(0.5) * (T1t - (cos(2 * gamma - T2t) * sin(T1t)));
    return P;
}

struct R4 { M3 r1, r2, r3, r4; };
struct R2 { M3 r5, r6; };

// f/BEMenerg_analiticIntg/BEMenerg_analiticIntg_CC.m:1-93
inline R4 intg_CC(const real& RS, const real& rhoS, const real& RP, const real& rhoP, const real& zeta,
                  const real& TH1, const real& TH2, const Info& f, const Bset& B) {
    real T1t = TH2 - TH1, T2t = TH2 + TH1;
    R4 o;
    if (zeta > 1.0e-6) {
        real I1 = RP - RS;
        real I2 = RP - RS + (zeta * zeta * (1 / RP - 1 / RS));
        real I3 = log((rhoP + RP) / (rhoS + RS)) - (rhoP / RP) + (rhoS / RS);
        real I4 = -(1 / RP) + (1 / RS);
        real I5 = -(1 / RP) + (1 / RS) + (zeta * zeta / 3) * ((1 / (RP * RP * RP)) - (1 / (RS * RS * RS)));
        real q1 = rhoP / RP, q2 = rhoS / RS;
        real I6 = (1 / (3 * zeta * zeta)) * (q1 * q1 * q1 - q2 * q2 * q2);
        real I7 = (real(-1) / 3) * ((1 / (RP * RP * RP)) - (1 / (RS * RS * RS)));
        Phi5 P = phiAll(T1t, T2t, f.gamma, f.cos_gamma);
        M3 B_1 = P.p[5] * B.B[3] + P.p[4] * B.B[4] + P.p[3] * B.B[5];
        M3 B_2 = P.p[2] * B.B[1] + P.p[1] * B.B[2];
        M3 B_3 = B.B[0];
        o.r1 = M3::eye(T1t * I1);
        o.r2 = (I2 * B_1) + (I3 * B_2) + ((T1t * I4) * B_3);
        o.r3 = M3::eye(T1t * I4);
        o.r4 = (I5 * B_1) + (I6 * B_2) + ((T1t * I7) * B_3);
    } else {
        real I1 = RP - RS;
        real I2 = I1;
        real I4 = -(1 / RP) + (1 / RS);
        real I5 = I4;
        Phi5 P = phiAll(T1t, T2t, f.gamma, f.cos_gamma);
        M3 B_1 = (P.p[5] * B.B[3]) + (P.p[4] * B.B[4]) + (P.p[3] * B.B[5]);
        o.r1 = M3::eye(T1t * I1);
        o.r2 = I2 * B_1;
        o.r3 = M3::eye(T1t * I4);
        o.r4 = I5 * B_1;
    }
    return o;
}

// f/BEMenerg_analiticIntg/BEMenerg_analiticIntg_SC_P.m:1-54
inline R4 intg_SC_P(const real& RP, const real& rhoP, const real& zeta, const real& TH1, const real& TH2,
                    const Info& f, const Bset& B) {
    real T1t = TH2 - TH1, T2t = TH2 + TH1;
    real I1 = RP - zeta;
    real I2 = RP + (zeta * zeta / RP) - (2 * zeta);
    real I3 = log((rhoP + RP) / zeta) - (rhoP / RP);
    real I4 = -(1 / RP) + (1 / zeta);
    real I5 = -(1 / RP) + (zeta * zeta / (3 * RP * RP * RP)) + (2 / (3 * zeta));
    real q1 = rhoP / RP;
    real I6 = (1 / (3 * zeta * zeta)) * (q1 * q1 * q1);
    real I7 = -(1 / (3 * RP * RP * RP)) + (1 / (3 * zeta * zeta * zeta));
    Phi5 P = phiAll(T1t, T2t, f.gamma, f.cos_gamma);
    M3 B_1 = P.p[5] * B.B[3] + P.p[4] * B.B[4] + P.p[3] * B.B[5];
    M3 B_2 = P.p[2] * B.B[1] + P.p[1] * B.B[2];
    M3 B_3 = B.B[0];
    R4 o;
    o.r1 = M3::eye(T1t * I1);
    o.r2 = (I2 * B_1) + (I3 * B_2) + ((T1t * I4) * B_3);
    o.r3 = M3::eye(T1t * I4);
    o.r4 = (I5 * B_1) + (I6 * B_2) + ((T1t * I7) * B_3);
    return o;
}

// f/BEMenerg_analiticIntg/BEMenerg_analiticIntg_SC_SP.m:1-75
inline R2 intg_SC_SP(const real& RS, const real& rhoS, const real& zeta, const real& TH1, const real& TH2,
                     const Info& f, const Bset& B) {
    real T1t = TH2 - TH1, T2t = TH2 + TH1;
    R2 o;
    if (zeta > 1.0e-6) {
        real I1 = RS - zeta;
        real I2 = RS + (zeta * zeta / RS) - (2 * zeta);
        real I3 = log((rhoS + RS) / zeta) - (rhoS / RS);
        real I4 = -(1 / RS) + (1 / zeta);
        Phi5 P = phiAll(T1t, T2t, f.gamma, f.cos_gamma);
        M3 B_1 = P.p[5] * B.B[3] + P.p[4] * B.B[4] + P.p[3] * B.B[5];
        M3 B_2 = P.p[2] * B.B[1] + P.p[1] * B.B[2];
        M3 B_3 = B.B[0];
        o.r5 = M3::eye(T1t * I1);
        o.r6 = (I2 * B_1) + (I3 * B_2) + ((T1t * I4) * B_3);
    } else {
        real I1 = RS, I2 = RS;
        real p3 = real(0.5) * (T1t - (cos(T2t) * sin(T1t)));
        real p4 = real(-0.5) * ((T1t * f.cos_gamma) - (sin(T1t) * cos(f.gamma - T2t)));
        real p5 = real(0.5) * (T1t - (cos(2 * f.gamma - T2t) * sin(T1t)));
        M3 B_1 = p5 * B.B[3] + p4 * B.B[4] + p3 * B.B[5];
        o.r5 = M3::eye(T1t * I1);
        o.r6 = I2 * B_1;
    }
    return o;
}

// f/BEMenerg_analiticIntg/coefficientiG/BEMenerg_analiticIntg_coeffG_TC.m:1-182
// Returns G(1..19) in g[1..19]; entries the reference never assigns stay 0.
inline void coeffG_TC(const real& zeta, const real& RS, const real& rhoS, const real& TH1, const real& TH2,
                      const Info& f, real G[20]) {
    for (int k = 0; k < 20; k++) G[k] = real(0);
    const real a = f.a, sin_beta = f.sin_beta, sin_alpha = f.sin_alpha;
    const real cos_alpha = f.cos_alpha, cos_beta = f.cos_beta, cos_gamma = f.cos_gamma;
    const real alpha = f.alpha, beta = f.beta, gamma = f.gamma;
    real T1t = TH2 - TH1, T2t = TH2 + TH1;
    real F = a * sin_beta;
    Phi5 P = phiAll(T1t, T2t, gamma, cos_gamma);
    if (zeta > 1.0e-6) {
        real R1 = F / sin(TH1 + beta);
        real R2 = F / sin(TH2 + beta);
        real FR1 = zeta / R1, FR2 = zeta / R2;
        real ADD = zeta * zeta + F * F;
        real g1 = sqrt(1 + FR1 * FR1);
        real g2 = sqrt(1 + FR2 * FR2);
        real c1b = cos(TH1 + beta), c2b = cos(TH2 + beta);
        real g3 = real(0.5) * (log((g1 + c1b) * (g2 - c2b)) - log((g1 - c1b) * (g2 + c2b)));
        real g4 = log((1 / FR1) + sqrt(1 + (1 / FR1) * (1 / FR1)));
        real g5 = log((1 / FR2) + sqrt(1 + (1 / FR2) * (1 / FR2)));
        real sq = sqrt(ADD);
        real g7 = real(PI) - acos_r((-zeta * c2b) / sq) - acos_r((zeta * c1b) / sq);
        real g8 = F * F / ADD;
        real L = (rhoS / RS) - log((rhoS + RS) / zeta);
        G[1] = -(RS * T1t) + (zeta * g7) + (F * g3);
        G[4] = (1 / RS * T1t) - (1 / zeta * g7);
        G[5] = cos(gamma - TH2) * g5 - cos(gamma - TH1) * g4 - cos_alpha * g3
               + L * (cos(gamma - TH2) - cos(gamma - TH1));
        G[6] = -cos(TH2) * g5 + cos(TH1) * g4 - cos_beta * g3
               - L * (cos(TH2) - cos(TH1));
        real Q = (RS * RS + zeta * zeta) / RS;
        G[7] = zeta * g7 - Q * P.p[5]
               + F * (-g1 * cos(alpha - gamma + TH1) + g2 * cos(alpha - gamma + TH2) + g3 * (sin_alpha * sin_alpha));
        G[8] = -zeta * cos_gamma * g7 - Q * P.p[4]
               + F * (-sin_alpha * sin_beta * g3 + g1 * cos(TH1 + alpha) - g2 * cos(TH2 + alpha));
        G[9] = zeta * g7 - Q * P.p[3]
               + F * ((sin_beta * sin_beta) * g3 + g1 * cos(TH1 - beta) - g2 * cos(TH2 - beta));
        real s1b = sin(TH1 + beta), s2b = sin(TH2 + beta);
        G[14] = 1 / (3 * RS * RS * RS) * T1t
                + 1 / (3 * zeta * zeta) * (F / ADD * (c1b / g1 - c2b / g2) - 1 / zeta * g7);
        real rs3 = rhoS * rhoS * rhoS;
        G[15] = -rs3 / (3 * zeta * zeta * RS * RS * RS) * P.p[2]
                + 1 / (3 * zeta * zeta) * ((sin_alpha * s2b - g8 * cos_alpha * c2b) / g2
                                           + (-sin_alpha * s1b + g8 * cos_alpha * c1b) / g1);
        G[16] = -rs3 / (3 * zeta * zeta * RS * RS * RS) * P.p[1]
                + 1 / (3 * zeta * zeta) * ((sin_beta * s1b + g8 * cos_beta * c1b) / g1
                                           + (-sin_beta * s2b - g8 * cos_beta * c2b) / g2);
        real K = ((1 / RS) - (zeta * zeta / (3 * RS * RS * RS)));
        G[17] = real(1) / 3 * (-(s2b * s2b) * cos(alpha - gamma + TH2) + g8 * (cos_alpha * cos_alpha) * c2b) / (F * g2)
                - real(1) / 3 * (-(s1b * s1b) * cos(alpha - gamma + TH1) + g8 * (cos_alpha * cos_alpha) * c1b) / (F * g1)
                - g7 / (3 * zeta)
                + K * P.p[5];
        G[18] = real(1) / 3 * ((s2b * s2b) * cos(alpha + TH2) + g8 * (cos_alpha * cos_beta * c2b)) / (F * g2)
                - real(1) / 3 * ((s1b * s1b) * cos(alpha + TH1) + g8 * (cos_alpha * cos_beta * c1b)) / (F * g1)
                + g7 / (3 * zeta) * cos_gamma
                + K * P.p[4];
        G[19] = real(1) / 3 * ((s2b * s2b) * cos(beta - TH2) + g8 * ((cos_beta * cos_beta) * c2b)) / (F * g2)
                - real(1) / 3 * ((s1b * s1b) * cos(beta - TH1) + g8 * ((cos_beta * cos_beta) * c1b)) / (F * g1)
                - g7 / (3 * zeta)
                + K * P.p[3];
    } else {
        real c1b = cos(TH1 + beta), c2b = cos(TH2 + beta);
        real s1b = sin(TH1 + beta), s2b = sin(TH2 + beta);
        real g_3 = real(0.5) * (log((1 + c1b) * (1 - c2b)) - log((1 - c1b) * (1 + c2b)));
        G[1] = (F * g_3) - (RS * T1t);
        G[4] = 1 / F * (c2b - c1b) + 1 / RS * T1t;
        G[7] = -RS * P.p[5] + F * (cos(alpha - gamma + TH2) - cos(alpha - gamma + TH1) + (sin_alpha * sin_alpha) * g_3);
        G[8] = -RS * P.p[4] + F * (cos(TH1 + alpha) - cos(TH2 + alpha) - sin_alpha * sin_beta * g_3);
        G[9] = -RS * P.p[3] + F * (cos(beta - TH1) - cos(beta - TH2) + (sin_beta * sin_beta) * g_3);
        G[17] = 1 / (3 * F) * (((1 + cos_alpha * cos_alpha) * c2b - (s2b * s2b) * cos(alpha - gamma + TH2))
                               - ((1 + cos_alpha * cos_alpha) * c1b - (s1b * s1b) * cos(alpha - gamma + TH1)))
                + 1 / RS * P.p[5];
        G[18] = 1 / (3 * F) * ((c2b * ((cos_alpha * cos_beta) + cos(alpha + beta)) + (s2b * s2b) * cos(alpha + TH2))
                               - (c1b * ((cos_alpha * cos_beta) + cos(alpha + beta)) + (s1b * s1b) * cos(alpha + TH1)))
                + 1 / RS * P.p[4];
        G[19] = 1 / (3 * F) * (((1 + cos_beta * cos_beta) * c2b + (s2b * s2b) * cos(TH2 - beta))
                               - ((1 + cos_beta * cos_beta) * c1b + (s1b * s1b) * cos(beta - TH1)))
                + 1 / RS * P.p[3];
    }
}

// f/BEMenerg_analiticIntg/coefficientiG/BEMenerg_analiticIntg_coeffG_TR_P.m:1-120
inline void coeffG_TR_P(const real& zeta, const real& TH1, const real& TH2, const Info& f, real G[20]) {
    for (int k = 0; k < 20; k++) G[k] = real(0);
    const real a = f.a, sin_beta = f.sin_beta, sin_alpha = f.sin_alpha;
    const real cos_alpha = f.cos_alpha, cos_beta = f.cos_beta, cos_gamma = f.cos_gamma;
    const real alpha = f.alpha, beta = f.beta, gamma = f.gamma;
    real T1t = TH2 - TH1, T2t = TH2 + TH1;
    real F = a * sin_beta;
    real R1 = F / sin(TH1 + beta);
    real R2 = F / sin(TH2 + beta);
    real FR1 = zeta / R1, FR2 = zeta / R2;
    real ADD = zeta * zeta + F * F;
    real p3 = real(0.5) * (T1t - (cos(T2t) * sin(T1t)));
    real p4 = real(-0.5) * (-(sin(T1t) * cos(gamma - T2t)) + (T1t * cos_gamma));
    real p5 = real(0.5) * (T1t - (cos(2 * gamma - T2t) * sin(T1t)));
    real g1 = sqrt(1 + FR1 * FR1);
    real g2 = sqrt(1 + FR2 * FR2);
    real c1b = cos(TH1 + beta), c2b = cos(TH2 + beta);
    real s1b = sin(TH1 + beta), s2b = sin(TH2 + beta);
    real g3 = real(0.5) * (log((g1 + c1b) * (g2 - c2b)) - log((g1 - c1b) * (g2 + c2b)));
    real g4 = log((1 / FR1) + sqrt(1 + (1 / FR1) * (1 / FR1)));
    real g5 = log((1 / FR2) + sqrt(1 + (1 / FR2) * (1 / FR2)));
    real sq = sqrt(ADD);
    real g7 = real(PI) - acos_r((-zeta * c2b) / sq) - acos_r((zeta * c1b) / sq);
    real g8 = F * F / ADD;
    G[1] = (zeta * (-T1t + g7)) + (F * g3);
    G[4] = 1 / zeta * (T1t - g7);
    G[5] = cos(gamma - TH2) * g5 - cos(gamma - TH1) * g4 - cos_alpha * g3;
    G[6] = -cos(TH2) * g5 + cos(TH1) * g4 - cos_beta * g3;
    G[7] = zeta * (g7 - 2 * p5) + F * (-g1 * cos(alpha - gamma + TH1) + g2 * cos(alpha - gamma + TH2) + g3 * (sin_alpha * sin_alpha));
    G[8] = -zeta * ((cos_gamma * g7) + 2 * p4) + F * (-sin_alpha * sin_beta * g3 + g1 * cos(TH1 + alpha) - g2 * cos(TH2 + alpha));
    G[9] = zeta * (g7 - 2 * p3) + F * ((sin_beta * sin_beta) * g3 + g1 * cos(TH1 - beta) - g2 * cos(TH2 - beta));
    G[14] = 1 / (3 * zeta * zeta) * (1 / zeta * (T1t - g7) + (F / ADD * (c1b / g1 - c2b / g2)));
    G[15] = 1 / (3 * zeta * zeta) * ((sin_alpha * s2b - g8 * cos_alpha * c2b) / g2
                                     + (-sin_alpha * s1b + g8 * cos_alpha * c1b) / g1);
    G[16] = 1 / (3 * zeta * zeta) * ((sin_beta * s1b + g8 * cos_beta * c1b) / g1
                                     + (-sin_beta * s2b - g8 * cos_beta * c2b) / g2);
    G[17] = (1 / (3 * F) * ((-(s2b * s2b) * cos(alpha - gamma + TH2) + g8 * (cos_alpha * cos_alpha) * c2b) / g2
                            - (-(s1b * s1b) * cos(alpha - gamma + TH1) + g8 * (cos_alpha * cos_alpha) * c1b) / g1))
            - (1 / (3 * zeta) * (g7 - 2 * p5));
    G[18] = (1 / (3 * F) * (((s2b * s2b) * cos(alpha + TH2) + g8 * (cos_alpha * cos_beta * c2b)) / g2
                            - ((s1b * s1b) * cos(alpha + TH1) + g8 * (cos_alpha * cos_beta * c1b)) / g1))
            + (1 / (3 * zeta) * ((g7 * cos_gamma) + 2 * p4));
    G[19] = (1 / (3 * F) * (((s2b * s2b) * cos(beta - TH2) + g8 * ((cos_beta * cos_beta) * c2b)) / g2
                            - ((s1b * s1b) * cos(beta - TH1) + g8 * ((cos_beta * cos_beta) * c1b)) / g1))
            - (1 / (3 * zeta) * (g7 - 2 * p3));
}

// f/BEMenerg_analiticIntg/coefficientiG/BEMenerg_analiticIntg_coeffG_TR_SP.m:1-111
inline void coeffG_TR_SP(const real& zeta, const real& TH1, const real& TH2, const Info& f, real G[20]) {
    for (int k = 0; k < 20; k++) G[k] = real(0);
    const real a = f.a, sin_beta = f.sin_beta, sin_alpha = f.sin_alpha;
    const real cos_alpha = f.cos_alpha, cos_beta = f.cos_beta, cos_gamma = f.cos_gamma;
    const real alpha = f.alpha, beta = f.beta, gamma = f.gamma;
    real T1t = TH2 - TH1, T2t = TH2 + TH1;
    real F = a * sin_beta;
    if (zeta > 1.0e-6) {
        real R1 = F / sin(TH1 + beta);
        real R2 = F / sin(TH2 + beta);
        real FR1 = zeta / R1, FR2 = zeta / R2;
        real ADD = zeta * zeta + F * F;
        real p3 = real(0.5) * (T1t - (cos(T2t) * sin(T1t)));
        real p4 = real(-0.5) * (-(sin(T1t) * cos(gamma - T2t)) + (T1t * cos_gamma));
        real p5 = real(0.5) * (T1t - (cos(2 * gamma - T2t) * sin(T1t)));
        real g1 = sqrt(1 + FR1 * FR1);
        real g2 = sqrt(1 + FR2 * FR2);
        real c1b = cos(TH1 + beta), c2b = cos(TH2 + beta);
        real g3 = real(0.5) * (log((g1 + c1b) * (g2 - c2b)) - log((g1 - c1b) * (g2 + c2b)));
        real g4 = log((1 / FR1) + sqrt(1 + (1 / FR1) * (1 / FR1)));
        real g5 = log((1 / FR2) + sqrt(1 + (1 / FR2) * (1 / FR2)));
        real sq = sqrt(ADD);
        real g7 = real(PI) - acos_r((-zeta * c2b) / sq) - acos_r((zeta * c1b) / sq);
        G[1] = (zeta * (-T1t + g7)) + (F * g3);
        G[4] = 1 / zeta * (T1t - g7);
        G[5] = cos(gamma - TH2) * g5 - cos(gamma - TH1) * g4 - cos_alpha * g3;
        G[6] = -cos(TH2) * g5 + cos(TH1) * g4 - cos_beta * g3;
        G[7] = zeta * (g7 - 2 * p5) + F * (-g1 * cos(alpha - gamma + TH1) + g2 * cos(alpha - gamma + TH2) + g3 * (sin_alpha * sin_alpha));
        G[8] = -zeta * ((cos_gamma * g7) + 2 * p4) + F * (-sin_alpha * sin_beta * g3 + g1 * cos(TH1 + alpha) - g2 * cos(TH2 + alpha));
        G[9] = zeta * (g7 - 2 * p3) + F * ((sin_beta * sin_beta) * g3 + g1 * cos(TH1 - beta) - g2 * cos(TH2 - beta));
    } else {
        real c1b = cos(TH1 + beta), c2b = cos(TH2 + beta);
        real g_3 = real(0.5) * (log((1 + c1b) * (1 - c2b)) - log((1 - c1b) * (1 + c2b)));
        G[1] = F * g_3;
        G[7] = F * (-cos(alpha - gamma + TH1) + cos(alpha - gamma + TH2) + (sin_alpha * sin_alpha) * g_3);
        G[8] = F * (-(sin_alpha * sin_beta * g_3) + cos(TH1 + alpha) - cos(TH2 + alpha));
        G[9] = F * ((sin_beta * sin_beta) * g_3 + cos(TH1 - beta) - cos(TH2 - beta));
    }
}

// f/BEMenerg_analiticIntg/BEMenerg_analiticIntg_TC.m:1-50
inline R4 intg_TC(const real& zeta, const real& RS, const real& rhoS, const real& TH1, const real& TH2,
                  const Info& f, const Bset& B) {
    real G[20];
    R4 o;
    if (zeta > 1.0e-6) {
        coeffG_TC(zeta, RS, rhoS, TH1, TH2, f, G);
        o.r1 = M3::eye(G[1]);
        o.r2 = G[4] * B.B[0] + G[5] * B.B[1] + G[6] * B.B[2] + G[7] * B.B[3] + G[8] * B.B[4] + G[9] * B.B[5];
        o.r3 = M3::eye(G[4]);
        o.r4 = G[14] * B.B[0] + G[15] * B.B[1] + G[16] * B.B[2] + G[17] * B.B[3] + G[18] * B.B[4] + G[19] * B.B[5];
    } else {
        coeffG_TC(real(0), RS, rhoS, TH1, TH2, f, G);
        o.r1 = M3::eye(G[1]);
        o.r2 = G[7] * B.B[3] + G[8] * B.B[4] + G[9] * B.B[5];
        o.r3 = M3::eye(G[4]);
        o.r4 = G[17] * B.B[3] + G[18] * B.B[4] + G[19] * B.B[5];
    }
    return o;
}

// f/BEMenerg_analiticIntg/BEMenerg_analiticIntg_TR_P.m:1-28
inline R4 intg_TR_P(const real& zeta, const real& TH1, const real& TH2, const Info& f, const Bset& B) {
    real G[20];
    coeffG_TR_P(zeta, TH1, TH2, f, G);
    R4 o;
    o.r1 = M3::eye(G[1]);
    o.r2 = G[4] * B.B[0] + G[5] * B.B[1] + G[6] * B.B[2] + G[7] * B.B[3] + G[8] * B.B[4] + G[9] * B.B[5];
    o.r3 = M3::eye(G[4]);
    o.r4 = G[14] * B.B[0] + G[15] * B.B[1] + G[16] * B.B[2] + G[17] * B.B[3] + G[18] * B.B[4] + G[19] * B.B[5];
    return o;
}

// f/BEMenerg_analiticIntg/BEMenerg_analiticIntg_TR_SP.m:1-40
inline R2 intg_TR_SP(const real& zeta, const real& TH1, const real& TH2, const Info& f, const Bset& B) {
    real G[20];
    R2 o;
    if (zeta > 1.0e-6) {
        coeffG_TR_SP(zeta, TH1, TH2, f, G);
        o.r5 = M3::eye(G[1]);
        o.r6 = G[4] * B.B[0] + G[5] * B.B[1] + G[6] * B.B[2] + G[7] * B.B[3] + G[8] * B.B[4] + G[9] * B.B[5];
    } else {
        coeffG_TR_SP(real(0), TH1, TH2, f, G);
        o.r5 = M3::eye(G[1]);
        o.r6 = G[7] * B.B[3] + G[8] * B.B[4] + G[9] * B.B[5];
    }
    return o;
}

enum IntgType { T_NONE = 0, T_SP_SP = 1, T_SP_P = 2, T_P = 3 };

struct R6 { M3 r[7]; };   // r[1..6] as ris1..ris6

// SA/BEMenerg_coreSA_calcIntgInt_childTriangle.m:1-235
inline R6 childTriangle(const real tri2D[3][2], const Info& f, const real& zeta, const real& RP, const real& rhoP,
                        const real& RS, const real& rhoS, const real& sign_prod, int type) {
    const real a = f.a, sinBeta = f.sin_beta, beta = f.beta, gamma = f.gamma;
    Bset matB = coeffB(zeta, f, sign_prod);
    real vt0 = (tri2D[2][0] - tri2D[1][0]) / f.c;
    real Bmezzi = a * vt0;
    real C = a * a - rhoP * rhoP;
    real DeltaP = Bmezzi * Bmezzi - C;
    C = a * a - rhoS * rhoS;
    real DeltaS = Bmezzi * Bmezzi - C;
    real rP = a * sinBeta / rhoP;
    real rS = a * sinBeta / rhoS;
    if (type == T_P) { rS = real(0); DeltaS = real(0); }

    R6 o;
    real TH1, TH2, TH3, TH4, TH5, TH6;
    if (DeltaP <= 1.0e-06) {
        TH1 = real(0); TH2 = gamma; TH3 = gamma; TH4 = gamma; TH5 = gamma; TH6 = gamma;
    } else if ((DeltaP > 1.0e-06) && (DeltaS <= 1.0e-06)) {
        real O1 = asin_r(rP) - beta;
        real O2 = real(PI) - asin_r(rP) - beta;
        real t1 = rmin(O1, O2), t2 = rmax(O1, O2);
        TH1 = real(0);
        TH2 = rmin(rmax(real(0), t1), gamma);
        TH3 = rmax(real(0), rmin(t2, gamma));
        TH4 = rmax(real(0), rmin(t2, gamma));
        TH5 = rmax(real(0), rmin(t2, gamma));
        TH6 = gamma;
    } else {
        real O1 = asin_r(rP) - beta;
        real O2 = real(PI) - asin_r(rP) - beta;
        real O3 = asin_r(rS) - beta;
        real O4 = real(PI) - asin_r(rS) - beta;
        real t1 = rmin(O1, O2), t2 = rmax(O1, O2);
        real t3 = rmin(O3, O4), t4 = rmax(O3, O4);
        TH1 = real(0);
        TH2 = rmin(rmax(real(0), t1), gamma);
        TH3 = rmin(rmax(real(0), t3), gamma);
        TH4 = rmax(real(0), rmin(t4, gamma));
        TH5 = rmax(real(0), rmin(t2, gamma));
        TH6 = gamma;
    }

    const bool spsp = (type == T_SP_SP);
    if (TH1 < TH2) {
        if (spsp) { R2 s = intg_SC_SP(RS, rhoS, zeta, TH1, TH2, f, matB); o.r[5] = o.r[5] + s.r5; o.r[6] = o.r[6] + s.r6; }
        R4 q = (type == T_P) ? intg_SC_P(RP, rhoP, zeta, TH1, TH2, f, matB)
                             : intg_CC(RS, rhoS, RP, rhoP, zeta, TH1, TH2, f, matB);
        o.r[1] = o.r[1] + q.r1; o.r[2] = o.r[2] + q.r2; o.r[3] = o.r[3] + q.r3; o.r[4] = o.r[4] + q.r4;
    }
    if (TH2 < TH3) {
        R2 s; if (spsp) s = intg_SC_SP(RS, rhoS, zeta, TH2, TH3, f, matB);
        R4 q = (type == T_P) ? intg_TR_P(zeta, TH2, TH5, f, matB)
                             : intg_TC(zeta, RS, rhoS, TH2, TH3, f, matB);
        o.r[1] = o.r[1] + q.r1; o.r[2] = o.r[2] + q.r2; o.r[3] = o.r[3] + q.r3; o.r[4] = o.r[4] + q.r4;
        if (spsp) { o.r[5] = o.r[5] + s.r5; o.r[6] = o.r[6] + s.r6; }
    }
    if (TH3 < TH4) {
        if (spsp) { R2 s = intg_TR_SP(zeta, TH3, TH4, f, matB); o.r[5] = o.r[5] + s.r5; o.r[6] = o.r[6] + s.r6; }
    }
    if (TH4 < TH5) {
        R2 s; if (spsp) s = intg_SC_SP(RS, rhoS, zeta, TH4, TH5, f, matB);
        R4 q = intg_TC(zeta, RS, rhoS, TH4, TH5, f, matB);
        o.r[1] = o.r[1] + q.r1; o.r[2] = o.r[2] + q.r2; o.r[3] = o.r[3] + q.r3; o.r[4] = o.r[4] + q.r4;
        if (spsp) { o.r[5] = o.r[5] + s.r5; o.r[6] = o.r[6] + s.r6; }
    }
    if (TH5 < TH6) {
        R2 s; if (spsp) s = intg_SC_SP(RS, rhoS, zeta, TH5, TH6, f, matB);
        R4 q = (type == T_P) ? intg_SC_P(RP, rhoP, zeta, TH5, TH6, f, matB)
                             : intg_CC(RS, rhoS, RP, rhoP, zeta, TH5, TH6, f, matB);
        o.r[1] = o.r[1] + q.r1; o.r[2] = o.r[2] + q.r2; o.r[3] = o.r[3] + q.r3; o.r[4] = o.r[4] + q.r4;
        if (spsp) { o.r[5] = o.r[5] + s.r5; o.r[6] = o.r[6] + s.r6; }
    }
    return o;
}

// SA/BEMenerg_coreSA_calcIntgInt_fieldTriangle.m:1-86
inline R6 fieldTriangle(const real& zeta, const real& RP, const real& rhoP, const real& RS, const real& rhoS,
                        const real children[3][3][2], const real c[3], const real& sign_prod, int type) {
    R6 o;
    for (int k = 0; k < 3; k++) {
        real child[3][2];
        for (int v = 0; v < 3; v++) { child[v][0] = children[k][v][0]; child[v][1] = children[k][v][1]; }
        real C = c[k];
        if (fabs(C) < 1.0e-06) continue;
        if (C < 0) {
            real t0 = child[1][0], t1 = child[1][1];
            child[1][0] = child[2][0]; child[1][1] = child[2][1];
            child[2][0] = t0; child[2][1] = t1;
        }
        real theta0 = atan2(child[1][1], child[1][0]);
        if (theta0 < 0) theta0 = fabs(theta0);
        else theta0 = 2 * real(PI) - theta0;
        real tri2D[3][2];
        Info f = calcoloDatiTriangolo(child, tri2D);
        R6 t = childTriangle(tri2D, f, zeta, RP, rhoP, RS, rhoS, sign_prod, type);
        real ct = cos(theta0), st = sin(theta0);
        M3 A;
        A.m[0][0] = ct; A.m[0][1] = st; A.m[0][2] = real(0);
        A.m[1][0] = -st; A.m[1][1] = ct; A.m[1][2] = real(0);
        A.m[2][0] = real(0); A.m[2][1] = real(0); A.m[2][2] = real(1);
        M3 At = transpose(A);
        t.r[2] = matmul(A, matmul(t.r[2], At));
        t.r[4] = matmul(A, matmul(t.r[4], At));
        t.r[6] = matmul(A, matmul(t.r[6], At));
        real coeff = sgn(C);
        for (int m = 1; m <= 6; m++) o.r[m] = o.r[m] + t.r[m] * coeff;
    }
    return o;
}

// SA/operazioniGeometriche/rotazioneInversaEulero.m:1-95 — the rotation
// matrix C only (it depends on the field triangle alone).
inline M3 eulerMatrix(const SdR& S, const real vnF[3]) {
    const real* X = S.e1;
    const real* Z = vnF;
    const real e1[3] = {real(1), real(0), real(0)};
    const real e3[3] = {real(0), real(0), real(1)};
    real cz[3]; cross3(e3, Z, cz);
    real ncz = sqrt(cz[0] * cz[0] + cz[1] * cz[1] + cz[2] * cz[2]);
    real phi, omega, psi;
    if (ncz < 1.0e-10) {
        real l[3] = {X[0], X[1], X[2]};
        phi = acos_r(dot3(e1, l));
        real cl[3]; cross3(e1, l, cl);
        if (dot3(cl, e3) < -1.0e-10) phi = 2 * real(PI) - phi;
        omega = (dot3(e3, Z) < 0) ? real(PI) : real(0);
        psi = real(0);
    } else {
        real l[3] = {cz[0] / ncz, cz[1] / ncz, cz[2] / ncz};
        phi = acos_r(dot3(e1, l));
        real cl[3]; cross3(e1, l, cl);
        if (dot3(cl, e3) < -1.0e-10) phi = 2 * real(PI) - phi;
        omega = acos_r(dot3(e3, Z));
        psi = acos_r(dot3(l, X));
        real clx[3]; cross3(l, X, clx);
        if (dot3(clx, Z) < -1.0e-10) psi = 2 * real(PI) - psi;
    }
    M3 Ap, Ao, Af;
    real cps = cos(psi), sps = sin(psi), co = cos(omega), so = sin(omega), cf = cos(phi), sf = sin(phi);
    Ap.m[0][0] = cps; Ap.m[0][1] = sps; Ap.m[1][0] = -sps; Ap.m[1][1] = cps; Ap.m[2][2] = real(1);
    Ao.m[0][0] = real(1); Ao.m[1][1] = co; Ao.m[1][2] = so; Ao.m[2][1] = -so; Ao.m[2][2] = co;
    Af.m[0][0] = cf; Af.m[0][1] = sf; Af.m[1][0] = -sf; Af.m[1][1] = cf; Af.m[2][2] = real(1);
    M3 C = matmul(matmul(Ap, Ao), Af);
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) if (fabs(C.m[i][j]) < 1.0e-14) C.m[i][j] = real(0);
    return C;
}

inline M3 rotazioneInversaEulero(const M3& C, const M3& ris) {
    return matmul(transpose(C), matmul(ris, C));
}

// rho_P / rho_S and the case split: SA/BEMenerg_coreSA_calcMatrixSubBlock.m:58-81
inline int classify(const real& zeta, const real& rP, const real& rS, const real& dMIN, real& rhoP, real& rhoS) {
    if (zeta == 0) { rhoP = rP; rhoS = rS; }
    else if (zeta < rS) { rhoP = sqrt(rP * rP - zeta * zeta); rhoS = sqrt(rS * rS - zeta * zeta); }
    else if (rS < zeta && zeta < rP) { rhoP = sqrt(rP * rP - zeta * zeta); rhoS = real(-1); }
    else { rhoP = real(-1); rhoS = real(-1); }
    if (dMIN < rhoS) return T_SP_SP;
    if (0 < rhoS && rhoS <= dMIN && dMIN < rhoP) return T_SP_P;
    if (rhoS <= 0 && dMIN < rhoP) return T_P;
    return T_NONE;
}

// Kernel combination of SA/BEMenerg_coreSA_calcMatrixSubBlock.m:101-104
inline M3 combine(const M3 r[7], const real& velP, const real& velS, const real& currT) {
    real vp2 = velP * velP, vs2 = velS * velS;
    real den = (velP * velS) * (velP * velS);
    M3 out;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
        real x = (r[1].m[i][j] - r[2].m[i][j]) / vp2
                 + (currT * currT) * (-r[3].m[i][j] + 3 * r[4].m[i][j])
                 + ((vp2 + vs2) * r[5].m[i][j] + (vp2 - vs2) * r[6].m[i][j]) / den;
        out.m[i][j] = x / 2;
    }
    return out;
}

}  // namespace oracle
