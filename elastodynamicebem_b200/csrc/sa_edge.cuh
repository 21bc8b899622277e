// Child-triangle integral of the semi-analytic method in the edge variable.
//
// The quantity is the reference's (SA/calcoloMatrice/
// BEMenerg_coreSA_calcIntgInt_childTriangle.m with the region integrals of
// f/BEMenerg_analiticIntg/*.m): for the child (O, V1, V2) of a projected
// outer node, the six kernel integrals over the parts of the child that lie
// between the S and P fronts (P terms) and inside the S front (P&S terms),
// already combined with the weights of BEMenerg_coreSA_calcMatrixSubBlock.m:101-104.
//
// The evaluation here is different and numerically stable (it does not
// reproduce the reference's rounding, it reproduces the exact value of its
// formulas — checked against a binary128 evaluation of them):
//
// * Orthonormal child frame.  The tensor parts are integrated against
//   cos^2, sin cos, sin^2, cos, sin of the polar angle directly, instead of
//   the skew basis A1 = (1,0,0), A2 = (cos g, sin g, 0) of coeffB.m whose
//   1/sin^2(g) factors amplify rounding by ~1e6 on thin children.
// * Edge variable.  Points of the edge V1V2 seen from O at angle phi from the
//   edge direction lie at distance R = F / sin(phi), F = 2 area / |V1V2|.
//   With s = -log(tan(phi/2)), R = F cosh(s), d(theta) = -sech(s) ds, and a
//   front of in-plane radius rho crosses the edge at s = +-acosh(rho / F).
//   Pieces whose radial limits are circles (or the projected node) have
//   closed-form angular integrals; pieces limited by the edge are integrated
//   by Gauss-Legendre in s on sub-pieces of length <= EBEM_EDGE_H.  In s the
//   integrands are analytic in the strip |Im s| < pi/2, so the rule converges
//   geometrically (10 nodes on sub-pieces of length <= 1: ~1e-14 relative).
// * Radial antiderivatives in r = sqrt(rho^2 + zeta^2):
//     A1 = r, A3 = -1/r                       (1/r, 1/r^3 times rho d rho)
//     B2 = r + zeta^2/r, C2 = ln(rho + r) - rho/r, D2 = -zeta^2/r
//                                             (in-plane, mixed, normal parts of r_i r_j / r^3)
//     B4 = -1/r + zeta^2/(3 r^3), C4 = -(r^2 + r rho + rho^2)/(3 (r + rho) r^3),
//     D4 = -zeta^2/(3 r^3)                    (same for r_i r_j / r^5; C4 is
//                                              rho^3/(3 zeta^2 r^3) minus its
//                                              constant 1/(3 zeta^2), free of the
//                                              1/zeta^2 cancellation)
// The front crossing decisions keep the reference's thresholds
// (DeltaP, DeltaS <= 1e-6 means "no crossing", childTriangle.m:62,75).
#pragma once

#include "sa_device.cuh"

#ifndef EBEM_EDGE_H
#define EBEM_EDGE_H 1.0
#endif
#ifndef EBEM_EDGE_NOINLINE
#define EBEM_EDGE_NOINLINE 1
#endif
#if EBEM_EDGE_NOINLINE && defined(__CUDACC__)
#define EBEM_EFN static __device__ __noinline__
#else
#define EBEM_EFN EBEM_DI
#endif

namespace ebem {

// 10-point Gauss-Legendre on [-1, 1] (positive half; symmetric)
#define EBEM_GL_N2 5
EBEM_HDI double gl_x(int k) {
    const double x[EBEM_GL_N2] = {0.14887433898163122, 0.4333953941292472, 0.6794095682990244,
                                  0.8650633666889845, 0.9739065285171717};
    return x[k];
}
EBEM_HDI double gl_w(int k) {
    const double w[EBEM_GL_N2] = {0.2955242247147528, 0.2692667193099965, 0.219086362515982,
                                  0.1494513491505804, 0.06667134430868814};
    return w[k];
}

// 6- and 8-point Gauss-Legendre on [-1, 1] (positive halves), for edge
// pieces shorter than 1/4 and 1/2 in s: the integrands are analytic in the
// strip |Im s| < pi/2, so on a piece of half-length h the n-point rule errs
// by about rho^(-2n), rho = (pi/2)/h + sqrt(((pi/2)/h)^2 + 1): 1.5e-17 for
// n = 6, h = 1/8; 2.3e-18 for n = 8, h = 1/4; 6.7e-17 for n = 10, h = 1/2.
EBEM_HDI double gl6_x(int k) {
    const double x[3] = {0.2386191860831969, 0.6612093864662645, 0.9324695142031519};
    return x[k];
}
EBEM_HDI double gl6_w(int k) {
    const double w[3] = {0.46791393457269104, 0.3607615730481387, 0.17132449237917027};
    return w[k];
}
EBEM_HDI double gl8_x(int k) {
    const double x[4] = {0.18343464249564978, 0.525532409916329, 0.7966664774136267, 0.9602898564975362};
    return x[k];
}
EBEM_HDI double gl8_w(int k) {
    const double w[4] = {0.36268378337836166, 0.3137066458778869, 0.22238103445337443, 0.10122853629037706};
    return w[k];
}

// The three rules in one table: nodes gt[0..23] (6-point at 0, 8-point at 6,
// 10-point at 14; each as -x then +x), weights gt[24..47] in the same order.
EBEM_HDI void gl_table_entry(int t, double& x, double& w) {
    int n = 10, j = t - 14;
    if (t < 6) { n = 6; j = t; }
    else if (t < 14) { n = 8; j = t - 6; }
    const int half = n / 2, k = j < half ? j : j - half;
    const double xk = n == 6 ? gl6_x(k) : n == 8 ? gl8_x(k) : gl_x(k);
    w = n == 6 ? gl6_w(k) : n == 8 ? gl8_w(k) : gl_w(k);
    x = j < half ? -xk : xk;
}

// Level-independent data of a child in the edge variable.
struct ChildE {
    double a, bm;            // |V1| and a*vt_x of the reference (for its DeltaP/DeltaS tests)
    double F;                // distance from O to the edge line
    double cb, sb, beta;     // cos/sin and value of the child angle at V1
    double gamma;            // child angle at O
    double s0, s1;           // s at theta = 0 (s0, largest) and at theta = gamma (s1)
    double ct, st;           // child frame -> plane frame rotation (V1 direction)
    double sgnC;
    double amax;             // max(|V1|, |V2|): a front of larger radius covers the whole edge
};

// Radial antiderivatives at in-plane radius rho (r = sqrt(rho^2+zeta^2)
// supplied by the caller).  The mixed (C) and normal (D) parts are only used
// for zeta > 0.
struct Rad { double A1, A3, B2, C2, D2, B4, C4, D4; };

EBEM_DI Rad radial_at(double rho, double r, double zeta) {
    Rad v;
    // one reciprocal gives both 1/r and 1/(r + rho)
    const double q = 1.0 / (r * (r + rho));
    const double ir = (r + rho) * q, ir3 = ir * ir * ir, z2 = zeta * zeta;
    v.A1 = r;
    v.A3 = -ir;
    v.B2 = r + z2 * ir;
    v.D2 = -z2 * ir;
    v.B4 = -ir + z2 * ir3 * (1.0 / 3.0);
    v.D4 = -z2 * ir3 * (1.0 / 3.0);
    if (zeta > 0) {
        v.C2 = m_log(rho + r) - rho * ir;
        v.C4 = -(r * r + r * rho + rho * rho) * ir3 * (r * q) * (1.0 / 3.0);
    } else {
        v.C2 = 0.0;
        v.C4 = 0.0;
    }
    return v;
}

EBEM_DI Rad rad_sub(const Rad& x, const Rad& y) {
    Rad v;
    v.A1 = x.A1 - y.A1; v.A3 = x.A3 - y.A3; v.B2 = x.B2 - y.B2; v.C2 = x.C2 - y.C2;
    v.D2 = x.D2 - y.D2; v.B4 = x.B4 - y.B4; v.C4 = x.C4 - y.C4; v.D4 = x.D4 - y.D4;
    return v;
}

// Radial vector -> (scalar, in-plane, mixed, normal) weights of the P terms
// (ris1..ris4 between the fronts) or of the P&S terms (ris5, ris6 inside S).
struct W4 { double sc, in, mx, zz; };

EBEM_DI W4 weigh(const Rad& v, bool p_terms, const LevelCtx& L) {
    W4 w;
    if (p_terms) {
        w.sc = L.k1 * v.A1 - L.t2 * v.A3;
        w.in = -L.k1 * v.B2 + 3 * L.t2 * v.B4;
        w.mx = -L.k1 * v.C2 + 3 * L.t2 * v.C4;
        w.zz = -L.k1 * v.D2 + 3 * L.t2 * v.D4;
    } else {
        w.sc = L.k5 * v.A1;
        w.in = L.k6 * v.B2;
        w.mx = L.k6 * v.C2;
        w.zz = L.k6 * v.D2;
    }
    return w;
}

// Accumulator in the child frame: S, T11, T12, T22, T13, T23, T33.
struct AccE { double S, t11, t12, t22, t13, t23, t33; };

// cos/sin of the polar angle theta (from V1) at edge variable s.
EBEM_DI void theta_cs(const ChildE& g, double s, double& c, double& sn) {
    double e = m_exp(s), ie = 1.0 / e;
    double ch = 0.5 * (e + ie);
    double sech = 1.0 / ch, th = (e - ie) / (e + ie);
    c = th * g.cb + sech * g.sb;
    sn = sech * g.cb - th * g.sb;
}

// Angle theta at a front crossing s = +-acosh(rho/F): phi = asin(F/rho) for
// s > 0, pi - asin(F/rho) for s < 0 (the reference's Omega values).
EBEM_DI void crossing_theta(const ChildE& g, double rho, bool positive, double& th, double& c, double& sn) {
    const double irho = 1.0 / rho;
    double sp = g.F * irho;                                      // sin(phi)
    double cp = sqrt_c((rho - g.F) * (rho + g.F)) * irho;        // |cos(phi)|
    double phi = asin_c(sp);
    if (!positive) { phi = kPi - phi; cp = -cp; }
    th = phi - g.beta;                                           // theta = phi - beta
    c = cp * g.cb + sp * g.sb;                                   // cos(phi - beta)
    sn = sp * g.cb - cp * g.sb;                                  // sin(phi - beta)
}

// Polar angle at edge variable sx = +-acosh(rho/F), clipped to the child's
// range [smin, smax]: beyond V1 (sx >= smax) it is 0, beyond V2 (sx <= smin)
// it is gamma.
EBEM_DI void clipped_theta(const ChildE& g, double rho, double sx, bool positive, double smin, double thg,
                           double cg, double sgm, double& th, double& c, double& sn) {
    if (sx >= g.s0) { th = 0.0; c = 1.0; sn = 0.0; }
    else if (sx <= smin) { th = thg; c = cg; sn = sgm; }
    else crossing_theta(g, rho, positive, th, c, sn);
}

// Both crossings s = +-sX, sX = acosh(rho/F), of a front of in-plane radius
// rho with the edge line (the caller has checked that it crosses), clipped to
// the child as clipped_theta does: (thA, cA, sA) at +sX, (thB, cB, sB) at -sX.
// One square root, one logarithm and at most one arcsine serve both sides
// (the angles are phi and pi - phi).
EBEM_DI void front_cross(const ChildE& g, double rho, double smin, double thg, double cg, double sgm, double& sX,
                         double& thA, double& cA, double& sA, double& thB, double& cB, double& sB) {
    const double q = sqrt_c((rho - g.F) * (rho + g.F));
    sX = m_log((rho + q) / g.F);
    const bool a0 = sX >= g.s0, ag = !a0 && sX <= smin;
    const bool b0 = -sX >= g.s0, bg = !b0 && -sX <= smin;
    double phi = 0.0, sp = 0.0, cp = 0.0;
    if (!(a0 || ag) || !(b0 || bg)) {
        const double irho = 1.0 / rho;
        sp = g.F * irho;
        cp = q * irho;
        phi = asin_c(sp);
    }
    if (a0) { thA = 0.0; cA = 1.0; sA = 0.0; }
    else if (ag) { thA = thg; cA = cg; sA = sgm; }
    else { thA = phi - g.beta; cA = cp * g.cb + sp * g.sb; sA = sp * g.cb - cp * g.sb; }
    if (b0) { thB = 0.0; cB = 1.0; sB = 0.0; }
    else if (bg) { thB = thg; cB = cg; sB = sgm; }
    else { thB = (kPi - phi) - g.beta; cB = -cp * g.cb + sp * g.sb; sB = sp * g.cb + cp * g.sb; }
}

// Circle-bounded piece between polar angles (tha; ca, sa) and (thb; cb_, sb_):
// the radial weights w are constant in theta.
EBEM_DI void add_circle(AccE& A, const W4& w, double tha, double ca, double sa, double thb, double cbb,
                        double sbb, double zs) {
    double dth = thb - tha;
    double s2 = 0.5 * (sbb * cbb - sa * ca);                      // (sin 2thb - sin 2tha)/4
    double icc = 0.5 * dth + s2, iss = 0.5 * dth - s2;
    double isc = -0.25 * ((cbb * cbb - sbb * sbb) - (ca * ca - sa * sa));
    double ic = sbb - sa, is = ca - cbb;
    A.S += w.sc * dth;
    A.t11 += w.in * icc;
    A.t12 += w.in * isc;
    A.t22 += w.in * iss;
    A.t13 += -zs * w.mx * ic;
    A.t23 += -zs * w.mx * is;
    A.t33 += w.zz * dth;
}

// Edge-bounded piece s in [slo, shi]: upper radial limit R(s) = F cosh s,
// lower limit fixed (its radial vector `lo`).
EBEM_EFN void add_edge(AccE& A, const ChildE& g, double slo, double shi, const Rad& lo, bool p_terms,
                      const LevelCtx& L, double zeta, double zs) {
    double len = shi - slo;
    if (!(len > 0)) return;
    int nsub = (int)ceil(len * (1.0 / EBEM_EDGE_H));
    if (nsub < 1) nsub = 1;
    double h = len / nsub;
    for (int p = 0; p < nsub; p++) {
        double mid = slo + (p + 0.5) * h, half = 0.5 * h;
#pragma unroll 2
        for (int q = 0; q < 2 * EBEM_GL_N2; q++) {
            int k = (q < EBEM_GL_N2) ? q : q - EBEM_GL_N2;
            double s = (q < EBEM_GL_N2) ? mid - half * gl_x(k) : mid + half * gl_x(k);
            double wq = half * gl_w(k);
            double e = m_exp(s), ie = 1.0 / e;
            double ch = 0.5 * (e + ie), sech = 1.0 / ch, th = (e - ie) / (e + ie);
            double c = th * g.cb + sech * g.sb;
            double sn = sech * g.cb - th * g.sb;
            double R = g.F * ch;
            double r = sqrt(R * R + zeta * zeta);
            Rad v = rad_sub(radial_at(R, r, zeta), lo);
            W4 w = weigh(v, p_terms, L);
            double f = wq * sech;
            A.S += f * w.sc;
            A.t11 += f * w.in * c * c;
            A.t12 += f * w.in * sn * c;
            A.t22 += f * w.in * sn * sn;
            A.t13 += -zs * f * w.mx * c;
            A.t23 += -zs * f * w.mx * sn;
            A.t33 += f * w.zz;
        }
    }
}

// log(tan(x/2)) for an angle x in (0, pi) given 2*area (cr) and the dot
// product (d) of the two edge vectors at that vertex with lengths product
// (p = |u||v|): tan(x/2) = cr / (p + d), with p + d = cr^2 / (p - d) when d < 0.
EBEM_DI double log_tan_half(double cr, double d, double p) {
    double pd = (d >= 0) ? (p + d) : (cr * cr) / (p - d);
    return m_log(cr / pd);
}

// Child (O, V1, V2) oriented counter-clockwise: level-independent data.
EBEM_DI void child_geo_e(ChildE& g, double v1x, double v1y, double v2x, double v2y, double sgnC) {
    double a = sqrt(v1x * v1x + v1y * v1y);
    double b = sqrt(v2x * v2x + v2y * v2y);
    double dx = v2x - v1x, dy = v2y - v1y;
    double c = sqrt(dx * dx + dy * dy);
    double cr = v1x * v2y - v1y * v2x;            // twice the child's area (> 0)
    double dg = v1x * v2x + v1y * v2y;            // angle at O
    double db = -(v1x * dx + v1y * dy);           // angle at V1
    double da = v2x * dx + v2y * dy;              // angle at V2
    g.a = a;
    g.F = cr / c;
    g.cb = db / (a * c);
    g.sb = cr / (a * c);
    g.bm = -db / c;
    g.beta = m_atan2(cr, db);
    g.gamma = m_atan2(cr, dg);
    g.s0 = -log_tan_half(cr, db, a * c);          // s at phi = beta
    g.s1 = log_tan_half(cr, da, b * c);           // s at phi = pi - alpha
    g.amax = fmax(a, b);
    g.ct = v1x / a;
    g.st = v1y / a;
    g.sgnC = sgnC;
}

// One child at one time level: S and the tensor in the plane frame, signed,
// added to (Sout, T[11,12,22,13,23,33]).
EBEM_DI void child_level_e(double& Sout, double T[6], const ChildE& g, const LevelCtx& L, double zeta, double sigma,
                           double rhoP, double rhoS, int type) {
    const bool isP = (type == T_P), spsp = (type == T_SP_SP);
    const double zs = zeta * sigma;
    // the reference's intersection tests (childTriangle.m:28-50, 62, 75)
    double DeltaP = g.bm * g.bm - (g.a * g.a - rhoP * rhoP);
    double DeltaS = isP ? 0.0 : g.bm * g.bm - (g.a * g.a - rhoS * rhoS);
    const bool xP = DeltaP > 1.0e-6, xS = xP && DeltaS > 1.0e-6;
    // lower radial limit of the P terms: the S front, or the node's
    // projection (r = zeta) when the S sphere misses the plane
    double rhoSe = isP ? 0.0 : rhoS;
    Rad VSe = radial_at(rhoSe, isP ? zeta : L.RS, zeta);
    Rad VP = radial_at(rhoP, L.RP, zeta);
    W4 wPc = weigh(rad_sub(VP, VSe), true, L);
    AccE A = {0, 0, 0, 0, 0, 0, 0};
    const double smax = g.s0, smin = g.s1;
    // boundary angles: theta = 0 at s0, gamma at s1
    const double th0 = 0.0, c0 = 1.0, sn0 = 0.0;
    double thg = g.gamma, cg, sgm;
    m_sincos(thg, &sgm, &cg);
    if (!xP) {
        add_circle(A, wPc, th0, c0, sn0, thg, cg, sgm, zs);
    } else {
        double sP = m_log((rhoP + sqrt_c((rhoP - g.F) * (rhoP + g.F))) / g.F);     // acosh(rhoP/F)
        // polar angles at s = +sP (phi < pi/2) and s = -sP, clipped to the child
        double thA, cA, sA, thB, cB, sB;
        clipped_theta(g, rhoP, sP, true, smin, thg, cg, sgm, thA, cA, sA);
        clipped_theta(g, rhoP, -sP, false, smin, thg, cg, sgm, thB, cB, sB);
        // circle pieces: s in [sP, smax] (theta from 0 to thA) and [smin, -sP] (thB to gamma)
        if (smax > sP) add_circle(A, wPc, th0, c0, sn0, thA, cA, sA, zs);
        if (-sP > smin) add_circle(A, wPc, thB, cB, sB, thg, cg, sgm, zs);
        // edge pieces of the P terms
        if (xS && !isP) {
            double sS = m_log((rhoS + sqrt_c((rhoS - g.F) * (rhoS + g.F))) / g.F);
            add_edge(A, g, fmax(sS, smin), fmin(sP, smax), VSe, true, L, zeta, zs);
            add_edge(A, g, fmax(-sP, smin), fmin(-sS, smax), VSe, true, L, zeta, zs);
        } else {
            add_edge(A, g, fmax(-sP, smin), fmin(sP, smax), VSe, true, L, zeta, zs);
        }
    }
    if (spsp) {
        // P&S terms: radial range [0, min(rhoS, R)]
        Rad V0 = radial_at(0.0, zeta, zeta);
        if (!(zeta > 0)) { V0.A1 = 0.0; V0.B2 = 0.0; V0.D2 = 0.0; }
        Rad VS = radial_at(rhoS, L.RS, zeta);
        W4 wSc = weigh(rad_sub(VS, V0), false, L);
        if (!xS) {
            add_circle(A, wSc, th0, c0, sn0, thg, cg, sgm, zs);
        } else {
            double sS = m_log((rhoS + sqrt_c((rhoS - g.F) * (rhoS + g.F))) / g.F);
            double thA, cA, sA, thB, cB, sB;
            clipped_theta(g, rhoS, sS, true, smin, thg, cg, sgm, thA, cA, sA);
            clipped_theta(g, rhoS, -sS, false, smin, thg, cg, sgm, thB, cB, sB);
            if (smax > sS) add_circle(A, wSc, th0, c0, sn0, thA, cA, sA, zs);
            if (-sS > smin) add_circle(A, wSc, thB, cB, sB, thg, cg, sgm, zs);
            add_edge(A, g, fmax(-sS, smin), fmin(sS, smax), V0, false, L, zeta, zs);
        }
    }
    // child frame -> plane frame: rotation by the direction of V1, signed
    const double c = g.ct, s = g.st, w = g.sgnC;
    const double cc = c * c, ss = s * s, cs = c * s;
    Sout += w * A.S;
    T[0] += w * (cc * A.t11 - 2 * cs * A.t12 + ss * A.t22);
    T[1] += w * (cs * A.t11 + (cc - ss) * A.t12 - cs * A.t22);
    T[2] += w * (ss * A.t11 + 2 * cs * A.t12 + cc * A.t22);
    T[3] += w * (c * A.t13 - s * A.t23);
    T[4] += w * (s * A.t13 + c * A.t23);
    T[5] += w * A.t33;
}

}  // namespace ebem
