// Warp-cooperative semi-analytic assembly: one warp per (source, field) pair.
//
// The value computed is the one of sa_assemble_kernel (thread per pair, the
// same closed-form child integrals of sa_edge.cuh); only the schedule differs:
//
// * Lane = child.  Lane 3 g + c owns child c of the projection of outer node g
//   of the source triangle onto the field plane.  Its
//   geometry (ChildE, the node's zeta, sigma, distance to the triangle and
//   weight) is level-independent and computed once per pair, not once per
//   level.
// * Per level a lane decides its pieces (BEMenerg_coreSA_calcIntgInt_childTriangle.m:
//   front crossings with the reference's DeltaP/DeltaS <= 1e-6 thresholds)
//   and evaluates the circle-bounded pieces in closed form.  An edge-bounded
//   piece int_{slo}^{shi} w(theta) [V(F cosh s) - V_lo] sech(s) ds is split
//   into int w V(F cosh s) sech ds (quadrature) minus V_lo int w dtheta over
//   the same angular interval (closed form, the circle formula).
// * Whole-range pieces (the piece spans the child's entire edge: the edge
//   lies between the fronts, or inside the S front) use per-child moments
//   int w V_f(F cosh s) sech ds of the eight radial functions, computed once
//   per child by the whole warp the first time they are needed: no quadrature
//   at later levels.
// * The remaining (partial) edge pieces of all lanes are put in a per-warp
//   list and their Gauss-Legendre nodes are evaluated by all 32 lanes, each
//   node weighted by its child's node weight and orientation sign and taken
//   in the plane frame, so every lane sums into the same pair value.
// * The per-level pair value is a warp reduction into per-level sums; after
//   a chunk of levels one lane per level forms F(t_k) (level_pair in
//   sa_assemble.cu).
//
// Rules with more than 30 children run their outer nodes in groups of 10.
#pragma once

#include "sa_pair.cuh"

namespace ebem {

#ifndef EBEM_GL_ADAPT
#define EBEM_GL_ADAPT 1   // 1: 6 or 8 Gauss-Legendre nodes on edge pieces up to 1/4 or 1/2 long, else 10
#endif

// Per-warp shared state for R children per lane (32 R child slots, at most
// 3 edge pieces per child and level).
template <int R>
struct WarpShared {
    double slo[96 * R], h[96 * R];
    int off[96 * R + 1];
    int who[96 * R];                            // child slot | (P terms ? 64 : 0)
    double F[32 * R], cbp[32 * R], sbp[32 * R], zeta[32 * R], zs[32 * R], scale[32 * R];
    double mom[14][32 * R];                     // per-child moments (child frame)
    double w0[4][32 * R];                       // S-term weights of the origin term (level-independent)
    double amax[32 * R];                        // max(|V1|, |V2|) of each child
    double sv[7][32 * R];                       // contribution of a child that has become static
    float Ff[32 * R], cbpf[32 * R], sbpf[32 * R], zetaf[32 * R], zsf[32 * R], scalef[32 * R];   // FP32 bulk
};

// FP32 bulk evaluation of one edge node (mixed precision): s and e^s in
// FP64 (the node position along the edge, whose relative error is |s| times
// the unit roundoff), everything after it in FP32.  Adds the weighted,
// plane-frame contribution to this lane's partial sums (S, T).
EBEM_DI void edge_node_f32(float& S, float T[6], double s, float wq, float Fc, float cb, float sb, float z, float zs,
                           float scale, bool pterm, float k1, float t2, float k5, float k6) {
    const double ed = m_exp(s);
    const float e = (float)ed, ie = (float)(1.0 / ed);
    const float ch = 0.5f * (e + ie), sech = __fdividef(1.0f, ch), th = 0.5f * (e - ie) * sech;
    const float c = th * cb + sech * sb, sn = sech * cb - th * sb;
    const float R = Fc * ch, z2 = z * z;
    const float r = sqrtf(R * R + z2);
    const float q = __fdividef(1.0f, r * (r + R));
    const float ir = (r + R) * q, ir3 = ir * ir * ir;
    const float A1 = r, A3 = -ir, B2 = r + z2 * ir, D2 = -z2 * ir;
    const float B4 = -ir + z2 * ir3 * (1.0f / 3.0f), D4 = -z2 * ir3 * (1.0f / 3.0f);
    float C2 = 0.0f, C4 = 0.0f;
    if (z > 0.0f) {
        C2 = __logf(R + r) - R * ir;
        C4 = -(r * r + r * R + R * R) * ir3 * (r * q) * (1.0f / 3.0f);
    }
    float wsc, win, wmx, wzz;
    if (pterm) {
        wsc = k1 * A1 - t2 * A3;
        win = -k1 * B2 + 3.0f * t2 * B4;
        wmx = -k1 * C2 + 3.0f * t2 * C4;
        wzz = -k1 * D2 + 3.0f * t2 * D4;
    } else {
        wsc = k5 * A1;
        win = k6 * B2;
        wmx = k6 * C2;
        wzz = k6 * D2;
    }
    const float f = wq * sech * scale;
    const float fin = f * win, fmx = -zs * f * wmx;
    S += f * wsc;
    T[0] += fin * c * c;
    T[1] += fin * sn * c;
    T[2] += fin * sn * sn;
    T[3] += fmx * c;
    T[4] += fmx * sn;
    T[5] += f * wzz;
}

struct Piece { double slo, shi; int pterm; };

// Radial antiderivatives at the edge point R = F cosh s (one reciprocal for
// both 1/r and 1/(r + R)).
EBEM_DI Rad radial_edge(double R, double zeta) {
    Rad v;
    double z2 = zeta * zeta;
    double r = sqrt(R * R + z2);
    double q = 1.0 / (r * (r + R));
    double ir = (r + R) * q, ir3 = ir * ir * ir;
    v.A1 = r;
    v.A3 = -ir;
    v.B2 = r + z2 * ir;
    v.D2 = -z2 * ir;
    v.B4 = -ir + z2 * ir3 * (1.0 / 3.0);
    v.D4 = -z2 * ir3 * (1.0 / 3.0);
    if (zeta > 0) {
        v.C2 = m_log(R + r) - R * ir;
        v.C4 = -(r * r + r * R + R * R) * ir3 * (r * q) * (1.0 / 3.0);
    } else {
        v.C2 = 0.0;
        v.C4 = 0.0;
    }
    return v;
}

// cosh(s), sech(s), tanh(s) from one exponential.
EBEM_DI void hyp(double s, double& ch, double& sech, double& th) {
    double e = m_exp(s), ie = 1.0 / e;
    ch = 0.5 * (e + ie);
    sech = 1.0 / ch;
    th = 0.5 * (e - ie) * sech;
}

// sech s, tanh s and the radial antiderivatives at the edge point R = F cosh s
// (radial_edge) of one Gauss-Legendre node.  With EBEM_GL_ONEDIV (default;
// the sphere of 1280 triangles 161 -> 157 ms per step against hyp() and
// radial_edge(), which divide three times per node) the
// reciprocals of e^s, 1 + e^2s, r' and r' + F (1 + e^2s) (r' = 2 e^s r) come
// from one division: 1/e^s, 1/cosh, 1/(r (r + R)) and 1/r then cost
// multiplications, and log(R + r) = log(r' + F (1 + e^2s)) - s - log 2.
#ifndef EBEM_GL_ONEDIV
#define EBEM_GL_ONEDIV 1
#endif
EBEM_DI void edge_point(double s, double Fc, double zeta, double& sech, double& th, Rad& v) {
#if EBEM_GL_ONEDIV
    const double e = m_exp(s), e2 = e * e, u = e2 + 1.0;
    const double z2 = zeta * zeta, Fu = Fc * u;
    const double rp = sqrt(Fu * Fu + 4.0 * z2 * e2);          // 2 e^s r
    const double a = rp + Fu;                                 // 2 e^s (r + R)
    const double ue = u * e, ra = rp * a;
    const double inv = 1.0 / (ue * ra);
    const double iu = e * ra * inv, ie = u * ra * inv, irp = ue * a * inv, ia = ue * rp * inv;
    sech = 2.0 * e * iu;
    th = (e2 - 1.0) * iu;
    const double r = 0.5 * rp * ie, R = 0.5 * Fu * ie;
    const double ir = 2.0 * e * irp, ir3 = ir * ir * ir;
    v.A1 = r;
    v.A3 = -ir;
    v.B2 = r + z2 * ir;
    v.D2 = -z2 * ir;
    v.B4 = -ir + z2 * ir3 * (1.0 / 3.0);
    v.D4 = -z2 * ir3 * (1.0 / 3.0);
    if (zeta > 0) {
        v.C2 = m_log(a) - (s + 0.69314718055994530942) - Fu * irp;
        v.C4 = -(r * r + r * R + R * R) * ir3 * (2.0 * e * ia) * (1.0 / 3.0);
    } else {
        v.C2 = 0.0;
        v.C4 = 0.0;
    }
#else
    double ch;
    hyp(s, ch, sech, th);
    v = radial_edge(Fc * ch, zeta);
#endif
}

// Moments of one child (child frame), this lane's share of the nodes
// n = lane, lane + 32, ... of the whole-range rule: sub-pieces of length
// h <= EBEM_EDGE_H, 6, 8 or 10 Gauss-Legendre nodes each for h up to 1/4,
// 1/2 or 1 (glx, glw: the table of gl_table_entry).
EBEM_DI void moment_share(double m[14], double F, double cb, double sb, double zeta, double s1, double s0, int lane,
                          const double* glx, const double* glw) {
#pragma unroll
    for (int e = 0; e < 14; e++) m[e] = 0.0;
    double len = s0 - s1;
    if (!(len > 0)) return;
    int nsub = (int)ceil(len * (1.0 / EBEM_EDGE_H));
    nsub = max(1, min(nsub, 4096));
    double h = len / nsub;
    const int ng = (EBEM_GL_ADAPT && h <= 0.25) ? 6 : ((EBEM_GL_ADAPT && h <= 0.5) ? 8 : 10);
    const int base = ng == 6 ? 0 : (ng == 8 ? 6 : 14);
    for (int idx = lane; idx < nsub * ng; idx += 32) {
        int sub = idx / ng, q = idx - ng * sub;
        double s = s1 + (sub + 0.5) * h + 0.5 * h * glx[base + q];
        double sech, th;
        Rad v;
        edge_point(s, F, zeta, sech, th, v);
        double c = th * cb + sech * sb, sn = sech * cb - th * sb;
        double f = 0.5 * h * glw[base + q] * sech;
        double cc = c * c, sc = sn * c, ss = sn * sn;
        m[0] += f * v.A1;
        m[1] += f * v.A3;
        m[2] += f * v.B2 * cc; m[3] += f * v.B2 * sc; m[4] += f * v.B2 * ss;
        m[5] += f * v.B4 * cc; m[6] += f * v.B4 * sc; m[7] += f * v.B4 * ss;
        m[8] += f * v.C2 * c;  m[9] += f * v.C2 * sn;
        m[10] += f * v.C4 * c; m[11] += f * v.C4 * sn;
        m[12] += f * v.D2;     m[13] += f * v.D4;
    }
}

// Whole-range piece from the moments with the level's weights (child frame).
template <int R>
EBEM_DI void apply_moments(AccE& A, const WarpShared<R>& W, int slot, bool pterm, const LevelCtx& L, double zs) {
    double m[14];
#pragma unroll
    for (int e = 0; e < 14; e++) m[e] = W.mom[e][slot];
    double sc, i0, i1, i2, x0, x1, zz;
    if (pterm) {
        sc = L.k1 * m[0] - L.t2 * m[1];
        i0 = -L.k1 * m[2] + 3 * L.t2 * m[5];
        i1 = -L.k1 * m[3] + 3 * L.t2 * m[6];
        i2 = -L.k1 * m[4] + 3 * L.t2 * m[7];
        x0 = -L.k1 * m[8] + 3 * L.t2 * m[10];
        x1 = -L.k1 * m[9] + 3 * L.t2 * m[11];
        zz = -L.k1 * m[12] + 3 * L.t2 * m[13];
    } else {
        sc = L.k5 * m[0];
        i0 = L.k6 * m[2];
        i1 = L.k6 * m[3];
        i2 = L.k6 * m[4];
        x0 = L.k6 * m[8];
        x1 = L.k6 * m[9];
        zz = L.k6 * m[12];
    }
    A.S += sc;
    A.t11 += i0; A.t12 += i1; A.t22 += i2;
    A.t13 += -zs * x0; A.t23 += -zs * x1;
    A.t33 += zz;
}

EBEM_DI W4 neg(W4 w) { w.sc = -w.sc; w.in = -w.in; w.mx = -w.mx; w.zz = -w.zz; return w; }
EBEM_DI W4 wsub(W4 a, const W4& b) { a.sc -= b.sc; a.in -= b.in; a.mx -= b.mx; a.zz -= b.zz; return a; }

// S-term weights of the radial functions at the node's projection (rho = 0,
// r = zeta): level-independent, computed once per child.
EBEM_DI W4 origin_weights(double zeta, const LevelCtx& L) {
    Rad V0 = radial_at(0.0, zeta, zeta);
    if (!(zeta > 0)) { V0.A1 = 0.0; V0.B2 = 0.0; V0.D2 = 0.0; }
    return weigh(V0, false, L);
}

// Per-lane child state, level-independent.
struct LaneChild {
    ChildE g;
    double cg, sg;          // cos/sin of gamma
    double zeta, sigma, dMIN, w;
    bool live;
};

// Level data of one projected outer node, shared by its three children: the
// case (BEMenerg_coreSA_calcMatrixSubBlock.m:58-81), the in-plane front radii
// and the radial weights of the circle-bounded pieces: wPc (P terms between
// the S circle, or the projection, and the P circle), wPlo (minus the P terms
// at the lower limit) and wSc (P&S terms of the S circle minus the origin).
struct NodeLevel {
    W4 wPc, wPlo, wSc;
    double rhoP, rhoS;
    int type;
};

// Decision phase of one child at one level from its node's level data:
// closed-form circle pieces and lo-subtractions into A (child frame),
// whole-range pieces flagged in full_mask (the caller applies the moments),
// partial edge pieces returned in pc[0..np).  Mirrors child_level_e piece by
// piece.
#ifndef EBEM_NOINLINE_DECIDE
#define EBEM_NOINLINE_DECIDE 0     // 1: one out-of-line copy of the decision phase
#endif
#if EBEM_NOINLINE_DECIDE
static __device__ __noinline__
#else
EBEM_DI
#endif
void child_decide_n(AccE& A, Piece pc[3], int& np, int& full_mask, const ChildE& g, double cg, double sgm, double zs,
                    const NodeLevel& n, const W4& w0, double amax) {
    const int type = n.type;
    const double rhoP = n.rhoP, rhoS = n.rhoS;
    const bool isP = (type == T_P), spsp = (type == T_SP_SP);
    np = 0;
    full_mask = 0;                          // bit 0: full P piece, bit 1: full S piece
    double DeltaP = g.bm * g.bm - (g.a * g.a - rhoP * rhoP);
    double DeltaS = isP ? 0.0 : g.bm * g.bm - (g.a * g.a - rhoS * rhoS);
    const bool xP = DeltaP > 1.0e-6, xS = xP && DeltaS > 1.0e-6;
    const W4& wPc = n.wPc;
    const W4& wPlo = n.wPlo;
    const double smax = g.s0, smin = g.s1;
    const double th0 = 0.0, c0 = 1.0, sn0 = 0.0;
    const double thg = g.gamma;
    // S crossing data (used by the P pieces when the S front crosses, and by the S terms)
    double sS = 0.0, thAS = 0.0, cAS = 1.0, sAS = 0.0, thBS = 0.0, cBS = 1.0, sBS = 0.0;
    // a front whose radius reaches both edge ends covers the whole edge: both
    // crossings lie beyond the child (clipped to theta = 0 and gamma)
    if (xS && !isP) {
        if (rhoS >= amax) {
            sS = 1e300; thAS = 0.0; cAS = 1.0; sAS = 0.0; thBS = thg; cBS = cg; sBS = sgm;
        } else {
            front_cross(g, rhoS, smin, thg, cg, sgm, sS, thAS, cAS, sAS, thBS, cBS, sBS);
        }
    }
    if (!xP) {
        add_circle(A, wPc, th0, c0, sn0, thg, cg, sgm, zs);
    } else {
        double sP, thA, cA, sA, thB, cB, sB;
        if (rhoP >= amax) {
            sP = 1e300; thA = 0.0; cA = 1.0; sA = 0.0; thB = thg; cB = cg; sB = sgm;
        } else {
            front_cross(g, rhoP, smin, thg, cg, sgm, sP, thA, cA, sA, thB, cB, sB);
        }
        if (smax > sP) add_circle(A, wPc, th0, c0, sn0, thA, cA, sA, zs);
        if (-sP > smin) add_circle(A, wPc, thB, cB, sB, thg, cg, sgm, zs);
        if (xS && !isP) {
            // [sS, sP] <-> theta in [thA, thAS];  [-sP, -sS] <-> [thBS, thB]
            // (either may span the child's whole edge: edge on one side of
            // the foot of the perpendicular, between the fronts)
            double lo1 = fmax(sS, smin), hi1 = fmin(sP, smax);
            if (hi1 - lo1 > 0) {
                add_circle(A, wPlo, thA, cA, sA, thAS, cAS, sAS, zs);
                if (sS <= smin && sP >= smax) full_mask |= 1;
                else pc[np++] = {lo1, hi1, 1};
            }
            double lo2 = fmax(-sP, smin), hi2 = fmin(-sS, smax);
            if (hi2 - lo2 > 0) {
                add_circle(A, wPlo, thBS, cBS, sBS, thB, cB, sB, zs);
                if (-sP <= smin && -sS >= smax) full_mask |= 1;
                else pc[np++] = {lo2, hi2, 1};
            }
        } else {
            double lo = fmax(-sP, smin), hi = fmin(sP, smax);
            if (hi - lo > 0) {
                add_circle(A, wPlo, thA, cA, sA, thB, cB, sB, zs);
                if (-sP <= smin && sP >= smax) full_mask |= 1;
                else pc[np++] = {lo, hi, 1};
            }
        }
    }
    if (spsp) {
        // P&S terms, radial range [0, min(rhoS, R)]: V_S is VSe (not isP here)
        const W4& wSc = n.wSc;
        if (!xS) {
            add_circle(A, wSc, th0, c0, sn0, thg, cg, sgm, zs);
        } else {
            if (smax > sS) add_circle(A, wSc, th0, c0, sn0, thAS, cAS, sAS, zs);
            if (-sS > smin) add_circle(A, wSc, thBS, cBS, sBS, thg, cg, sgm, zs);
            double lo = fmax(-sS, smin), hi = fmin(sS, smax);
            if (hi - lo > 0) {
                add_circle(A, neg(w0), thAS, cAS, sAS, thBS, cBS, sBS, zs);
                if (-sS <= smin && sS >= smax) full_mask |= 2;
                else pc[np++] = {lo, hi, 0};
            }
        }
    }
}

// The same decision with the node's level data computed here (one child).
EBEM_DI void child_decide(AccE& A, Piece pc[3], int& np, int& full_mask, const LaneChild& C, const LevelCtx& L,
                          double rhoP, double rhoS, int type, const W4& w0, double amax) {
    NodeLevel n;
    n.type = type;
    n.rhoP = rhoP;
    n.rhoS = rhoS;
    const bool isP = (type == T_P);
    const double zeta = C.zeta;
    const double rhoSe = isP ? 0.0 : rhoS;
    Rad VSe = radial_at(rhoSe, isP ? zeta : L.RS, zeta);
    Rad VP = radial_at(rhoP, L.RP, zeta);
    n.wPc = weigh(rad_sub(VP, VSe), true, L);
    n.wPlo = neg(weigh(VSe, true, L));
    if (type == T_SP_SP) n.wSc = wsub(weigh(VSe, false, L), w0);
    child_decide_n(A, pc, np, full_mask, C.g, C.cg, C.sg, C.zeta * C.sigma, n, w0, amax);
}

// Child frame -> plane frame (rotation by the direction of V1), times the
// node weight and the orientation sign, added to (S, T[6]).
EBEM_DI void child_to_plane(double& S, double T[6], const AccE& A, const ChildE& g, double wsc) {
    const double c = g.ct, s = g.st;
    const double cc = c * c, ss = s * s, cs = c * s;
    S += wsc * A.S;
    T[0] += wsc * (cc * A.t11 - 2 * cs * A.t12 + ss * A.t22);
    T[1] += wsc * (cs * A.t11 + (cc - ss) * A.t12 - cs * A.t22);
    T[2] += wsc * (ss * A.t11 + 2 * cs * A.t12 + cc * A.t22);
    T[3] += wsc * (c * A.t13 - s * A.t23);
    T[4] += wsc * (s * A.t13 + c * A.t23);
    T[5] += wsc * A.t33;
}

EBEM_DI double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One halving step of a warp reduce-scatter: lanes with bit m of their index
// set keep the upper half of v[0..2h), the others the lower half; each adds
// its partner's copy of the half it keeps.
template <int M, int H>
EBEM_DI void rs_step(double* v, int lane) {
    const bool up = (lane & M) != 0;
#pragma unroll
    for (int k = 0; k < H; k++) {
        const double send = up ? v[k] : v[k + H];
        const double keep = up ? v[k + H] : v[k];
        v[k] = keep + __shfl_xor_sync(0xffffffffu, send, M);
    }
}

// Warp sums of 16 per-lane values with 15 shuffles: lane l returns the total
// of value scatter16_index(l).
EBEM_DI double warp_reduce_scatter16(double v[16], int lane) {
    rs_step<16, 8>(v, lane);
    rs_step<8, 4>(v, lane);
    rs_step<4, 2>(v, lane);
    rs_step<2, 1>(v, lane);
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}
EBEM_DI int scatter16_index(int lane) {
    return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}

// Warp sums of 8 per-lane values with 9 shuffles: lane l returns the total of
// value 4 b4 + 2 b3 + b2 (b = bits of l); scatter8_lane(e) holds value e.
EBEM_DI double warp_reduce_scatter8(double v[8], int lane) {
    rs_step<16, 4>(v, lane);
    rs_step<8, 2>(v, lane);
    rs_step<4, 1>(v, lane);
    double x = v[0];
    x += __shfl_xor_sync(0xffffffffu, x, 2);
    x += __shfl_xor_sync(0xffffffffu, x, 1);
    return x;
}
EBEM_DI int scatter8_lane(int e) { return ((e >> 2) & 1) << 4 | ((e >> 1) & 1) << 3 | (e & 1) << 2; }

EBEM_DI int warp_excl_scan(int v, int lane, int& total) {
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

}  // namespace ebem
