// Semi-analytic assembly in two passes: the combined kernel integral F(t_k)
// of every (pair, level), then the energetic second difference written as
// dense blocks.
//
// The value is the reference's (BEMenerg_coreSA_calcMatrixSubBlock.m:1-111
// with the child integrals of BEMenerg_coreSA_calcIntgInt_childTriangle.m,
// evaluated in the edge-variable form of sa_edge.cuh, the same per-child
// arithmetic as sa_assemble_warp_kernel: child_decide_n, the whole-edge
// moments and the Gauss-Legendre nodes of the partial edge pieces); the null
// test and clean-up are those of BEMenerg_coreSA_calcMatrixBlock.m:57-61,77.
//
// Pass 1, sa_level_kernel: one warp per (source, field) pair.  The work of a
// pair is the set of items (outer node g, level k) over the pair's levels,
// taken level-major in rounds of 32: every lane of a round owns one item.  A
// lane computes its node's level data once (case, front radii, radial
// weights; node_level) and then decides the node's three children in turn,
// so all 32 lanes work and the node-level transcendentals are shared by the
// three children (the one-warp-per-pair kernel gives a lane one child at one
// level: 21 of 32 lanes busy for the 7-node rule, the node work done three
// times).  Per round:
//   * the lanes' closed-form contributions (plane frame) are summed per level
//     by a segmented warp scan (the items of a level are adjacent lanes);
//   * the lanes stage their partial edge pieces in shared memory; the
//     Gauss-Legendre nodes of each level's pieces are evaluated by all 32
//     lanes and reduced;
//   * levels whose items are all done are finished by one lane each: static
//     children added (a child lying inside the S front with its whole edge
//     contributes a level-independent value, computed once at its first such
//     level), rotation to global axes with the field triangle's Euler matrix,
//     F_k (6 symmetric entries) stored.
// Items are numbered from the pair's first non-null level over all lags, so
// the rounds, and with them every sum, are the same whatever lag window is
// requested: results do not depend on the window, and there are no atomics.
//
// Pass 2, sa_emit_kernel: E_l = (F_{l+1} - 2 F_l + F_{l-1}) / (4 pi rho) for
// every (source, field, lag) of the window, zero outside the pair's band,
// clean-up |x| < 1e-14 -> 0, written (or added) column by column: one thread
// per output entry, consecutive threads consecutive rows, so the 4.7 GB of the
// 1280-triangle sphere are written in full sectors.
//
// The F buffer holds (field columns of a chunk) x (levels) x (sources) x 6
// doubles; the columns are processed in chunks that keep it within a budget.
#include "ebem_internal.h"

#include <climits>
#include "sa_pair.cuh"
#include "sa_warp.cuh"

namespace ebem {

namespace {

constexpr int kRing = 16;              // level accumulators in flight per warp
constexpr int kLanePieces = 9;         // partial edge pieces per item: 3 children x 3

// Per-warp shared state for NG outer nodes (3 NG children).
template <int NG>
struct LvlShared {
    static constexpr int NC = 3 * NG;
    ChildE g[NC];
    double cg[NC], sg[NC];
    double cbp[NC], sbp[NC], scale[NC];         // plane-frame data of the edge nodes
    double zeta[NG], zs[NG], dmin[NG];
    double w0[4][NG];
    double mom[14][NC];                         // whole-edge moments (child frame)
    double sv[7][NC];                           // value of a static child (plane frame)
    double acc[kRing][7];                       // per-level sums (plane frame)
    double pslo[32 * kLanePieces], ph[32 * kLanePieces];
    int pinfo[32 * kLanePieces];                // slot | pterm << 6 | nsub << 7
    int pcnt[32];
    int noff[33];                               // Gauss-Legendre node offsets per lane
    int kstat[NC];                              // first static level (INT_MAX: none yet)
    unsigned long long hasmom;                  // bit per child slot
    float Ff[NC], cbpf[NC], sbpf[NC], zetaf[NC], zsf[NC], scalef[NC];   // FP32 copies (mixed precision)
};

struct LvlArgs {
    const TriGeom* geo;
    const NodeW* nodes;
    int N, n_gh;
    double velP, velS, dt;
    int lag0, nlag;
    int src0, nsrc;             // source rows of the panel
    int j0, nj;                 // field columns of this chunk
    int kbase, KL;              // levels [kbase, kbase + KL) held in F
    double* F;                  // ((jj KL + k - kbase) nsrc + ii) x 6
    int2* band;                 // (jj nsrc + ii): non-null lags (llo, lhi) in the window, llo = -1 if none
    unsigned long long* count;
};

// First lag >= 0 that passes the null test (-1: none); independent of any
// lag window, so the item numbering of a pair is too.
__device__ __forceinline__ int first_nonnull_lag(double velP, double velS, double dt, double distMin, double distMax) {
    for (int l = 0; l < (1 << 20); l++) {
        if (lag_nonnull(l, velP, velS, dt, distMin, distMax)) return l;
        if ((l - 1) * velS * dt >= distMax) return -1;
    }
    return -1;
}

__device__ __forceinline__ void apply_mom(AccE& A, const double* m, int stride, bool pterm, const LevelCtx& L,
                                          double zs) {
    double sc, i0, i1, i2, x0, x1, zz;
    if (pterm) {
        sc = L.k1 * m[0] - L.t2 * m[stride];
        i0 = -L.k1 * m[2 * stride] + 3 * L.t2 * m[5 * stride];
        i1 = -L.k1 * m[3 * stride] + 3 * L.t2 * m[6 * stride];
        i2 = -L.k1 * m[4 * stride] + 3 * L.t2 * m[7 * stride];
        x0 = -L.k1 * m[8 * stride] + 3 * L.t2 * m[10 * stride];
        x1 = -L.k1 * m[9 * stride] + 3 * L.t2 * m[11 * stride];
        zz = -L.k1 * m[12 * stride] + 3 * L.t2 * m[13 * stride];
    } else {
        sc = L.k5 * m[0];
        i0 = L.k6 * m[2 * stride];
        i1 = L.k6 * m[3 * stride];
        i2 = L.k6 * m[4 * stride];
        x0 = L.k6 * m[8 * stride];
        x1 = L.k6 * m[9 * stride];
        zz = L.k6 * m[12 * stride];
    }
    A.S += sc;
    A.t11 += i0; A.t12 += i1; A.t22 += i2;
    A.t13 += -zs * x0; A.t23 += -zs * x1;
    A.t33 += zz;
}

__device__ __forceinline__ LevelCtx level_ctx(int k, double dt, double velP, double velS) {
    const double t = k * dt;
    const double vp2 = velP * velP, vs2 = velS * velS, den = vp2 * vs2;
    LevelCtx L;
    L.t2 = t * t;
    L.RP = velP * t;
    L.RS = velS * t;
    L.k1 = 1.0 / vp2;
    L.k5 = (vp2 + vs2) / den;
    L.k6 = (vp2 - vs2) / den;
    return L;
}

// Segmented inclusive sum over lanes with equal key (adjacent lanes).
__device__ __forceinline__ double seg_sum(double v, int key, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, v, o);
        const int ky = __shfl_up_sync(0xffffffffu, key, o);
        if (lane >= o && ky == key) v += y;
    }
    return v;
}

}  // namespace

template <int NG, bool MIXED>
__device__ __forceinline__ void level_pair(const LvlArgs& A, LvlShared<NG>& W, const double* glx, const double* glw,
                                           int ii, int jj, int lane) {
    constexpr int NC = 3 * NG;
    const int i = A.src0 + ii, j = A.j0 + jj;
    const TriGeom& F = A.geo[j];
    const TriGeom& Sg = A.geo[i];
    const long long rec = (long long)jj * A.nsrc + ii;
    int llo = -1, lhi = -2;
    pair_band(F, Sg, A.velP, A.velS, A.dt, A.lag0, A.nlag, &llo, &lhi);
    if (lane == 0) {
        A.band[rec] = make_int2(llo, lhi);
        if (A.count && llo >= 0) atomicAdd(A.count, (unsigned long long)(lhi - llo + 1));
    }
    if (llo < 0) return;
    // levels to compute, and the pair's item origin
    const int kp_lo = max(1, llo - 1), kp_hi = lhi + 1;
    int kref;
    {
        const double v0 = F.ctr[0] - Sg.ctr[0], v1 = F.ctr[1] - Sg.ctr[1], v2 = F.ctr[2] - Sg.ctr[2];
        const double d = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        const int lf = first_nonnull_lag(A.velP, A.velS, A.dt, d - F.maxL - Sg.maxL, d + F.maxL + Sg.maxL);
        kref = max(1, (lf < 0 ? llo : lf) - 1);
        if (kref > kp_lo) kref = kp_lo;
    }
    // child geometry (level-independent), one child per lane and pass
    for (int slot = lane; slot < NC; slot += 32) {
        const int g = slot / 3, c = slot - 3 * g;
        const NodeW sp = A.nodes[(size_t)i * NG + g];
        NodeGeo G;
        node_geo(G, sp, F);
        ChildE cg = {};                       // sgnC = 0 marks a skipped (degenerate) child
        const bool live = node_child_e(cg, G, c);
        double sgm = 0.0, cgm = 1.0;
        if (live) m_sincos(cg.gamma, &sgm, &cgm);
        W.g[slot] = cg;
        W.cg[slot] = cgm;
        W.sg[slot] = sgm;
        W.kstat[slot] = INT_MAX;
        if (live) {
            W.cbp[slot] = cg.cb * cg.ct + cg.sb * cg.st;     // cos(beta - theta_V1)
            W.sbp[slot] = cg.sb * cg.ct - cg.cb * cg.st;     // sin(beta - theta_V1)
            W.scale[slot] = sp.w * cg.sgnC;
            if (MIXED) {
                W.Ff[slot] = (float)cg.F;
                W.cbpf[slot] = (float)W.cbp[slot];
                W.sbpf[slot] = (float)W.sbp[slot];
                W.zetaf[slot] = (float)G.zeta;
                W.zsf[slot] = (float)(G.zeta * G.sigma);
                W.scalef[slot] = (float)W.scale[slot];
            }
        }
        if (c == 0) {
            W.zeta[g] = G.zeta;
            W.zs[g] = G.zeta * G.sigma;
            W.dmin[g] = G.dMIN;
            LevelCtx L0;
            L0.k5 = (A.velP * A.velP + A.velS * A.velS) / ((A.velP * A.velS) * (A.velP * A.velS));
            L0.k6 = (A.velP * A.velP - A.velS * A.velS) / ((A.velP * A.velS) * (A.velP * A.velS));
            const W4 w0 = origin_weights(G.zeta, L0);
            W.w0[0][g] = w0.sc;
            W.w0[1][g] = w0.in;
            W.w0[2][g] = w0.mx;
            W.w0[3][g] = w0.zz;
        }
    }
    if (lane == 0) W.hasmom = 0ull;
    for (int e = lane; e < kRing * 7; e += 32) (&W.acc[0][0])[e] = 0.0;
    __syncwarp();
    const long long q_lo = (long long)(kp_lo - kref) * NG, q_hi = (long long)(kp_hi - kref) * NG + NG - 1;
    int kfin = kp_lo;                     // next level to finish
    for (long long r0 = (q_lo / 32) * 32; r0 <= q_hi; r0 += 32) {
        const long long q = r0 + lane;
        const int k = kref + (int)(q / NG), g = (int)(q % NG);
        const bool act = q >= q_lo && q <= q_hi;
        // node level data at k (and the case at k - 1 for the static test)
        const LevelCtx L = level_ctx(k, A.dt, A.velP, A.velS);
        NodeLevel n;
        n.type = T_NONE;
        n.rhoP = -1.0;
        n.rhoS = -1.0;
        NodeLevel nm1;
        nm1.type = T_NONE;
        nm1.rhoP = -1.0;
        nm1.rhoS = -1.0;
        W4 w0;
        w0.sc = w0.in = w0.mx = w0.zz = 0.0;
        double zsn = 0.0;
        if (act) {
            w0.sc = W.w0[0][g];
            w0.in = W.w0[1][g];
            w0.mx = W.w0[2][g];
            w0.zz = W.w0[3][g];
            zsn = W.zs[g];
            node_level(n, W.zeta[g], W.dmin[g], L, w0);
            if (k > kp_lo) {
                const LevelCtx Lm = level_ctx(k - 1, A.dt, A.velP, A.velS);
                nm1.type = classify(W.zeta[g], Lm.RP, Lm.RS, W.dmin[g], nm1.rhoP, nm1.rhoS);
            }
        }
        double S = 0.0, T[6] = {0, 0, 0, 0, 0, 0};
        int npl = 0, nnodes = 0;
#pragma unroll 1
        for (int c = 0; c < 3; c++) {
            const int slot = 3 * g + c;
            const ChildE& cgeo = W.g[act ? slot : 0];
            const bool live = act && cgeo.sgnC != 0.0;
            bool stat_k = false, stat_m1 = false;
            if (live && n.type == T_SP_SP) {
                stat_k = child_static(cgeo, n);
                stat_m1 = stat_k && k > kp_lo && child_static(cgeo, nm1);
            }
            AccE Ac = {0, 0, 0, 0, 0, 0, 0};
            Piece pc[3];
            int np = 0, full = 0;
            const bool work = live && n.type != T_NONE && !stat_m1;
            if (work) {
                const ChildE gc = cgeo;
                child_decide_n(Ac, pc, np, full, gc, W.cg[slot], W.sg[slot], zsn, n, w0, gc.amax);
            }
            // whole-edge moments, computed by the whole warp once per child
            const bool need = work && full && !((W.hasmom >> slot) & 1ull);
            unsigned mm = __ballot_sync(0xffffffffu, need);
            while (mm) {
                const int b = __ffs(mm) - 1;
                mm &= mm - 1;
                const int sb = __shfl_sync(0xffffffffu, slot, b);
                if ((W.hasmom >> sb) & 1ull) continue;           // another lane's item did this child
                const ChildE& gb = W.g[sb];
                double m[16];
                moment_share(m, gb.F, gb.cb, gb.sb, W.zeta[sb / 3], gb.s1, gb.s0, lane, glx, glw);
                m[14] = 0.0;
                m[15] = 0.0;
                const double tot = warp_reduce_scatter16(m, lane);
                const int e = scatter16_index(lane);
                if (!(lane & 1) && e < 14) W.mom[e][sb] = tot;
                __syncwarp();
                if (lane == 0) W.hasmom |= 1ull << sb;
                __syncwarp();
            }
            if (work) {
                if (full & 1) apply_mom(Ac, &W.mom[0][slot], NC, true, L, zsn);
                if (full & 2) apply_mom(Ac, &W.mom[0][slot], NC, false, L, zsn);
                double Sc = 0.0, Tc[6] = {0, 0, 0, 0, 0, 0};
                const ChildE gc = cgeo;
                child_to_plane(Sc, Tc, Ac, gc, W.scale[slot]);
                S += Sc;
#pragma unroll
                for (int e = 0; e < 6; e++) T[e] += Tc[e];
                if (stat_k) {                                      // first static level of this child
                    W.sv[0][slot] = Sc;
#pragma unroll
                    for (int e = 0; e < 6; e++) W.sv[1 + e][slot] = Tc[e];
                    W.kstat[slot] = k;
                }
                // stage the partial edge pieces of this item
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    if (t < np) {
                        const double len = pc[t].shi - pc[t].slo;
                        int ns = (int)ceil(len * (1.0 / EBEM_EDGE_H));
                        ns = max(1, min(ns, 4096));
                        const int at = lane * kLanePieces + npl;
                        W.pslo[at] = pc[t].slo;
                        W.ph[at] = len / ns;
                        W.pinfo[at] = slot | (pc[t].pterm ? 64 : 0) | (ns << 7);
                        npl++;
                        nnodes += 10 * ns;
                    }
                }
            }
        }
        // per-level sums of the closed-form parts: segmented over adjacent lanes
        const int key = act ? k : INT_MIN + lane;
        const int knext = __shfl_down_sync(0xffffffffu, key, 1);
        const bool seg_end = act && (lane == 31 || knext != key);
        {
            double v[7] = {S, T[0], T[1], T[2], T[3], T[4], T[5]};
#pragma unroll
            for (int e = 0; e < 7; e++) v[e] = seg_sum(v[e], key, lane);
            if (seg_end) {
                double* a = W.acc[k & (kRing - 1)];
#pragma unroll
                for (int e = 0; e < 7; e++) a[e] += v[e];
            }
        }
        // Gauss-Legendre nodes of the staged pieces, level by level
        W.pcnt[lane] = npl;
        int tot = 0;
        const int off = warp_excl_scan(nnodes, lane, tot);
        W.noff[lane] = off;
        if (lane == 31) W.noff[32] = tot;
        __syncwarp();
        const int k_first = __shfl_sync(0xffffffffu, act ? k : INT_MAX, __ffs(__ballot_sync(0xffffffffu, act)) - 1);
        const int k_last = kref + (int)(min(q_hi, r0 + 31) / NG);
        for (int kk = k_first; kk <= k_last; kk++) {
            // lanes [la, lb) hold level kk's items
            const unsigned in_k = __ballot_sync(0xffffffffu, act && k == kk);
            if (!in_k) continue;
            const int la = __ffs(in_k) - 1, lb = 32 - __clz(in_k);
            const int n0 = W.noff[la], n1 = W.noff[lb];
            double Sl = 0.0, Tl[6] = {0, 0, 0, 0, 0, 0};
            const LevelCtx Lk = level_ctx(kk, A.dt, A.velP, A.velS);
            if (n1 > n0) {
                int own = la, t = 0, base = n0;         // cursor: owner lane, its piece, first node of the piece
                float Sf = 0.0f, Tf[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                for (int idx = n0 + lane; idx < n1; idx += 32) {
                    int info = 0;
                    while (own < lb) {                  // bounded: the level's nodes lie in lanes [la, lb)
                        if (t >= W.pcnt[own]) { own++; t = 0; continue; }
                        info = W.pinfo[own * kLanePieces + t];
                        const int cnt = 10 * (info >> 7);
                        if (idx < base + cnt) break;
                        base += cnt;
                        t++;
                    }
                    if (own >= lb) break;
                    const int u = idx - base, sub = u / 10, qn = u - 10 * sub;
                    const double h = W.ph[own * kLanePieces + t];
                    const double s = W.pslo[own * kLanePieces + t] + (sub + 0.5) * h + 0.5 * h * glx[qn];
                    const int cl = info & 63;
                    const bool pterm = (info & 64) != 0;
                    if (MIXED) {
                        edge_node_f32(Sf, Tf, s, (float)(0.5 * h * glw[qn]), W.Ff[cl], W.cbpf[cl], W.sbpf[cl],
                                      W.zetaf[cl], W.zsf[cl], W.scalef[cl], pterm, (float)Lk.k1, (float)Lk.t2,
                                      (float)Lk.k5, (float)Lk.k6);
                    } else {
                        double ch, sech, th;
                        hyp(s, ch, sech, th);
                        const double cbq = W.cbp[cl], sbq = W.sbp[cl];
                        const double cq = th * cbq + sech * sbq, sq = sech * cbq - th * sbq;
                        const double zc = W.zeta[cl / 3];
                        Rad v = radial_edge(W.g[cl].F * ch, zc);
                        W4 w = weigh(v, pterm, Lk);
                        const double f = 0.5 * h * glw[qn] * sech * W.scale[cl];
                        const double fin = f * w.in, fmx = -W.zs[cl / 3] * f * w.mx;
                        Sl += f * w.sc;
                        Tl[0] += fin * cq * cq;
                        Tl[1] += fin * sq * cq;
                        Tl[2] += fin * sq * sq;
                        Tl[3] += fmx * cq;
                        Tl[4] += fmx * sq;
                        Tl[5] += f * w.zz;
                    }
                }
                if (MIXED) {
                    Sl += (double)Sf;
#pragma unroll
                    for (int e = 0; e < 6; e++) Tl[e] += (double)Tf[e];
                }
                double v[8] = {Sl, Tl[0], Tl[1], Tl[2], Tl[3], Tl[4], Tl[5], 0.0};
                const double sum = warp_reduce_scatter8(v, lane);
                // lane scatter8_lane(e) holds the sum of value e
#pragma unroll
                for (int e = 0; e < 7; e++)
                    if (lane == scatter8_lane(e)) W.acc[kk & (kRing - 1)][e] += sum;
            }
            __syncwarp();
        }
        // finish the levels whose items are all done
        const int kdone = kref + (int)((min(q_hi, r0 + 31) + 1) / NG) - 1;     // last level with all items done
        const int kend = (r0 + 31 >= q_hi) ? kp_hi : min(kdone, kp_hi);
        __syncwarp();
        const int kf = kfin + lane;
        if (kf <= kend) {
            double* a = W.acc[kf & (kRing - 1)];
            double Sv = a[0], Tv[6] = {a[1], a[2], a[3], a[4], a[5], a[6]};
            for (int slot = 0; slot < NC; slot++) {
                if (W.kstat[slot] < kf) {
                    Sv += W.sv[0][slot];
#pragma unroll
                    for (int e = 0; e < 6; e++) Tv[e] += W.sv[1 + e][slot];
                }
            }
            // F(t_k) = (S I + C^T M C) / 2 in global axes
            const double M[3][3] = {{Tv[0], Tv[1], Tv[3]}, {Tv[1], Tv[2], Tv[4]}, {Tv[3], Tv[4], Tv[5]}};
            const double* Cm = F.C;
            double MC[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int cc = 0; cc < 3; cc++) MC[r][cc] = M[r][0] * Cm[cc] + M[r][1] * Cm[3 + cc] + M[r][2] * Cm[6 + cc];
            double Rm[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int cc = r; cc < 3; cc++)
                    Rm[r][cc] = Cm[r] * MC[0][cc] + Cm[3 + r] * MC[1][cc] + Cm[6 + r] * MC[2][cc];
            double* dst = A.F + (((long long)jj * A.KL + (kf - A.kbase)) * A.nsrc + ii) * 6;
            dst[0] = 0.5 * (Sv + Rm[0][0]);
            dst[1] = 0.5 * Rm[0][1];
            dst[2] = 0.5 * Rm[0][2];
            dst[3] = 0.5 * (Sv + Rm[1][1]);
            dst[4] = 0.5 * Rm[1][2];
            dst[5] = 0.5 * (Sv + Rm[2][2]);
#pragma unroll
            for (int e = 0; e < 7; e++) a[e] = 0.0;
        }
        kfin = max(kfin, kend + 1);
        __syncwarp();
    }
}

#ifndef EBEM_LVL_WPB
#define EBEM_LVL_WPB 4     // warps per block
#endif
#ifndef EBEM_LVL_MINB
#define EBEM_LVL_MINB 2    // blocks per SM the register allocation aims at (2: 240 registers, no spills)
#endif

template <int NG, bool MIXED>
__global__ void __launch_bounds__(32 * EBEM_LVL_WPB, EBEM_LVL_MINB) sa_level_kernel(LvlArgs A) {
    extern __shared__ __align__(16) unsigned char lvl_smem[];
    __shared__ double glx[10], glw[10];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    LvlShared<NG>& W = reinterpret_cast<LvlShared<NG>*>(lvl_smem)[wib];
    if (threadIdx.x < 10) {
        const int k = threadIdx.x < 5 ? threadIdx.x : threadIdx.x - 5;
        glx[threadIdx.x] = (threadIdx.x < 5 ? -1.0 : 1.0) * gl_x(k);
        glw[threadIdx.x] = gl_w(k);
    }
    __syncthreads();
    const long long NP = (long long)A.nj * A.nsrc;
    const long long nwarps = (long long)gridDim.x * EBEM_LVL_WPB;
    for (long long p = (long long)blockIdx.x * EBEM_LVL_WPB + wib; p < NP; p += nwarps)
        level_pair<NG, MIXED>(A, W, glx, glw, (int)(p % A.nsrc), (int)(p / A.nsrc), lane);
}

// E_l of the window from F, one thread per entry of a column.
__global__ void __launch_bounds__(256) sa_emit_kernel(const double* __restrict__ Fb, const int2* __restrict__ band,
                                                      int nsrc, int j0, int nj, int kbase, int KL, int lag0, int nlag,
                                                      double c4, double* __restrict__ E, size_t ld, size_t ld_lag,
                                                      int accumulate) {
    const long long rows = 3LL * nsrc;
    const long long r3 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r3 >= rows) return;
    const int col = blockIdx.y;                   // 3 jj + c
    const int jj = col / 3, c = col - 3 * jj;
    const int q = blockIdx.z, l = lag0 + q;
    const int ii = (int)(r3 / 3), r = (int)(r3 - 3LL * ii);
    const int2 b = band[(long long)jj * nsrc + ii];
    double v = 0.0;
    if (b.x >= 0 && l >= b.x && l <= b.y) {
        const int e = (r == 0) ? c : (c == 0 ? r : r + c + 1);        // (r, c) -> 11,12,13,22,23,33
        const double* f = Fb + ((long long)jj * KL * nsrc + ii) * 6 + e;
        const long long ks = (long long)nsrc * 6;                       // one level
        const double fk1 = f[(l + 1 - kbase) * ks];
        const double fk = (l >= 1) ? f[(l - kbase) * ks] : 0.0;            // F_0 = 0
        const double fkm = (l - 1 >= 1) ? f[(l - 1 - kbase) * ks] : 0.0;
        v = ((fk1 + (-2.0) * fk) + fkm) / c4;
        if (fabs(v) < 1.0e-14) v = 0.0;
    }
    double* dst = E + (size_t)q * ld_lag + (3 * (size_t)(j0 + jj) + c) * ld + (size_t)r3;
    if (accumulate) *dst += v;
    else *dst = v;
}

template <int NG, bool MIXED>
static int launch_levels_t(const LvlArgs& A, int device, cudaStream_t s) {
    const size_t shmem = sizeof(LvlShared<NG>) * EBEM_LVL_WPB;
    static bool attr_set[64] = {};
    if (device >= 0 && device < 64 && !attr_set[device]) {
        EBEM_CUDA_TRY(cudaFuncSetAttribute(sa_level_kernel<NG, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)shmem));
        attr_set[device] = true;
    }
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    EBEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sa_level_kernel<NG, MIXED>,
                                                                32 * EBEM_LVL_WPB, shmem));
    if (per_sm < 1) return fail(EBEM_ERR_INVALID, "level kernel does not fit on an SM");
    const long long NP = (long long)A.nj * A.nsrc;
    long long want = (NP + EBEM_LVL_WPB - 1) / EBEM_LVL_WPB;
    const long long cap = (long long)sms * per_sm * 8;
    const unsigned blocks = (unsigned)std::max<long long>(1, std::min(want, cap));
    sa_level_kernel<NG, MIXED><<<blocks, 32 * EBEM_LVL_WPB, shmem, s>>>(A);
    EBEM_CUDA_TRY(cudaGetLastError());
    return EBEM_OK;
}

int launch_sa_levels(const MeshData& m, const PhysParams& P, int n_gh, int lag0, int nlag, int src0, int nsrc,
                     double* d_E, size_t ld, size_t ld_lag, int accumulate, unsigned long long* d_count, int mixed,
                     cudaStream_t s) {
    if (n_gh != 3 && n_gh != 7 && n_gh != 12 && n_gh != 19)
        return fail(EBEM_ERR_INVALID, "outer rule must have 3, 7, 12 or 19 nodes");
    const int kbase = std::max(1, lag0 - 1);
    const int KL = lag0 + nlag + 1 - kbase;           // levels kbase .. lag0 + nlag
    const size_t per_col = (size_t)KL * nsrc * 6 * sizeof(double) + (size_t)nsrc * sizeof(int2);
    if (3LL * m.nt > 65535 || nlag > 65535) return fail(EBEM_ERR_INVALID, "mesh or lag window too large for one launch");
    // within what the workspace pool keeps reserved between calls, so that a
    // repeated call maps no new memory; equal chunks of field columns
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t budget = std::max<size_t>((size_t)64 << 20, std::min<size_t>(free_b / 4, (size_t)3 << 29));
    const int most = (int)std::max<size_t>(1, std::min<size_t>((size_t)m.nt, budget / per_col));
    const int chunks = (m.nt + most - 1) / most;
    const int cols = (m.nt + chunks - 1) / chunks;
    double* Fb = nullptr;
    if (ws_malloc(&Fb, per_col * cols, s) != cudaSuccess)
        return fail(EBEM_ERR_NOMEM, "assembly workspace allocation failed");
    int2* band = reinterpret_cast<int2*>(reinterpret_cast<unsigned char*>(Fb) + (size_t)KL * nsrc * 6 * sizeof(double) * cols);
    int rc = EBEM_OK;
    for (int j0 = 0; j0 < m.nt && rc == EBEM_OK; j0 += cols) {
        LvlArgs A;
        A.geo = m.d_geo;
        A.nodes = m.d_nodes;
        A.N = m.nt;
        A.n_gh = n_gh;
        A.velP = P.velP;
        A.velS = P.velS;
        A.dt = P.dt;
        A.lag0 = lag0;
        A.nlag = nlag;
        A.src0 = src0;
        A.nsrc = nsrc;
        A.j0 = j0;
        A.nj = std::min(cols, m.nt - j0);
        A.kbase = kbase;
        A.KL = KL;
        A.F = Fb;
        A.band = band;
        A.count = d_count;
        switch (n_gh) {
            case 3: rc = mixed ? launch_levels_t<3, true>(A, m.device, s) : launch_levels_t<3, false>(A, m.device, s); break;
            case 7: rc = mixed ? launch_levels_t<7, true>(A, m.device, s) : launch_levels_t<7, false>(A, m.device, s); break;
            case 12: rc = mixed ? launch_levels_t<12, true>(A, m.device, s) : launch_levels_t<12, false>(A, m.device, s); break;
            default: rc = mixed ? launch_levels_t<19, true>(A, m.device, s) : launch_levels_t<19, false>(A, m.device, s); break;
        }
        if (rc) break;
        const long long rows = 3LL * nsrc;
        dim3 grid((unsigned)((rows + 255) / 256), (unsigned)(3 * A.nj), (unsigned)nlag);
        sa_emit_kernel<<<grid, 256, 0, s>>>(Fb, band, nsrc, j0, A.nj, kbase, KL, lag0, nlag, 4 * kPi * P.rho, d_E, ld,
                                            ld_lag, accumulate);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(EBEM_ERR_CUDA, std::string("emission kernel: ") + cudaGetErrorString(e));
    }
    ws_free(Fb, s);
    return rc;
}

}  // namespace ebem
