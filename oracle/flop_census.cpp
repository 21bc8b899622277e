// ORACLE — test infrastructure only.  FP64 operation census of the
// semi-analytic assembly, taken by compiling the oracle restatement with an
// operation-counting scalar (counted.hpp).
//
// For each sampled (source, field) pair the census evaluates, with the
// reference's formulas, the combined kernel integral F(t_k) at every time
// level k its non-null lags need (what a level-reusing assembly must
// compute), and separately the reference's own cost, three instants per
// non-null lag (SA/calcoloMatrice/BEMenerg_coreSA_calcMatrixSubBlock.m:26).
#include "counted.hpp"
namespace oracle_count { thread_local Tally tally; }
#define ORACLE_REAL oracle_count::CD
#include "sa_oracle.hpp"

#include <vector>
#include <cstdint>

using namespace oracle;

namespace {

struct TriC {
    real V[3][3];
    real vn[3];
    SdR S;
    M3 C;
    std::vector<real> nodes, w;
};

long long total(const oracle_count::Tally& t) { return t.add + t.mul + t.div + t.sqrt + t.trans; }

}  // namespace

extern "C" {

// out[0] flops over all needed levels, out[1] transcendental calls over
// those levels, out[2] number of (pair, level) evaluations, out[3] number of
// non-null pair-lags, out[4] flops of the reference's 3-instants-per-lag
// schedule.  Node tables (nodes: N x nGH x 3, w: N x nGH) and per-triangle
// data come from the caller so that the census matches the assembled mesh.
int or_flop_census(const double* coords, int nv, const int* tris, int nt,
                   const double* normal, const double* area, const double* center, const double* maxL,
                   double velP, double velS, double dt, int L, int nGH,
                   const double* bary, const double* wstd,
                   int npairs, const int* src, const int* fld, double* out) {
    std::vector<TriC> tc(nt);
    for (int t = 0; t < nt; t++) {
        for (int v = 0; v < 3; v++) for (int c = 0; c < 3; c++) tc[t].V[v][c] = coords[3 * tris[3 * t + v] + c];
        for (int c = 0; c < 3; c++) tc[t].vn[c] = normal[3 * t + c];
    }
    double flops = 0, trans = 0, nlev = 0, nlag = 0, fref = 0;
    for (int q = 0; q < npairs; q++) {
        int i = src[q], j = fld[q];
        TriC& F = tc[j];
        TriC& Sx = tc[i];
        // per-triangle constants (not counted: computed once per triangle)
        oracle_count::Tally saved = oracle_count::tally;
        F.S = calcoloSistemaRiferimento(F.V, F.vn);
        F.C = eulerMatrix(F.S, F.vn);
        Sx.nodes.assign(3 * nGH, real(0)); Sx.w.assign(nGH, real(0));
        for (int g = 0; g < nGH; g++) {
            for (int c = 0; c < 3; c++)
                Sx.nodes[3 * g + c] = real(bary[3 * g] * (double)Sx.V[0][c] + bary[3 * g + 1] * (double)Sx.V[1][c] + bary[3 * g + 2] * (double)Sx.V[2][c]);
            Sx.w[g] = real(area[i] * (2.0 * wstd[g]));
        }
        oracle_count::tally = saved;
        // non-null lag window (BEMenerg_coreSA_calcMatrixBlock.m:57-61)
        double v[3];
        for (int c = 0; c < 3; c++) v[c] = center[3 * j + c] - center[3 * i + c];
        double d = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        double dmin = d - maxL[j] - maxL[i], dmax = d + maxL[j] + maxL[i];
        int llo = -1, lhi = -2;
        for (int l = 0; l < L; l++)
            if (((l - 1) * velS * dt < dmax) && ((l + 1) * velP * dt >= dmin)) { if (llo < 0) llo = l; lhi = l; }
        if (llo < 0) continue;
        nlag += lhi - llo + 1;
        int klo = std::max(1, llo - 1), khi = lhi + 1;
        std::vector<double> cost(khi + 2, 0.0);
        for (int k = klo; k <= khi; k++) {
            oracle_count::Tally before = oracle_count::tally;
            real currT = real(k * dt);
            real rP = real(velP) * currT, rS = real(velS) * currT;
            M3 r[7];
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
                for (int kk = 1; kk <= 6; kk++) r[kk] = r[kk] + t.r[kk] * Sx.w[g];
            }
            M3 rist = combine(r, real(velP), real(velS), currT);
            (void)rist;
            oracle_count::Tally after = oracle_count::tally;
            double c = (double)(total(after) - total(before));
            flops += c;
            trans += (double)(after.trans - before.trans);
            nlev += 1;
            cost[k] = c;
        }
        for (int l = llo; l <= lhi; l++)
            for (int k = l - 1; k <= l + 1; k++) if (k >= 1) fref += cost[k] + 9 * 2;   // + the 1,-2,1 accumulation
    }
    out[0] = flops; out[1] = trans; out[2] = nlev; out[3] = nlag; out[4] = fref;
    return 0;
}

}  // extern "C"
