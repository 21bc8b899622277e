// Gauss-Hammer triangle rules (host code).
//
// The node/weight values are the literal constants of the reference's
// f/utility/quadRules/GaussHammer_base.m:19-409 (a quadrature table is data
// that must be identical for parity; the 7-point values carry 13 digits
// there and so do they here).  They are encoded as symmetry orbits:
//   S3   the centroid,
//   S21  (a, b, b) and its two rotations, b = given or (1 - a)/2,
//   S111 the six permutations of (a, b, 1 - a - b),
// emitted in the reference's node order.  The composite rule follows
// f/utility/quadRules/GaussHammerComposite.m:1-55: n_sub congruent
// sub-triangles visited row by row, weights scaled by 2/n_sub.
#include "ebem_internal.h"

#include <cmath>

namespace ebem {
namespace {

enum OrbitKind { S3, S21, S21H, S111 };   // S21H: b = (1 - a)/2
struct Orbit { OrbitKind kind; double a, b, w; };

int emit(const Orbit* orb, int norb, double bary[][3], double w[]) {
    int n = 0;
    for (int k = 0; k < norb; k++) {
        const Orbit& o = orb[k];
        if (o.kind == S3) {
            bary[n][0] = bary[n][1] = bary[n][2] = 1.0 / 3; w[n++] = o.w;
        } else if (o.kind == S21 || o.kind == S21H) {
            double a = o.a, b = (o.kind == S21H) ? (1 - o.a) / 2 : o.b;
            double t[3][3] = {{a, b, b}, {b, a, b}, {b, b, a}};
            for (int r = 0; r < 3; r++) { for (int c = 0; c < 3; c++) bary[n][c] = t[r][c]; w[n++] = o.w; }
        } else {
            double a = o.a, b = o.b, c3 = 1 - a - b;
            double t[6][3] = {{a, b, c3}, {a, c3, b}, {b, a, c3}, {b, c3, a}, {c3, a, b}, {c3, b, a}};
            for (int r = 0; r < 6; r++) { for (int c = 0; c < 3; c++) bary[n][c] = t[r][c]; w[n++] = o.w; }
        }
    }
    return n;
}

}  // namespace

int gh_base(int n, double bary[][3], double w[]) {
    switch (n) {
    case 1: {
        const Orbit o[] = {{S3, 0, 0, 0.5}};
        return emit(o, 1, bary, w);
    }
    case 3: {
        const Orbit o[] = {{S21, 2.0 / 3, 1.0 / 6, 1.0 / 6}};
        return emit(o, 1, bary, w);
    }
    case 7: {
        // listed by (x, y) with the third coordinate 1 - x - y (GaussHammer_base.m:54-71)
        const double x[7] = {0.1012865073235, 0.7974269853531, 0.1012865073235, 0.4701420641051,
                             0.4701420641051, 0.0597158717898, 0.3333333333333};
        const double y[7] = {0.1012865073235, 0.1012865073235, 0.7974269853531, 0.0597158717898,
                             0.4701420641051, 0.4701420641051, 0.3333333333333};
        const double ww[7] = {0.1259391805448 / 2, 0.1259391805448 / 2, 0.1259391805448 / 2,
                              0.1323941527885 / 2, 0.1323941527885 / 2, 0.1323941527885 / 2, 0.225 / 2};
        for (int i = 0; i < 7; i++) { bary[i][0] = x[i]; bary[i][1] = y[i]; bary[i][2] = 1 - x[i] - y[i]; w[i] = ww[i]; }
        return 7;
    }
    case 12: {
        const double w1 = 0.050844906370207 / 2, w2 = 0.116786275726379 / 2;
        const Orbit o[] = {{S21H, 0.873821971016996, 0, w1},
                           {S21H, 0.501426509658179, 0, w2},
                           {S111, 0.636502499121399, 0.310352451033784, (0.5 - 3 * w1 - 3 * w2) / 6}};
        return emit(o, 3, bary, w);
    }
    case 19: {
        const Orbit o[] = {{S3, 0, 0, 0.09713579628279610 / 2},
                           {S21, 0.02063496160252593, 0.48968251919873700, 0.09400410068141950 / 6},
                           {S21, 0.1258208170141290, 0.4370895914929355, 0.2334826230143263 / 6},
                           {S21, 0.6235929287619356, 0.1882035356190322, 0.2389432167816273 / 6},
                           {S21, 0.91054097321109410, 0.04472951339445297, 0.07673302697609430 / 6},
                           {S111, 0.03683841205473626, 0.74119859878449800, 0.2597012362637364 / 12}};
        return emit(o, 6, bary, w);
    }
    case 28: {
        const Orbit o[] = {{S3, 0, 0, 0.08797730116222190 / 2},
                           {S21, 0.94802171814342330, 0.02598914092828833, 0.02623293466120857 / 6},
                           {S21, 0.81142499470415460, 0.09428750264792270, 0.1142447159818060 / 6},
                           {S21, 0.01072644996557060, 0.49463677501721470, 0.05656634416839376 / 6},
                           {S21, 0.5853132347709715, 0.2073433826145142, 0.2164790926342230 / 6},
                           {S21, 0.1221843885990187, 0.4389078057004907, 0.2079874161166116 / 6},
                           {S111, 0.0, 0.8588702812826364, 0.04417430269980344 / 12},
                           {S111, 0.04484167758913055, 0.67793765488259020, 0.2463378925757316 / 12}};
        return emit(o, 8, bary, w);
    }
    default:
        return 0;
    }
}

int gh_composite(int n_nodes, int n_sub, double* nodes, double* weights) {
    double bary[28][3], w[28];
    if (gh_base(n_nodes, bary, w) != n_nodes || n_nodes <= 0) return EBEM_ERR_INVALID;
    if (n_sub < 1) return EBEM_ERR_INVALID;
    int nd = (int)std::lround(std::sqrt((double)n_sub));
    if (nd * nd != n_sub) return EBEM_ERR_INVALID;
    const double f = 1.0 / nd;
    int s = 0;
    for (int row = 1; row <= nd; row++) {
        double zlo = (row - 1) * f, zhi = row * f;
        // sub-triangle vertices in barycentric (x, y, z): a sliding window over
        // the row, alternating upward and downward triangles
        double X[3] = {1 - zlo, 1 - zlo, 1 - zlo - f};
        double Y[3] = {-f, 0, 0};
        double Z[3] = {0, 0, 0};
        for (int k = 1; k <= 2 * (nd - row) + 1; k++) {
            double nx3 = (k & 1) ? X[2] : X[2] - f;
            double ny3 = (k & 1) ? Y[2] + f : Y[2];
            X[0] = X[1]; X[1] = X[2]; X[2] = nx3;
            Y[0] = Y[1]; Y[1] = Y[2]; Y[2] = ny3;
            if (k & 1) { Z[0] = zlo; Z[1] = zhi; Z[2] = zlo; }
            else { Z[0] = zhi; Z[1] = zlo; Z[2] = zhi; }
            for (int g = 0; g < n_nodes; g++) {
                double* o = nodes + 3 * ((size_t)s * n_nodes + g);
                o[0] = bary[g][0] * X[0] + bary[g][1] * X[1] + bary[g][2] * X[2];
                o[1] = bary[g][0] * Y[0] + bary[g][1] * Y[1] + bary[g][2] * Y[2];
                o[2] = bary[g][0] * Z[0] + bary[g][1] * Z[1] + bary[g][2] * Z[2];
            }
            s++;
        }
    }
    for (int g = 0; g < n_nodes; g++) weights[g] = (2.0 / n_sub) * w[g];
    return EBEM_OK;
}

}  // namespace ebem
