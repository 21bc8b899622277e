// ORACLE — test infrastructure only (see sa_oracle.hpp).  The manufactured
// datum 'TEST' of the reference: the boundary value whose solution on the
// screen [-1, 1]^2 (z = 0) is the constant density phi = (1, 1, 1).
//
// Restates functions/BEMenerg_indir/BEMenerg_core/BEMenerg_core_calcTn/
// BEMenerg_core_calcNucleoTn.m:13-132: for a source point x = (x1, x2) on the
// screen and the instants t0 < t1,
//   ris_c = (1 / 4 pi rho) int_{[-L,L]^2} nucl_c(y) dy,   L = 1,
//   nucl_c = f_c(t1) - f_c(t0),
// with r = |y - x|, c = (y1 - x1)/r, s = (y2 - x2)/r and, per instant t,
//   J_v = H(t - r/v) / (v^2 r),   I_v = H(t - r/v) (t - r/v)(t + r/v) / (2 r^3),
//   A = J_P - J_S,  B = I_P - I_S,  S = J_S,
//   f_1 = A c^2 + B (3 c^2 - 1) + S + c s (A + 3 B),
//   f_2 = A s^2 + B (3 s^2 - 1) + S + c s (A + 3 B),
//   f_3 = S - B
// (the sums of nucl_1, nucl_2, nucl_3 of :97-125 regrouped by instant).  The
// reference integrates with integral2 (BEMenerg_core_TnTest_classic.m:11-13,
// RelTol 1e-5); here polar coordinates about x: the square is cut into the
// four triangles (x, side), the angle is integrated along each side by
// composite Gauss-Legendre (graded toward the foot of the perpendicular and
// split at every crossing of a front circle r = v t with the side), the
// radius by Gauss-Legendre on the pieces between the front radii, where r f
// is smooth.  Where both fronts have passed
// the t^2 / r^3 parts of I_P - I_S cancel and B = (1/c_S^2 - 1/c_P^2) / (2 r)
// is used instead of the difference.
#include <algorithm>
#include <cmath>
#include <vector>

namespace {

const double kPi = 3.14159265358979323846;

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    // Newton's iteration on P_n from the Chebyshev-like initial guesses; nodes
    // on (-1, 1), ascending.
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; i++) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), dp = 1;
        for (int it = 0; it < 100; it++) {
            double p0 = 1, p1 = z;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) p0 = 1;
            dp = n * (z * p1 - p0) / (z * z - 1);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[n - 1 - i] = z;
        w[n - 1 - i] = 2 / ((1 - z * z) * dp * dp);
    }
}

struct Speeds {
    double cP, cS;
};

// r f_c(r, theta; t) for the three components (the polar Jacobian included).
void rf(double r, double c, double s, double t, const Speeds& v, double out[3]) {
    out[0] = out[1] = out[2] = 0;
    if (t <= 0) return;
    const double hP = (t - r / v.cP > 0) ? 1.0 : 0.0, hS = (t - r / v.cS > 0) ? 1.0 : 0.0;
    const double rA = hP / (v.cP * v.cP) - hS / (v.cS * v.cS);
    const double rS = hS / (v.cS * v.cS);
    double rB;
    if (hS > 0) rB = 0.5 * (1 / (v.cS * v.cS) - 1 / (v.cP * v.cP));
    else if (hP > 0) rB = (t - r / v.cP) * (t + r / v.cP) / (2 * r * r);
    else rB = 0;
    out[0] = rA * c * c + rB * (3 * c * c - 1) + rS + c * s * (rA + 3 * rB);
    out[1] = rA * s * s + rB * (3 * s * s - 1) + rS + c * s * (rA + 3 * rB);
    out[2] = rS - rB;
}

// int over the square of f_c(t1) - f_c(t0): per side, the angle as the
// position u along the side from the foot of the perpendicular (distance d):
// R = sqrt(d^2 + u^2), dtheta = d du / R^2; u cut at the foot, at +-d 2^j
// (the integrand's singularities sit at u = +-i d) and at the front
// crossings; nang nodes on each of nsplit equal parts of a piece.
void square_integral(double x1, double x2, double t0, double t1, const Speeds& v, int nang, int nsplit, int nrad,
                     double acc[3]) {
    std::vector<double> ga, wa, gr, wr;
    gauss_legendre(nang, ga, wa);
    gauss_legendre(nrad, gr, wr);
    const double cx[4] = {-1, 1, 1, -1}, cy[4] = {-1, -1, 1, 1};
    std::vector<double> radii;
    for (double t : {t0, t1})
        if (t > 0) {
            radii.push_back(v.cS * t);
            radii.push_back(v.cP * t);
        }
    acc[0] = acc[1] = acc[2] = 0;
    for (int k = 0; k < 4; k++) {
        const double ax = cx[k] - x1, ay = cy[k] - x2;
        const double bx = cx[(k + 1) % 4] - x1, by = cy[(k + 1) % 4] - x2;
        const double len = std::hypot(bx - ax, by - ay), ex = (bx - ax) / len, ey = (by - ay) / len;
        const double s0 = -(ax * ex + ay * ey);
        const double fx = ax + s0 * ex, fy = ay + s0 * ey;
        const double d = fx * ey - fy * ex;
        const double ulo = -s0, uhi = len - s0;
        std::vector<double> cuts = {ulo, uhi};
        auto add = [&](double u) { if (u > ulo && u < uhi) cuts.push_back(u); };
        add(0.0);
        for (double rho : radii)
            if (rho > d) {
                add(-std::sqrt(rho * rho - d * d));
                add(std::sqrt(rho * rho - d * d));
            }
        for (double g = d; g < std::max(-ulo, uhi); g *= 2) {
            add(-g);
            add(g);
        }
        std::sort(cuts.begin(), cuts.end());
        for (size_t q = 0; q + 1 < cuts.size(); q++) {
            const double h = (cuts[q + 1] - cuts[q]) / nsplit;
            for (int m = 0; m < nsplit; m++)
                for (int ia = 0; ia < nang; ia++) {
                    const double u = cuts[q] + h * (m + 0.5 * (ga[ia] + 1));
                    const double R = std::hypot(d, u);
                    const double wth = 0.5 * h * wa[ia] * d / (R * R);
                    const double c = (fx + u * ex) / R, s = (fy + u * ey) / R;
                    std::vector<double> rb = {0.0, R};
                    for (double rho : radii)
                        if (rho < R) rb.push_back(rho);
                    std::sort(rb.begin(), rb.end());
                    for (size_t p = 0; p + 1 < rb.size(); p++) {
                        const double lo = rb[p], ln = rb[p + 1] - rb[p];
                        if (ln <= 0) continue;
                        for (int ir = 0; ir < nrad; ir++) {
                            const double r = lo + 0.5 * ln * (gr[ir] + 1), wrr = 0.5 * ln * wr[ir];
                            double f1[3], f0[3];
                            rf(r, c, s, t1, v, f1);
                            rf(r, c, s, t0, v, f0);
                            for (int e = 0; e < 3; e++) acc[e] += wth * wrr * (f1[e] - f0[e]);
                        }
                    }
                }
        }
    }
}

}  // namespace

extern "C" {

// ris of BEMenerg_core_calcNucleoTn.m:13-132 ('TEST'), divided by 4 pi rho
// as at :128; nang x nsplit angular and nrad radial nodes per piece.
int or_tn_test(double x1, double x2, double t0, double t1, double rho, double mu, double lambda, int nang, int nsplit,
               int nrad, double* out) {
    if (nang < 1 || nsplit < 1 || nrad < 1 || !(std::fabs(x1) < 1) || !(std::fabs(x2) < 1)) return -1;
    Speeds v{std::sqrt((lambda + 2 * mu) / rho), std::sqrt(mu / rho)};
    double acc[3];
    square_integral(x1, x2, t0, t1, v, nang, nsplit, nrad, acc);
    for (int e = 0; e < 3; e++) out[e] = acc[e] / (4 * kPi * rho);
    return 0;
}

}  // extern "C"
