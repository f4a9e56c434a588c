// Zolotarev rational approximation of 1/sqrt(x) on [amin, amax], as used by the
// overlap operator: (h_W^2)^(-1/2) ~ sum_l b_l / (h_W^2 + d_l).
//
// The steps follow OverlapOperations::ZolotarevCoefficients
// (FERMIONS/OVERLAP/OPERATOR/ZolotarevCoefficients.cpp:5-175) so that the
// coefficients agree with the reference's to rounding: the complete elliptic
// integral by Carlson's duplication (:5-49), Jacobi sn through the descending
// Landen/AGM sequence (:93-121), pole residues as ratios of the c_l (:51-69,
// 124-128) and a normalisation that centres the relative error on 1 over a
// 5000-point logarithmic scan (:130-163).  The reference evaluates two square
// roots in single precision (sqrtf at :97, :106 and :148); they are kept, since
// they move the coefficients at the 1e-7 level.
#include <cmath>
#include <vector>

namespace ovl {

static double carlson_k(double kappa, double err) {
    double X = 0.0, Y = 1.0 - kappa, Z = 1.0;
    double mu = (X + Y + Z) / 3.0;
    double dx = 2.0 - (mu + X) / mu, dy = 2.0 - (mu + Y) / mu, dz = 2.0 - (mu + Z) / mu;
    double eps = err;
    while (eps >= err) {
        mu = (X + Y + Z) / 3.0;
        dx = 2.0 - (mu + X) / mu;
        dy = 2.0 - (mu + Y) / mu;
        dz = 2.0 - (mu + Z) / mu;
        eps = std::fabs(dx);
        if (std::fabs(dy) > eps) eps = std::fabs(dy);
        if (std::fabs(dz) > eps) eps = std::fabs(dz);
        const double sx = std::sqrt(X), sy = std::sqrt(Y), sz = std::sqrt(Z);
        const double lambda = sx * (sy + sz) + sy * sz;
        X = 0.25 * (X + lambda);
        Y = 0.25 * (Y + lambda);
        Z = 0.25 * (Z + lambda);
    }
    const double e2 = dx * dy - dz * dz, e3 = dx * dy * dz;
    const double s = 1.0 + (e2 / 24.0 - 0.1 - e3 / 44.0) * e2 + e3 / 14.0;
    return s / std::sqrt(mu);
}

// residue of pole n: prod_i (c_{2i+1} - c_{2n}) / prod_{j != n} (c_{2j} - c_{2n})
static double residue(const std::vector<double> &c, int n, int order) {
    double prod = 1.0;
    int j = 0;
    for (int i = 0; i < order - 1; i++) {
        prod *= (c[2 * i + 1] - c[2 * n]);
        if (i == n) j++;
        prod /= (c[2 * j] - c[2 * n]);
        j++;
    }
    return prod;
}

double zolotarev(double amin, double amax, double errtol, int no, double *b, double *d) {
    std::vector<double> alpha(4000), gamma(4000), c(2 * no);
    const double kappa = std::sqrt(1.0 - amin / amax);
    const double K = carlson_k(kappa, errtol);
    const double zn = 0.5 * K / no;
    for (int l = 0; l < 2 * no - 1; l++) {
        const double xn = (l + 1) * zn;
        alpha[0] = 1.0;
        double beta = sqrtf(1.0 - kappa);
        gamma[0] = std::sqrt(kappa);
        int i = 1;
        double pow2 = 1.0;
        while (std::fabs(gamma[i - 1] / alpha[i - 1]) >= errtol) {
            const double prev = beta;
            alpha[i] = (alpha[i - 1] + prev) * 0.5;
            beta = sqrtf(alpha[i - 1] * prev);
            gamma[i] = (alpha[i - 1] - prev) * 0.5;
            i++;
            pow2 *= 2.0;
        }
        i -= 1;
        double phi = pow2 * alpha[i] * xn;
        while (i >= 1) {
            phi = 0.5 * (phi + std::asin(gamma[i] * std::sin(phi) / alpha[i]));
            i -= 1;
        }
        c[l] = std::tan(phi) * std::tan(phi);
    }
    for (int l = 0; l < no; l++) {
        d[l] = c[2 * l] * amin;
        b[l] = residue(c, l, no);
    }
    const int npoints = 5000;
    const double dx = (std::log(amax) - std::log(amin)) / npoints;
    double yn = std::log(amin) - dx;
    double fmin = 1.0, fmax = 0.0;
    for (int i = 0; i < npoints; i++) {
        yn += dx;
        const double x = std::exp(yn);
        double f = 0.0;
        for (int l = 0; l < no; l++) f += b[l] / (x + d[l]);
        f *= sqrtf(x);
        if (f > fmax) fmax = f;
        if (f < fmin) fmin = f;
    }
    const double norm = 2.0 / (fmin + fmax);
    for (int k = 0; k < no; k++) b[k] *= norm;
    return (fmax - fmin) / (fmax + fmin);
}

}  // namespace ovl
