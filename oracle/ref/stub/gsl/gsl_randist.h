/* Gaussian deviates by the Marsaglia polar method.  The hot path does not use
 * them (inputs are generated outside the reference). */
#pragma once
#include <cmath>
static inline double gsl_ran_gaussian(gsl_rng *r, double sigma) {
    double x, y, r2;
    do {
        x = -1.0 + 2.0 * gsl_rng_uniform_pos(r);
        y = -1.0 + 2.0 * gsl_rng_uniform_pos(r);
        r2 = x * x + y * y;
    } while (r2 > 1.0 || r2 == 0.0);
    return sigma * y * std::sqrt(-2.0 * std::log(r2) / r2);
}
