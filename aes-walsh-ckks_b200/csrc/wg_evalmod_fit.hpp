// EvalMod polynomial fit and K bound (wg_evalmod_fit.cpp).
#pragma once
#include <cstddef>
#include <vector>

namespace wg {
namespace fit {

struct EvalModFit {
    std::vector<double> coeffs;  // Chebyshev coefficients on [interval_min, interval_max]
    double max_error = 0.0;      // over the validation points of every interval
    double interval_min = 0.0, interval_max = 0.0;
    size_t degree = 0;
    size_t pruned = 0;
};

// Chebyshev series of 1/2 - 1/2 cos(2 pi K u / 2^double_angle) on the 2K - 1 intervals of
// radius interval_radius / K around the multiples of 1/(2K) (Han-Ki multi-interval fit).
EvalModFit fit_evalmod(double K, size_t degree, size_t double_angle, double interval_radius, size_t points,
                       double prune);

// EvalMod K for a sparse secret of `hamming_weight` over `coefficients` coefficients at the
// given failure probability.
size_t evalmod_k_bound(size_t coefficients, size_t hamming_weight, long double failure_probability);

}  // namespace fit
}  // namespace wg
