// Stand-in for src/math/poly_approx.cpp when the reference is compiled without MPFR headers
// (this image has the MPFR runtime but no headers, and the reference build is restricted to
// its own sources).  TEST INFRASTRUCTURE ONLY.
//
// The reference fits the EvalMod polynomial with MPFR (binboot_han_ki_discrete_multi_interval_
// approximate, poly_approx.cpp:565-681): a Chebyshev series on [interval_min, interval_max] of
// f(u) = 1/2 - 1/2 cos(2 pi K u / 2^double_angle), which double_angle iterations of
// x -> 4 x (1 - x) turn into sin^2(pi K u).  This stand-in interpolates the same f in double
// precision at degree+1 Chebyshev nodes on [-1, 1] and zeroes the odd coefficients as the
// reference does.  It is NOT the reference's fit: bootstrapping contexts built from this
// library have different EvalMod coefficients, and only tests that take the coefficients the
// context reports (never fixed ones) may use them.
#include <cmath>
#include <stdexcept>
#include <vector>

#include "poly_approx.hpp"

PolynomialApproximation binboot_han_ki_discrete_multi_interval_approximate(
    double K, size_t degree, size_t double_angle, double interval_radius, size_t, double prune) {
    if (!(K > 0.0) || degree == 0 || double_angle > 30 || !(interval_radius > 0.0))
        throw std::invalid_argument("EvalMod stand-in fit: invalid parameters");
    const double pi = std::acos(-1.0);
    const double shrink = std::ldexp(1.0, (int)double_angle);
    const size_t n = degree + 1;
    std::vector<double> fx(n);
    for (size_t j = 0; j < n; ++j) {
        const double theta = pi * ((double)j + 0.5) / (double)n;
        const double u = std::cos(theta);
        fx[j] = 0.5 - 0.5 * std::cos(2.0 * pi * K * u / shrink);
    }
    std::vector<double> c(n, 0.0);
    for (size_t k = 0; k < n; ++k) {
        double acc = 0.0;
        for (size_t j = 0; j < n; ++j) acc += fx[j] * std::cos(pi * (double)k * ((double)j + 0.5) / (double)n);
        c[k] = (k == 0 ? 1.0 : 2.0) * acc / (double)n;
    }
    for (size_t k = 1; k < n; k += 2) c[k] = 0.0;
    for (double& v : c)
        if (v != 0.0 && std::abs(v) < prune) v = 0.0;
    PolynomialApproximation out;
    out.chebyshev_coeffs = std::move(c);
    out.interval_min = -1.0;
    out.interval_max = 1.0;
    out.degree = degree;
    out.max_error = 0.0;
    return out;
}
