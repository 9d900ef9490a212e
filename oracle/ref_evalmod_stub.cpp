// Stand-in for src/math/poly_approx.cpp when the reference is compiled without MPFR headers.
// The EvalMod Chebyshev fit is only run while building a bootstrapping context; contexts
// built by the harness have no bootstrapping keys, so reaching this is a harness misuse.
#include <stdexcept>

#include "poly_approx.hpp"

PolynomialApproximation binboot_han_ki_discrete_multi_interval_approximate(
    double, size_t, size_t, double, size_t, double) {
    throw std::runtime_error(
        "EvalMod polynomial fit is unavailable: the reference was compiled without MPFR");
}
