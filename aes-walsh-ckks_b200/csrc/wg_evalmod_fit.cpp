// EvalMod polynomial fit on the host: the Chebyshev series that the bootstrap's EvalMod step
// evaluates, built once per parameter set when a context is created.
//
// The method is the multi-interval cosine approximation of K. Han and D. Ki, "Better
// Bootstrapping for Approximate Homomorphic Encryption" (CT-RSA 2020, ePrint 2019/688), as the
// reference applies it to binary bootstrapping (binboot_han_ki_discrete_multi_interval_approximate,
// src/math/poly_approx.cpp:565-681, with han_ki_gen_degrees :233-312, han_ki_gen_nodes :314-357,
// han_ki_solve_system :359-458):
//   1. distribute degree + 1 nodes over the 2K - 1 intervals around the integers -K+1 .. K-1
//      (after scaling by 1/(2K)) by repeatedly raising the degree of the interval whose
//      log2 error bound is largest;
//   2. place Chebyshev nodes cos(2 pi j / 2d_i) on each interval and evaluate the target
//      1/2 - 1/2 cos(2 pi K u / 2^double_angle) there;
//   3. form the Newton divided differences, evaluate the interpolant at the degree + 1
//      Chebyshev extrema of [-K', K'] and solve the Chebyshev-basis system by Gaussian
//      elimination with partial pivoting;
//   4. round to double, zero the odd coefficients, drop those below the prune threshold.
// Steps 2-3 run in 256-bit MPFR arithmetic with round-to-nearest, one correctly rounded
// operation per step in the reference's order, so the doubles are the reference's bit for bit
// (the residues of every bootstrap depend on them through the encoded constants).  Step 1 and
// the validation run in double with the reference's operation order, including the one
// product the reference's compiler contracts into a fused multiply-add (this file is built
// without contraction and spells it out).
//
// Also the EvalMod K bound of sparse-secret bootstrapping (required_binboot_k_bound,
// src/math/binboot_k_bound.cpp:53-89): the smallest K whose Irwin-Hall tail bound over the
// ring's coefficients is below the target failure probability, plus one.
#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <utility>
#include <vector>

#include "mpfr_decl/mpfr.h"
#include "wg_evalmod_fit.hpp"

namespace wg {
namespace fit {
namespace {

constexpr mpfr_prec_t kBits = 256;
constexpr double kPi = 3.141592653589793238462643383279502884;

// A 256-bit MPFR number; every arithmetic step below names its MPFR call explicitly.
class Mp {
public:
    Mp() {
        mpfr_init2(v_, kBits);
        mpfr_set_ui(v_, 0, MPFR_RNDN);
    }
    static Mp from_d(double x) {
        Mp r;
        mpfr_set_d(r.v_, x, MPFR_RNDN);
        return r;
    }
    static Mp from_i(long x) {
        Mp r;
        mpfr_set_si(r.v_, x, MPFR_RNDN);
        return r;
    }
    static Mp pi() {
        Mp r;
        mpfr_const_pi(r.v_, MPFR_RNDN);
        return r;
    }
    static Mp pow2(unsigned long e) {
        Mp r;
        mpfr_set_ui_2exp(r.v_, 1, (mpfr_exp_t)e, MPFR_RNDN);
        return r;
    }
    Mp(const Mp& o) {
        mpfr_init2(v_, kBits);
        mpfr_set(v_, o.v_, MPFR_RNDN);
    }
    Mp(Mp&& o) noexcept {
        mpfr_init2(v_, kBits);
        mpfr_swap(v_, o.v_);
    }
    Mp& operator=(const Mp& o) {
        if (this != &o) mpfr_set(v_, o.v_, MPFR_RNDN);
        return *this;
    }
    Mp& operator=(Mp&& o) noexcept {
        if (this != &o) mpfr_swap(v_, o.v_);
        return *this;
    }
    ~Mp() { mpfr_clear(v_); }
    mpfr_ptr p() { return v_; }
    mpfr_srcptr p() const { return v_; }
    double d() const { return mpfr_get_d(v_, MPFR_RNDN); }

private:
    mpfr_t v_;
};

Mp add(const Mp& a, const Mp& b) {
    Mp r;
    mpfr_add(r.p(), a.p(), b.p(), MPFR_RNDN);
    return r;
}
Mp sub(const Mp& a, const Mp& b) {
    Mp r;
    mpfr_sub(r.p(), a.p(), b.p(), MPFR_RNDN);
    return r;
}
Mp mul(const Mp& a, const Mp& b) {
    Mp r;
    mpfr_mul(r.p(), a.p(), b.p(), MPFR_RNDN);
    return r;
}
Mp div(const Mp& a, const Mp& b) {
    Mp r;
    mpfr_div(r.p(), a.p(), b.p(), MPFR_RNDN);
    return r;
}
Mp neg(const Mp& a) {
    Mp r;
    mpfr_neg(r.p(), a.p(), MPFR_RNDN);
    return r;
}
Mp mcos(const Mp& a) {
    Mp r;
    mpfr_cos(r.p(), a.p(), MPFR_RNDN);
    return r;
}
Mp mabs(const Mp& a) {
    Mp r;
    mpfr_abs(r.p(), a.p(), MPFR_RNDN);
    return r;
}
void add_to(Mp& a, const Mp& b) { mpfr_add(a.p(), a.p(), b.p(), MPFR_RNDN); }
void sub_from(Mp& a, const Mp& b) { mpfr_sub(a.p(), a.p(), b.p(), MPFR_RNDN); }
void mul_by(Mp& a, const Mp& b) { mpfr_mul(a.p(), a.p(), b.p(), MPFR_RNDN); }
void div_by(Mp& a, const Mp& b) { mpfr_div(a.p(), a.p(), b.p(), MPFR_RNDN); }
bool greater(const Mp& a, const Mp& b) { return mpfr_cmp(a.p(), b.p()) > 0; }

// Step 1: interval degrees (d_0 for the centre interval, d_i for +-i) and the node count.
std::vector<int> interval_degrees(int degree, int intervals, double dev, int& total) {
    const int bound = degree + 1;
    total = 2 * intervals - 1;
    const double err = 1.0 / dev;
    const double log2_2pi = std::log2(2.0 * kPi);
    std::vector<int> deg(intervals, 1);
    std::vector<double> lb(intervals, 0.0);
    double base = 0.0;
    for (int i = 1; i <= 2 * intervals - 1; ++i) base -= std::log2((double)i);
    base = std::fma(2.0 * (double)intervals - 1.0, log2_2pi, base);
    base += std::log2(err);
    for (int i = 0; i < intervals; ++i) {
        lb[i] = base;
        for (int j = 1; j <= intervals - 1 - i; ++j) lb[i] += std::log2((double)j + err);
        for (int j = 1; j <= intervals - 1 + i; ++j) lb[i] += std::log2((double)j + err);
    }
    for (int it = 0; it < 200 && total < bound; ++it) {
        const int worst = (int)(std::max_element(lb.begin(), lb.end()) - lb.begin());
        if (worst != 0) {
            // a side interval takes two more nodes (its mirror image too)
            if (total + 2 > bound) break;
            for (int i = 0; i < intervals; ++i) {
                lb[i] -= std::log2((double)(total + 1));
                lb[i] -= std::log2((double)(total + 2));
                lb[i] += 2.0 * log2_2pi;
                if (i != worst) {
                    lb[i] += std::log2(std::abs((double)(i - worst)) + err);
                    lb[i] += std::log2((double)(i + worst) + err);
                } else {
                    lb[i] += std::log2(err) - 1.0;
                    lb[i] += std::log2(2.0 * (double)i + err);
                }
            }
            total += 2;
        } else {
            lb[0] -= std::log2((double)(total + 1));
            lb[0] += std::log2(err) - 1.0;
            lb[0] += log2_2pi;
            for (int i = 1; i < intervals; ++i) {
                lb[i] -= std::log2((double)(total + 1));
                lb[i] += log2_2pi;
                lb[i] += std::log2((double)i + err);
            }
            total += 1;
        }
        ++deg[worst];
    }
    return deg;
}

// Clenshaw evaluation of a Chebyshev series at t in [-1, 1] (the reference's contraction).
double clenshaw(const std::vector<double>& c, double t) {
    double b1 = 0.0, b2 = 0.0;
    for (size_t k = c.size(); k > 1; --k) {
        const double b0 = std::fma(2.0 * t, b1, -b2) + c[k - 1];
        b2 = b1;
        b1 = b0;
    }
    return c.empty() ? 0.0 : std::fma(t, b1, c[0]) - b2;
}

double target(double u, double period) { return 0.5 * (1.0 - std::cos(2.0 * kPi * u / period)); }

}  // namespace

EvalModFit fit_evalmod(double K, size_t degree, size_t double_angle, double interval_radius, size_t points,
                       double prune) {
    if (!std::isfinite(K) || K <= 0.0) throw std::invalid_argument("evalmod fit: K must be positive");
    if (double_angle > 30) throw std::invalid_argument("evalmod fit: double_angle is too large");
    if (!std::isfinite(interval_radius) || interval_radius <= 0.0 || interval_radius >= 0.25)
        throw std::invalid_argument("evalmod fit: interval_radius must be in (0, 0.25)");
    if (points < 2) throw std::invalid_argument("evalmod fit: at least 2 validation points per interval");
    if (!std::isfinite(prune) || prune < 0.0) throw std::invalid_argument("evalmod fit: invalid prune threshold");
    if (degree == 0) throw std::invalid_argument("evalmod fit: degree must be positive");
    const int intervals = (int)std::llround(2.0 * K);
    if (std::abs((double)intervals - 2.0 * K) > 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, K))
        throw std::invalid_argument("evalmod fit: K must be an integer or half-integer");
    const double spacing = 0.5 / K;
    const double radius = interval_radius / K;  // normalised to the 1/(2K) spacing
    const double local = radius / spacing;
    if (!(radius > 0.0) || radius > 0.5 * spacing) throw std::invalid_argument("evalmod fit: radius too large");
    const double dev = 1.0 / local;

    int total = 0;
    const std::vector<int> deg = interval_degrees((int)degree, intervals, dev, total);

    // Step 2: nodes and target values.
    const Mp width = div(Mp::from_i(1), Mp::from_d(dev));
    const Mp mspacing = Mp::from_d(spacing);
    const Mp pi = Mp::pi();
    std::vector<Mp> x(total);
    int n = (deg[0] & 1) ? 1 : 0;  // an odd centre degree keeps the node at 0
    auto chebyshev_offset = [&](int j, int d) {
        Mp th = mul(pi, Mp::from_i(2 * j));
        div_by(th, Mp::from_i(2 * d));
        return mul(mcos(th), width);
    };
    for (int i = intervals - 1; i > 0; --i)
        for (int j = 0; j < deg[i]; ++j) {
            x[n] = mul(add(Mp::from_i(i), chebyshev_offset(j, deg[i])), mspacing);
            x[n + 1] = neg(x[n]);
            n += 2;
        }
    for (int j = 0; j < deg[0] / 2; ++j) {
        x[n] = mul(chebyshev_offset(j, deg[0]), mspacing);
        x[n + 1] = neg(x[n]);
        n += 2;
    }
    const Mp half = Mp::from_d(0.5);
    const Mp shrink = Mp::pow2(double_angle);
    std::vector<Mp> y(total);
    for (int i = 0; i < total; ++i) {
        const Mp u = div(x[i], shrink);
        const Mp arg = mul(mul(mul(Mp::from_i(2), pi), Mp::from_d(K)), u);
        y[i] = sub(half, mul(half, mcos(arg)));
    }

    // Step 3: divided differences, the interpolant at the Chebyshev extrema, the system.
    for (int j = 1; j < total; ++j)
        for (int i = 0; i < total - j; ++i) {
            y[i] = sub(y[i + 1], y[i]);
            div_by(y[i], sub(x[i + j], x[i]));
        }
    const int m = total + 1;
    const Mp kscale = div(mul(Mp::from_i(intervals), Mp::from_d(spacing)), shrink);
    std::vector<Mp> ext(m), rhs(m);
    for (int i = 0; i < m; ++i) {
        Mp th = mul(pi, Mp::from_i(i));
        div_by(th, Mp::from_i(m - 1));
        ext[i] = mul(kscale, mcos(th));
    }
    for (int i = 0; i < m; ++i) {
        rhs[i] = y[0];
        for (int j = 1; j < m - 1; ++j) {
            mul_by(rhs[i], sub(ext[i], x[j]));
            add_to(rhs[i], y[j]);
        }
    }
    std::vector<std::vector<Mp>> T(m, std::vector<Mp>(m));
    const Mp two = Mp::from_i(2);
    for (int i = 0; i < m; ++i) {
        T[i][0] = Mp::from_i(1);
        T[i][1] = div(ext[i], kscale);
        for (int j = 2; j < m; ++j) {
            const Mp t = div(ext[i], kscale);
            T[i][j] = sub(mul(mul(two, t), T[i][j - 1]), T[i][j - 2]);
        }
    }
    for (int i = 0; i < m - 1; ++i) {
        int piv = i;
        Mp best = mabs(T[i][i]);
        for (int j = i + 1; j < m; ++j) {
            Mp cand = mabs(T[j][i]);
            if (greater(cand, best)) {
                best = std::move(cand);
                piv = j;
            }
        }
        if (piv != i) {
            std::swap(T[i], T[piv]);
            std::swap(rhs[i], rhs[piv]);
        }
        for (int j = i + 1; j < m; ++j) div_by(T[i][j], T[i][i]);
        div_by(rhs[i], T[i][i]);
        T[i][i] = Mp::from_i(1);
        for (int j = i + 1; j < m; ++j) {
            sub_from(rhs[j], mul(T[j][i], rhs[i]));
            for (int l = i + 1; l < m; ++l) sub_from(T[j][l], mul(T[j][i], T[i][l]));
            T[j][i] = Mp();
        }
    }
    std::vector<Mp> coef(m);
    coef[m - 1] = rhs[m - 1];
    for (int i = m - 2; i >= 0; --i) {
        coef[i] = rhs[i];
        for (int j = i + 1; j < m; ++j) sub_from(coef[i], mul(T[i][j], coef[j]));
    }

    // Step 4: doubles, even part, pruning; interval and validation as the reference reports them.
    EvalModFit out;
    out.coeffs.resize(total);
    for (int i = 0; i < total; ++i) out.coeffs[i] = coef[i].d();
    const double iscale = std::pow(2.0, (double)double_angle);
    out.interval_min = -spacing * (double)intervals / iscale;
    out.interval_max = spacing * (double)intervals / iscale;
    for (size_t i = 1; i < out.coeffs.size(); i += 2) out.coeffs[i] = 0.0;
    for (double& c : out.coeffs)
        if (c != 0.0 && std::abs(c) < prune) {
            c = 0.0;
            ++out.pruned;
        }
    double worst = 0.0;
    for (int ci = -(intervals - 1); ci <= intervals - 1; ++ci) {
        const double centre = 0.5 * (double)ci;
        for (size_t j = 0; j < points; ++j) {
            const double a = (double)j / (double)(points - 1);
            const double xv = std::fma(interval_radius, 2.0 * a - 1.0, centre);
            const double u = xv / K;
            const double expect = target(u, 1.0 / K);
            const double t = (2.0 * u - out.interval_min - out.interval_max) / (out.interval_max - out.interval_min);
            double got = clenshaw(out.coeffs, t);
            for (size_t k = 0; k < double_angle; ++k) got = 4.0 * got * (1.0 - got);
            if (!std::isfinite(expect) || !std::isfinite(got))
                throw std::runtime_error("evalmod fit: non-finite validation value");
            worst = std::max(worst, std::abs(got - expect));
        }
    }
    out.max_error = worst;
    out.degree = out.coeffs.empty() ? 0 : out.coeffs.size() - 1;
    return out;
}

namespace {

long double binomial(size_t n, size_t k) {
    if (k > n) return 0.0L;
    k = std::min(k, n - k);
    long double r = 1.0L;
    for (size_t i = 1; i <= k; ++i) {
        r *= (long double)(n - k + i);
        r /= (long double)i;
    }
    return r;
}

// P(|S - h/2| >= K) for S a sum of h uniforms on [0, 1] (two Irwin-Hall tails).
long double irwin_hall_tail(size_t h, size_t K) {
    const long double half_h = (long double)h / 2.0L;
    if ((long double)K >= half_h) return 0.0L;
    const long double x = half_h - (long double)K;
    if (x <= 0.0L) return 0.0L;
    if (x >= (long double)h) return 2.0L;
    const size_t top = (size_t)std::floor(x);
    long double s = 0.0L;
    for (size_t k = 0; k <= top; ++k) {
        const long double term = binomial(h, k) * std::pow(x - (long double)k, (long double)h);
        s += (k & 1U) == 0U ? term : -term;
    }
    return 2.0L * (s / std::tgammal((long double)h + 1.0L));
}

}  // namespace

size_t evalmod_k_bound(size_t coefficients, size_t hamming_weight, long double failure_probability) {
    if (coefficients == 0 || hamming_weight == 0) throw std::invalid_argument("evalmod K bound: invalid sizes");
    if (!std::isfinite(failure_probability) || failure_probability <= 0.0L || failure_probability >= 1.0L)
        throw std::invalid_argument("evalmod K bound: invalid failure probability");
    const size_t max_k = (hamming_weight + 1) / 2;
    for (size_t K = 0; K <= max_k; ++K) {
        const long double total = std::min(1.0L, (long double)coefficients * irwin_hall_tail(hamming_weight, K));
        if (total <= failure_probability) return K + 1;
    }
    return max_k + 1;
}

}  // namespace fit
}  // namespace wg
