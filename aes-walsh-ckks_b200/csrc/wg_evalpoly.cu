// Chebyshev polynomial evaluation (the EvalMod / LUT polynomial step) over a batch of
// ciphertexts that share level and scale: every homomorphic operation of the evaluation is one
// set of batched launches for the whole batch.
//
// Reference: ckks_evalchebyshev_preconditioned, src/ckks/operations/evalpoly/ckks_evalpoly.cpp
// (1221-1256), with its power basis (:834-938), scale-aware Paterson-Stockmeyer plan (:548-836,
// the strategy of Bossuat et al., EUROCRYPT 2021, Section 3) and plan evaluation (:940-1219).
// The residues the evaluation produces depend on the exact order of operations and on every
// scalar it rounds, so the host side follows the reference's steps one for one: the same power
// generation order, the same long-double scale bookkeeping (exact scales as seed powers over
// moduli), the same constant rounding (round, then fmod by q, in long double), the same
// baby-step / giant-step schedule.  The device side supplies the operations (tensor product,
// relinearisation, rescale, scalar multiply / multiply-add / add, add, subtract).
#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <map>
#include <optional>
#include <stdexcept>
#include <utility>
#include <vector>

#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_internal.hpp"
#include "wg_ctops.cuh"

namespace wg {
using namespace bk;

namespace {

// ------------------------------------------------------------------------------------------
// Host side: scalars, exact scales and the Paterson-Stockmeyer schedule
// ------------------------------------------------------------------------------------------
size_t bit_length(size_t v) { return v == 0 ? 0 : (size_t)(std::numeric_limits<size_t>::digits - __builtin_clzl(v)); }

size_t ceil_log2(size_t degree) { return degree <= 1 ? 0 : bit_length(degree - 1); }

size_t eval_depth(size_t degree) { return degree <= 1 ? 0 : bit_length(degree) - 1; }

size_t split_log(size_t log_degree) {
    size_t ls = log_degree >> 1;
    const size_t a = (size_t{1} << ls) + (size_t{1} << (log_degree - ls)) + log_degree - ls - 3;
    const size_t b = (size_t{1} << (ls + 1)) + (size_t{1} << (log_degree - ls - 1)) + log_degree - ls - 4;
    if (a > b) ++ls;
    return ls;
}

std::pair<size_t, size_t> split_degree(size_t degree) {
    if (degree == 0) throw std::invalid_argument("ckks_evalchebyshev: cannot split degree zero");
    if ((degree & (degree - 1)) == 0) return {degree >> 1, degree >> 1};
    const size_t k = bit_length(degree - 1) - 1;
    return {(size_t{1} << k) - 1, degree + 1 - (size_t{1} << k)};
}

// round(value * scale) mod q, in long double.
uint64_t scaled_constant_mod(double value, long double scale, uint64_t q) {
    const long double scaled = static_cast<long double>(value) * scale;
    if (!std::isfinite(scaled)) throw std::invalid_argument("ckks_evalpoly: non-finite scaled constant");
    long double residue = std::fmod(std::round(scaled), static_cast<long double>(q));
    if (residue < 0.0L) residue += static_cast<long double>(q);
    uint64_t out = static_cast<uint64_t>(residue);
    if (out >= q) out %= q;
    return out;
}

bool scales_close(double lhs, double rhs, double rel_tol = 0x1p-45) {
    if (!std::isfinite(lhs) || !std::isfinite(rhs)) return false;
    const long double l = lhs, r = rhs;
    const long double m = std::max<long double>({1.0L, std::abs(l), std::abs(r)});
    return std::abs(l - r) <= static_cast<long double>(rel_tol) * m;
}

bool is_integer(double v, double rel_tol = 0x1p-20) {
    if (!std::isfinite(v)) return false;
    return std::abs(v - std::round(v)) <= rel_tol * std::max(1.0, std::abs(v));
}

// A scale seed^seed_exp / prod q_i^den[i], kept exactly.
struct ExactScale {
    uint64_t seed = 1;
    int seed_exp = 0;
    std::vector<int> den;

    static ExactScale of(double value, size_t nmod) {
        if (!std::isfinite(value) || value < 0.0) throw std::invalid_argument("ckks_evalchebyshev: invalid exact scale seed");
        const long double r = std::round(static_cast<long double>(value));
        const long double tol = std::max<long double>(1.0L, std::abs(static_cast<long double>(value))) * 0x1p-20L;
        if (std::abs(static_cast<long double>(value) - r) > tol)
            throw std::invalid_argument("ckks_evalchebyshev: non-integral initial scale is unsupported");
        if (r > static_cast<long double>(std::numeric_limits<uint64_t>::max()))
            throw std::invalid_argument("ckks_evalchebyshev: initial scale exceeds uint64_t");
        ExactScale e;
        e.seed = static_cast<uint64_t>(r);
        e.seed_exp = 1;
        e.den.assign(nmod, 0);
        return e;
    }
    long double value(const std::vector<uint64_t>& q) const {
        long double v = 1.0L;
        for (int i = 0; i < seed_exp; ++i) v *= static_cast<long double>(seed);
        for (size_t i = 0; i < den.size(); ++i)
            for (int e = 0; e < den[i]; ++e) v /= static_cast<long double>(q[i]);
        return v;
    }
    double value_d(const std::vector<uint64_t>& q) const { return static_cast<double>(value(q)); }
};

ExactScale times(const ExactScale& x, const ExactScale& y) {
    ExactScale o;
    o.seed = x.seed;
    o.seed_exp = x.seed_exp + y.seed_exp;
    o.den = x.den;
    if (o.den.size() < y.den.size()) o.den.resize(y.den.size(), 0);
    for (size_t i = 0; i < y.den.size(); ++i) o.den[i] += y.den[i];
    return o;
}

uint64_t ratio_u64(const ExactScale& num, const ExactScale& den, const std::vector<uint64_t>& q) {
    if (num.seed != den.seed) throw std::invalid_argument("ckks_evalchebyshev: mixed exact-scale seeds are unsupported");
    long double r = 1.0L;
    const int d = num.seed_exp - den.seed_exp;
    for (int i = 0; i < d; ++i) r *= static_cast<long double>(num.seed);
    for (int i = 0; i < -std::min(d, 0); ++i) r /= static_cast<long double>(num.seed);
    for (size_t i = 0; i < q.size(); ++i) {
        const int ne = i < num.den.size() ? num.den[i] : 0;
        const int de = i < den.den.size() ? den.den[i] : 0;
        const int diff = de - ne;
        for (int e = 0; e < diff; ++e) r *= static_cast<long double>(q[i]);
        for (int e = 0; e < -diff; ++e) r /= static_cast<long double>(q[i]);
    }
    const long double f = std::floor(r);
    if (!std::isfinite(f) || f < 0.0L || f > static_cast<long double>(std::numeric_limits<uint64_t>::max()))
        throw std::runtime_error("ckks_evalchebyshev: exact-scale ratio exceeds uint64_t");
    return static_cast<uint64_t>(f);
}

struct SimOperand {
    size_t level = 0;
    long double scale = 0.0L;
};

struct Poly {
    std::vector<double> coeffs;
    size_t max_degree = 0;
    bool lead = true;
    size_t level = 0;
    long double scale = 0.0L;
    bool even = false, odd = false;
    size_t degree() const { return coeffs.empty() ? 0 : coeffs.size() - 1; }
};

// Scale / level simulation and the recursive plan (leaves in evaluation order).
class Planner {
public:
    explicit Planner(const std::vector<uint64_t>& q) : q_(q) {}

    void rescale(SimOperand& o) const {
        o.scale /= static_cast<long double>(q_[o.level]);
        --o.level;
    }
    SimOperand mul(const SimOperand& x, const SimOperand& y) const {
        return SimOperand{std::min(x.level, y.level), x.scale * y.scale};
    }
    void powers(size_t n, std::map<size_t, SimOperand>& pb) const {
        if (n < 2 || pb.count(n)) return;
        const auto [a, b] = split_degree(n);
        powers(a, pb);
        powers(b, pb);
        pb[n] = mul(pb.at(a), pb.at(b));
        rescale(pb.at(n));
    }

    std::pair<std::vector<Poly>, SimOperand> plan(size_t log_split, size_t target_level, const Poly& poly,
                                                  const std::map<size_t, SimOperand>& pb, long double out_scale) const {
        const size_t degree = poly.degree();
        const size_t base = size_t{1} << log_split;
        if (degree < base) {
            if (poly.lead && log_split > 1 &&
                poly.max_degree > ((size_t{1} << bit_length(poly.max_degree)) - (size_t{1} << (log_split - 1))))
                return plan(split_log(bit_length(degree)), target_level, poly, pb, out_scale);
            Poly leaf = poly;
            leaf.level = target_level;
            leaf.scale = poly.lead ? out_scale * static_cast<long double>(q_[target_level]) : out_scale;
            return {std::vector<Poly>{leaf}, SimOperand{leaf.level, leaf.scale}};
        }
        size_t next = base;
        while (next < (degree >> 1) + 1) next <<= 1;
        const SimOperand& xpow = pb.at(next);
        const auto [quot, rem] = factorize(poly, next);
        const uint64_t qi = poly.lead ? q_[target_level] : q_[target_level + 1];
        const long double qscale = out_scale * static_cast<long double>(qi) / xpow.scale;
        auto [qv, res] = plan(log_split, target_level + 1, quot, pb, qscale);
        rescale(res);
        res = mul(res, xpow);
        auto [rv, tmp] = plan(log_split, target_level, rem, pb, res.scale);
        if (!scales_close(static_cast<double>(res.scale), static_cast<double>(tmp.scale)))
            throw std::runtime_error("ckks_evalchebyshev: simulated PS scale mismatch");
        qv.insert(qv.end(), rv.begin(), rv.end());
        return {std::move(qv), res};
    }

private:
    static std::pair<Poly, Poly> factorize(const Poly& p, size_t split) {
        const size_t degree = p.degree();
        if (split < (degree >> 1)) throw std::invalid_argument("ckks_evalchebyshev: invalid recursive PS split");
        Poly quot, rem;
        quot.coeffs.assign(degree - split + 1, 0.0);
        rem.coeffs.assign(split, 0.0);
        for (size_t i = 0; i < split && i < p.coeffs.size(); ++i) rem.coeffs[i] = p.coeffs[i];
        if (split < p.coeffs.size()) quot.coeffs[0] = p.coeffs[split];
        for (size_t i = split + 1, j = 1; i <= degree; ++i, ++j) {
            const double c = p.coeffs[i];
            if (c == 0.0) continue;
            quot.coeffs[i - split] += 2.0 * c;
            rem.coeffs[split - j] -= c;
        }
        quot.max_degree = p.max_degree;
        quot.lead = p.lead;
        quot.even = p.even;
        quot.odd = p.odd;
        rem.max_degree = p.max_degree == degree ? (split == 0 ? 0 : split - 1) : p.max_degree - (degree - split + 1);
        rem.lead = false;
        rem.even = p.even;
        rem.odd = p.odd;
        return {std::move(quot), std::move(rem)};
    }

    const std::vector<uint64_t>& q_;
};

// ------------------------------------------------------------------------------------------
// The evaluation
// ------------------------------------------------------------------------------------------
class ChebyshevEval {
public:
    ChebyshevEval(Context& c, DeviceOps& ops, long double default_scale)
        : c_(c), ops_(ops), default_scale_(default_scale) {}

    CtBatch run(const CtBatch& x, const std::vector<double>& coeffs, size_t degree, double target_scale) {
        Poly poly;
        poly.coeffs.assign(coeffs.begin(), coeffs.begin() + degree + 1);
        poly.max_degree = degree;
        poly.lead = true;
        poly.even = parity(coeffs, 1);
        poly.odd = parity(coeffs, 0);
        const size_t log_degree = bit_length(degree);
        const size_t log_split = split_log(log_degree);

        values_.emplace(1, ops_.clone(x));
        exact_.emplace(1, ExactScale::of(static_cast<double>(x.scale), c_.q.size()));
        gen_power(size_t{1} << (log_degree - 1));
        for (size_t i = (size_t{1} << log_split) - 1; i > 2; --i)
            if ((!poly.even && !poly.odd) || ((i & 1U) == 0U && poly.even) || ((i & 1U) == 1U && poly.odd))
                gen_power(i);

        // plan
        Planner pl(c_.q);
        std::map<size_t, SimOperand> sim;
        sim[1] = SimOperand{x.level, x.scale};
        pl.powers(size_t{1} << log_degree, sim);
        auto leaves = pl.plan(log_split, x.level - eval_depth(degree), poly, sim,
                              static_cast<long double>(target_scale)).first;

        // baby steps (stored in reverse order), then giant-step merges
        struct Step {
            size_t degree;
            std::optional<CtBatch> value;
        };
        const size_t split = leaves.size();
        std::vector<std::optional<Step>> steps(split);
        for (size_t i = 0; i < split; ++i)
            steps[split - i - 1] = Step{leaves[i].degree(), eval_leaf(leaves[i].level, leaves[i])};
        while (steps.size() != 1) {
            std::vector<int> kind(steps.size(), 0);
            for (size_t i = 0; i < steps.size(); ++i) {
                if (i == steps.size() - 1) {
                    kind[i] = 2;
                } else if (steps[i]->degree == steps[i + 1]->degree) {
                    kind[i] = 1;
                    ++i;
                }
            }
            for (size_t i = 0; i < steps.size(); ++i) {
                if (kind[i] == 2) {
                    steps[i]->degree = steps[i - 1]->degree;
                } else if (kind[i] == 1) {
                    Step& even = *steps[i];
                    Step& odd = *steps[i + 1];
                    const size_t deg = size_t{1} << bit_length(even.degree);
                    monomial(*even.value, *odd.value, values_.at(deg));
                    odd.degree = 2 * deg - 1;
                    steps[i].reset();
                    ++i;
                }
            }
            size_t w = 0;
            for (size_t i = 0; i < steps.size(); ++i)
                if (steps[i].has_value()) {
                    if (w != i) steps[w] = std::move(steps[i]);
                    ++w;
                }
            steps.resize(w);
        }
        CtBatch out = std::move(*steps.front()->value);
        if (out.np == 3) ops_.relin(out);
        ops_.rescale(out);
        out.scale = static_cast<long double>(target_scale);
        return out;
    }

private:
    static bool parity(const std::vector<double>& coeffs, size_t first) {
        for (size_t i = first; i < coeffs.size(); i += 2)
            if (coeffs[i] != 0.0) return false;
        return true;
    }

    std::vector<uint64_t> constants(double value, long double scale, size_t level) const {
        std::vector<uint64_t> v(level + 1);
        for (size_t l = 0; l <= level; ++l) v[l] = scaled_constant_mod(value, scale, c_.q[l]);
        return v;
    }

    void add_constant(CtBatch& x, double value, long double scale) {
        if (value == 0.0) return;
        ops_.scalar(x, nullptr, constants(value, scale, x.level), kScalarAdd);
    }

    // the integer of multiply_by_integer_scalar_inplace, with its checks
    static uint64_t checked_integer(long double scalar) {
        if (!std::isfinite(scalar) || scalar < 0.0L) throw std::invalid_argument("ckks_evalchebyshev: invalid scalar scale-up");
        const long double r = std::round(scalar);
        if (r < 1.0L || std::abs(scalar - r) > std::max<long double>(1.0L, std::abs(scalar)) * 0x1p-20L)
            throw std::invalid_argument("ckks_evalchebyshev: non-integral scalar scale-up");
        if (r > static_cast<long double>(std::numeric_limits<uint64_t>::max()))
            throw std::invalid_argument("ckks_evalchebyshev: scalar scale-up is too large");
        return static_cast<uint64_t>(r);
    }

    // multiply_by_integer_scalar_inplace
    void mul_integer(CtBatch& x, long double scalar, long double out_scale) {
        const uint64_t s = checked_integer(scalar);
        if (s != 1) {
            std::vector<uint64_t> v(x.level + 1);
            for (size_t l = 0; l <= x.level; ++l) v[l] = s % c_.q[l];
            ops_.scalar(x, nullptr, v, kScalarMul);
        }
        x.scale = static_cast<double>(out_scale);
    }

    long double rescale_product(size_t level) const {
        const size_t levels = std::log2(default_scale_) <= 64.0 ? 1 : 2;
        if (level + 1 < levels) throw std::invalid_argument("ckks_evalchebyshev: insufficient level for rescale modulus product");
        long double s = 1.0L;
        for (size_t i = 0; i < levels; ++i) s *= static_cast<long double>(c_.q[level - i]);
        return s;
    }

    void align(CtBatch& x, size_t level, double scale, int np) {
        if (level > x.level) throw std::invalid_argument("ckks_drop_to_level_inplace: cannot raise ciphertext level");
        x.level = level;
        x.scale = scale;
        ops_.pad(x, np);
    }

    // A leaf of the Paterson-Stockmeyer evaluation, accumulated lazily: its metadata (level,
    // polynomial count, scale) follows the reference's steps one by one, while the data steps
    // (constant adds, multiply-adds of the powers, integer scale-ups of the running sum) are
    // folded into one constant per power and limb and formed by one linear-combination launch.
    // Every step is an exact modular operation on canonical residues, so the sum equals the
    // step-by-step result.
    struct Leaf {
        size_t level;
        int np;
        long double scale;
        std::vector<uint64_t> cadd;
        std::vector<DeviceOps::LinTerm> terms;
    };

    static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((unsigned __int128)a * b % q); }

    void leaf_align(Leaf& r, size_t level, double scale, int np) {
        if (level > r.level) throw std::invalid_argument("ckks_drop_to_level_inplace: cannot raise ciphertext level");
        if (np < r.np) throw std::invalid_argument("ckks_evalchebyshev: cannot shrink ciphertext degree by padding");
        r.level = level;
        r.scale = scale;
        r.np = np;
    }

    void leaf_add_constant(Leaf& r, double value, long double scale) {
        if (value == 0.0) return;
        const std::vector<uint64_t> v = constants(value, scale, r.level);
        for (size_t l = 0; l <= r.level; ++l) r.cadd[l] = add_mod(r.cadd[l], v[l], c_.q[l]);
    }

    // multiply_by_integer_scalar_inplace on the running sum
    void leaf_mul_integer(Leaf& r, long double scalar, long double out_scale) {
        const uint64_t s = checked_integer(scalar);
        if (s != 1)
            for (size_t l = 0; l <= r.level; ++l) {
                const uint64_t q = c_.q[l], sl = s % q;
                r.cadd[l] = mulmod(r.cadd[l], sl, q);
                for (auto& t : r.terms) t.c[l] = mulmod(t.c[l], sl, q);
            }
        r.scale = static_cast<double>(out_scale);
    }

    void leaf_scale_up_to(Leaf& r, long double target) {
        const double cur = static_cast<double>(r.scale), tgt = static_cast<double>(target);
        const double m = std::max({1.0, std::abs(cur), std::abs(tgt)});
        if (std::isfinite(cur) && std::isfinite(tgt) && std::abs(cur - tgt) <= 0x1p-45 * m) {
            r.scale = static_cast<double>(target);
            return;
        }
        if (r.scale > target) throw std::invalid_argument("ckks_evalchebyshev: cannot scale down ciphertext during scale alignment");
        leaf_mul_integer(r, target / r.scale, target);
    }

    // multhenadd_real_scalar_scale_aware_inplace: out += scalar * x, scales reconciled.
    void leaf_mul_then_add(const CtBatch& x, double scalar, Leaf& out) {
        if (scalar == 0.0) return;
        const size_t level = std::min(x.level, out.level);
        const double out_scale = static_cast<double>(out.scale);
        const int np = std::max(x.np, out.np);
        leaf_align(out, level, out_scale, np);
        // x aligned to (level, its own scale): metadata only, x's buffers are read as they are
        CtBatch xa = x;
        xa.level = level;
        xa.scale = static_cast<double>(x.scale);
        long double scale_rlwe = 0.0L;
        if (scales_close(static_cast<double>(xa.scale), static_cast<double>(out.scale))) {
            if (is_integer(scalar)) {
                scale_rlwe = 1.0L;
            } else {
                scale_rlwe = rescale_product(level);
                leaf_scale_up_to(out, out.scale * scale_rlwe);
            }
        } else if (xa.scale < out.scale) {
            scale_rlwe = out.scale / xa.scale;
        } else {
            throw std::invalid_argument("ckks_evalchebyshev: MulThenAdd requires op0.Scale <= opOut.Scale");
        }
        const long double term_scale = xa.scale * scale_rlwe;
        if (!scales_close(static_cast<double>(term_scale), static_cast<double>(out.scale)))
            throw std::runtime_error("ckks_evalchebyshev: MulThenAdd scale mismatch");
        out.terms.push_back({xa, constants(scalar, scale_rlwe, out.level)});
    }

    CtBatch eval_leaf(size_t target_level, const Poly& p) {
        const size_t degree = p.degree();
        Leaf r{target_level, 2, static_cast<double>(p.scale), std::vector<uint64_t>(target_level + 1, 0), {}};
        if (p.even && p.coeffs[0] != 0.0) leaf_add_constant(r, p.coeffs[0], p.scale);
        if (degree > 0)
            for (size_t e = degree; e > 0; --e) {
                const double cf = p.coeffs[e];
                if (cf == 0.0) continue;
                if (!((!p.even && !p.odd) || ((e & 1U) == 0U && p.even) || ((e & 1U) == 1U && p.odd))) continue;
                leaf_align(r, target_level, static_cast<double>(p.scale), r.np);
                leaf_mul_then_add(values_.at(e), cf, r);
            }
        return ops_.lincomb(r.level, r.np, r.scale, r.cadd, r.terms);
    }

    // evaluate_monomial: odd <- even + rescale(relin(odd)) * xpow
    void monomial(CtBatch& even, CtBatch& odd, const CtBatch& xpow) {
        if (odd.np == 3) ops_.relin(odd);
        ops_.rescale(odd);
        CtBatch xp = xpow;  // read only by the tensor product
        if (odd.level > xp.level) throw std::invalid_argument("ckks_drop_to_level_inplace: cannot raise ciphertext level");
        xp.level = odd.level;
        const long double prod = odd.scale * xp.scale;
        ops_.tensor(odd, xp);
        odd.scale = prod;
        align(even, odd.level, static_cast<double>(even.scale), odd.np);
        if (!scales_close(static_cast<double>(even.scale), static_cast<double>(odd.scale)))
            throw std::runtime_error("ckks_evalchebyshev: EvaluateMonomial scale mismatch");
        const double common = static_cast<double>(std::max(even.scale, odd.scale));
        even.scale = common;
        odd.scale = common;
        ops_.add(odd, even, false);
    }

    void rescale_power(size_t n) {
        CtBatch& v = values_.at(n);
        const size_t before = v.level;
        ops_.rescale(v);
        ExactScale& e = exact_.at(n);
        if (e.den.size() < before + 1) e.den.resize(before + 1, 0);
        e.den[before] += 1;
        v.scale = e.value_d(c_.q);
    }

    void gen_power(size_t n) {
        if (n < 2 || values_.count(n)) return;
        if (gen_power_rec(n)) rescale_power(n);
    }

    bool gen_power_rec(size_t n) {
        if (values_.count(n)) return false;
        const auto [a, b] = split_degree(n);
        const bool ra = gen_power_rec(a);
        const bool rb = gen_power_rec(b);
        if (ra) rescale_power(a);
        if (rb) rescale_power(b);
        CtBatch out = ops_.clone(values_.at(a));
        const size_t level = a == b ? out.level : std::min(out.level, values_.at(b).level);
        out.level = level;
        const ExactScale prod = times(exact_.at(a), exact_.at(b));
        CtBatch rhs = values_.at(b);  // read only by the tensor product (out is a fresh copy)
        rhs.level = level;
        ops_.tensor(out, rhs);
        ops_.relin(out);
        out.scale = prod.value_d(c_.q);
        mul_integer(out, 2.0L, prod.value(c_.q));
        const size_t cdeg = a > b ? a - b : b - a;
        if (cdeg == 0) {
            add_constant(out, -1.0, prod.value(c_.q));
        } else {
            gen_power(cdeg);
            // out -= ratio * T_cdeg as one multiply-add by -ratio (T_cdeg itself is only read)
            CtBatch corr = values_.at(cdeg);
            const uint64_t ratio = ratio_u64(prod, exact_.at(cdeg), c_.q);
            corr.scale = exact_.at(cdeg).value_d(c_.q);
            align(corr, out.level, static_cast<double>(corr.scale), out.np);
            const uint64_t s = checked_integer(static_cast<long double>(ratio));
            if (s == 1) {
                ops_.add(out, corr, true);
            } else {
                std::vector<uint64_t> v(out.level + 1);
                for (size_t l = 0; l <= out.level; ++l) v[l] = (c_.q[l] - s % c_.q[l]) % c_.q[l];
                ops_.scalar(out, &corr, v, kScalarMulAdd);
            }
        }
        values_.insert_or_assign(n, std::move(out));
        exact_.insert_or_assign(n, prod);
        return true;
    }

    Context& c_;
    DeviceOps& ops_;
    long double default_scale_;
    std::map<size_t, CtBatch> values_;
    std::map<size_t, ExactScale> exact_;
};

// ckks_evalchebyshev_preconditioned on a batch (the input is read only).
CtBatch chebyshev(Context& c, DeviceOps& ops, const CtBatch& x, const double* coeffs, size_t ncoeffs,
                  double target_scale, double default_scale) {
    if (ncoeffs == 0) throw std::invalid_argument("ckks_evalpoly: polynomial must have at least one coefficient");
    std::vector<double> cf(coeffs, coeffs + ncoeffs);
    for (double v : cf)
        if (!std::isfinite(v)) throw std::invalid_argument("ckks_evalpoly: polynomial coefficients must be finite");
    size_t degree = 0;
    for (size_t i = cf.size(); i > 0; --i)
        if (cf[i - 1] != 0.0) {
            degree = i - 1;
            break;
        }
    const double tgt = target_scale > 0.0 ? target_scale : static_cast<double>(x.scale);
    if (!std::isfinite(tgt) || tgt <= 0.0) throw std::invalid_argument("ckks_evalpoly: invalid scale");
    if (x.level >= c.nq) throw std::invalid_argument("ckks_evalpoly: invalid ciphertext level");
    if (x.level < ceil_log2(degree))
        throw std::invalid_argument(
            "ckks_evalchebyshev_preconditioned: ciphertext level is too small for Chebyshev evaluation depth");
    if (degree == 0) {
        CtBatch out = ops.zeros(x.level, tgt);
        if (cf[0] != 0.0) {
            std::vector<uint64_t> v(x.level + 1);
            for (size_t l = 0; l <= x.level; ++l)
                v[l] = scaled_constant_mod(cf[0], static_cast<long double>(tgt), c.q[l]);
            ops.scalar(out, nullptr, v, kScalarAdd);
        }
        return out;
    }
    if (x.level < eval_depth(degree)) throw std::invalid_argument("ckks_evalchebyshev: insufficient level for polynomial depth");
    ChebyshevEval ev(c, ops, static_cast<long double>(default_scale));
    return ev.run(x, cf, degree, tgt);
}

// multiply_by_real_scalar_to_scale_inplace (ckks_bootstrap_evalmod_inplace.cpp:220-263)
void mul_real_to_scale(Context& c, DeviceOps& ops, CtBatch& x, double scalar, long double out_scale) {
    if (!std::isfinite(scalar) || !std::isfinite(out_scale) || out_scale <= 0.0L || x.scale <= 0.0L)
        throw std::invalid_argument("evalmod_binary_inplace: invalid double-angle scalar scaling");
    const long double ss = out_scale / x.scale;
    std::vector<uint64_t> v(x.level + 1);
    for (size_t l = 0; l <= x.level; ++l) v[l] = scaled_constant_mod(scalar, ss, c.q[l]);
    ops.scalar(x, nullptr, v, kScalarMul);
    x.scale = static_cast<double>(out_scale);
}

}  // namespace

// ckks_batch_bootstrap_evalmod_from_complex_packed (ckks_bootstrap_evalmod_inplace.cpp:265-434)
// for a batch of packed ciphertexts at level p.s2c_depth whose scale equals p.scale:
// SlotToCoeff, dense-to-sparse switch, ModRaise to p.depth, sparse-to-dense switch, sparse-slot
// trace, CoeffToSlot, conjugate split into (ct + conj) and -i (ct - conj), then EvalMod (the
// Chebyshev series at scale 2^evalmod_log_scale, then the double-angle steps) on both halves
// as one batch of 2 x count.  b[i] / a[i] need room for depth+1 limbs and are overwritten.
void bootstrap_evalmod(Context& c, const BootstrapParams& p, const S2cPlan* plans, size_t nplans,
                       const LtStage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs, size_t count,
                       double in_scale, uint64_t* const* b, uint64_t* const* a, uint64_t* const* out0_b,
                       uint64_t* const* out0_a, uint64_t* const* out1_b, uint64_t* const* out1_a, size_t* out_level,
                       double* out_scale, cudaStream_t s) {
    if (count == 0) return;
    if (p.s2c_depth == 0 || p.depth >= c.nq || p.depth < p.s2c_depth)
        throw std::invalid_argument("ckks EvalMod: invalid bootstrap depths");
    // evalmod_input_scale_ratio: the SlotToCoeff plan depends on input scale / parameter scale
    const long double s2c_target = p.scale, input = in_scale;
    if (!std::isfinite(input) || input <= 0.0L) throw std::invalid_argument("ckks EvalMod: invalid ciphertext scale");
    if (input < s2c_target) throw std::invalid_argument("ckks EvalMod: EvalMod input scale is below the S2C target scale");
    const long double ratio = input / s2c_target, rounded = std::round(ratio);
    if (rounded < 1.0L || rounded > static_cast<long double>(std::numeric_limits<uint64_t>::max()) ||
        std::abs(ratio - rounded) > std::max<long double>(1.0L, std::abs(ratio)) * 1e-3L)
        throw std::invalid_argument("ckks EvalMod: EvalMod entry scale ratio is not an exact integer");
    const S2cPlan* plan = nullptr;
    for (size_t k = 0; k < nplans; ++k)
        if (plans[k].ratio == static_cast<uint64_t>(rounded)) plan = &plans[k];
    if (!plan) throw std::invalid_argument("ckks EvalMod: no SlotToCoeff plan for this input scale ratio");
    const LtStage* const* s2c = plan->stages;
    const size_t ns2c = plan->n;
    const size_t N = c.N;
    size_t level = p.s2c_depth;
    // SlotToCoeff
    for (size_t k = 0; k < ns2c; ++k) {
        WG_SPAN("boot.s2c");
        if (lt_stage_level(*s2c[k]) != level) throw std::invalid_argument("ckks_linear_transform: stage level mismatch");
        lt_stage_apply(c, *s2c[k], count, b, a, s);
        if (lt_stage_rescales(*s2c[k])) --level;
    }
    if (level != 0) throw std::invalid_argument("ckks EvalMod: SlotToCoeff must end at level 0");
    // secret switch, ModRaise, switch back
    q0p0_switch(c, count, b, a, c.key(WG_KEY_DENSE_TO_SPARSE, 0), s);
    modraise(c, count, p.depth, b, a, s);
    level = p.depth;
    {
        const KeyEntry& k = c.key(WG_KEY_SPARSE_TO_DENSE, 0);
        std::vector<KsItem> items(count);
        for (size_t i = 0; i < count; ++i) {
            KsItem& it = items[i];
            it.level = level;
            it.key_term = a[i];
            it.key = &k;
            it.b_in = b[i];
            it.a_in = a[i];
            it.b = b[i];
            it.a = a[i];
            it.b_add = 1;
            it.a_add = 0;
            it.galois = 0;
        }
        batch_keyswitch(c, items.data(), count, s);
    }
    DeviceOps ops(c, count, s);
    // sparse-slot trace: ct += rotate(ct, r) for r = active, 2 active, ... < slots
    for (size_t r = p.active_slots; r < p.slots; r <<= 1) {
        WG_SPAN("boot.trace");
        CtBatch x = ops.wrap(b, a, level, 0.0L);
        CtBatch rot = ops.clone(x);
        const KeyEntry& k = c.key(WG_KEY_ROTATION, (int64_t)r);
        std::vector<KsItem> items(count);
        for (size_t i = 0; i < count; ++i) {
            KsItem& it = items[i];
            it.level = level;
            it.key_term = rot.p[i][1];
            it.key = &k;
            it.b_in = rot.p[i][0];
            it.a_in = rot.p[i][1];
            it.b = rot.p[i][0];
            it.a = rot.p[i][1];
            it.b_add = 1;
            it.a_add = 0;
            it.galois = host::powmod(5, r, 2 * N);
        }
        batch_keyswitch(c, items.data(), count, s);
        ops.add(x, rot, false);
    }
    // CoeffToSlot
    for (size_t k = 0; k < nc2s; ++k) {
        WG_SPAN("boot.c2s");
        if (lt_stage_level(*c2s[k]) != level) throw std::invalid_argument("ckks_linear_transform: stage level mismatch");
        lt_stage_apply(c, *c2s[k], count, b, a, s);
        if (lt_stage_rescales(*c2s[k])) --level;
    }
    // conjugate split into the 2 x count EvalMod batch (out0 rows, then out1 rows)
    CtBatch packed = ops.wrap(b, a, level, 0.0L);
    CtBatch conj = ops.conjugate(packed);
    std::vector<uint64_t*> eb(2 * count), ea(2 * count);
    for (size_t i = 0; i < count; ++i) {
        eb[i] = out0_b[i];
        ea[i] = out0_a[i];
        eb[count + i] = out1_b[i];
        ea[count + i] = out1_a[i];
        for (int poly = 0; poly < 2; ++poly) {
            uint64_t* dst0 = poly ? out0_a[i] : out0_b[i];
            uint64_t* dst1 = poly ? out1_a[i] : out1_b[i];
            check_cuda(cudaMemcpyAsync(dst0, packed.p[i][poly], (level + 1) * N * 8, cudaMemcpyDeviceToDevice, s), "split");
            check_cuda(cudaMemcpyAsync(dst1, packed.p[i][poly], (level + 1) * N * 8, cudaMemcpyDeviceToDevice, s), "split");
        }
    }
    {
        CtBatch o0 = ops.wrap(out0_b, out0_a, level, 0.0L);
        CtBatch o1 = ops.wrap(out1_b, out1_a, level, 0.0L);
        ops.add(o0, conj, false);
        ops.add(o1, conj, true);
        ops.mul_complex_constant(o1, 0.0, -1.0, 1.0);
    }
    // EvalMod on both halves at once
    DeviceOps ops2(c, 2 * count, s);
    CtBatch x = ops2.wrap(eb.data(), ea.data(), level, static_cast<long double>(std::exp2((double)p.evalmod_log_scale)));
    CtBatch y = [&] {
        WG_SPAN("boot.evalmod");
        return chebyshev(c, ops2, x, coeffs, ncoeffs, p.scale, p.scale);
    }();
    y.scale = p.scale;
    const long double target = y.scale;
    for (size_t i = 0; i < p.double_angle; ++i) {
        if (y.level == 0) throw std::invalid_argument("evalmod_binary_inplace: insufficient level for BinBoot double-angle");
        CtBatch sq = ops2.clone(y);
        CtBatch sq2 = ops2.clone(y);
        const long double prod = sq.scale * sq.scale;
        ops2.tensor(sq, sq2);
        sq.scale = prod;
        ops2.relin(sq);
        ops2.rescale(sq);
        mul_real_to_scale(c, ops2, sq, -4.0, target);
        y.level = sq.level;
        mul_real_to_scale(c, ops2, y, 4.0, target);
        ops2.add(y, sq, false);
        y.scale = target;
    }
    y.scale = p.scale;
    ops2.copy_out(y, eb.data(), ea.data());
    *out_level = y.level;
    *out_scale = static_cast<double>(y.scale);
}

void evalchebyshev(Context& c, size_t count, size_t level, double scale, const double* coeffs, size_t ncoeffs,
                   double target_scale, double default_scale, uint64_t* const* b, uint64_t* const* a,
                   uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                   cudaStream_t s) {
    if (level >= c.nq) throw std::invalid_argument("ckks_evalpoly: invalid ciphertext level");
    if (count == 0) return;
    DeviceOps ops(c, count, s);
    CtBatch x = ops.wrap(b, a, level, static_cast<long double>(scale));
    CtBatch out = chebyshev(c, ops, x, coeffs, ncoeffs, target_scale, default_scale);
    ops.copy_out(out, out_b, out_a);
    *out_level = out.level;
    *out_scale = static_cast<double>(out.scale);
}

}  // namespace wg
