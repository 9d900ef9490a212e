// CKKSParams of the reference API: the configuration checks and derivations of the reference's
// src/ckks/parameters/ckks_params.cpp (chain layout, depth, bootstrap getters, the 128-bit
// log(PQ) bounds), with the primes from the device library's prime search.
#include <numeric>
#include <stdexcept>
#include <string>

#include "../../../include/walsh_gpu.h"
#include "binboot_k_bound.hpp"
#include "ckks_params.hpp"
#include "poly_approx.hpp"

namespace {

size_t linear_transform_depth(const CKKSBootstrapParams& p, size_t which) {
    const auto& sched = p.linear_transform_log_plaintext_scales[which];
    return sched.empty() ? p.linear_transform_depths[which] : sched.size();
}

// One Q limb per scale group, bottom (last group) first; `fallback_depth` limbs of the default
// width when no schedule is given.
void append_group_bits(std::vector<uint64_t>& bits, const CKKSBootstrapDftScaleSchedule& sched, uint64_t fallback,
                       size_t fallback_depth) {
    if (sched.empty()) {
        bits.insert(bits.end(), fallback_depth, fallback);
        return;
    }
    for (size_t r = 0; r < sched.size(); ++r) {
        const auto& g = sched[sched.size() - 1 - r];
        if (g.empty()) throw std::runtime_error("CKKSParams: DFT scale schedule groups must not be empty");
        bits.push_back((uint64_t)std::accumulate(g.begin(), g.end(), size_t{0}));
    }
}

// Largest log2(PQ) with 128-bit security at ring degree N: the Homomorphic Encryption Standard
// table for uniform ternary secrets, the fixed Hamming weight 256 and 192 tables otherwise
// (the reference's ckks_params.hpp:190-229).
size_t max_log_pq(size_t N, size_t h) {
    struct Row {
        size_t n, bits;
    };
    static const Row standard[] = {{1u << 13, 214}, {1u << 14, 430}, {1u << 15, 868}, {1u << 16, 1747}};
    static const Row h256[] = {{1u << 13, 210}, {1u << 14, 422}, {1u << 15, 853}, {1u << 16, 1720}};
    static const Row h192[] = {{1u << 15, 808}};
    const Row* rows = nullptr;
    size_t n = 0;
    if (h == 0) {
        rows = standard;
        n = 4;
    } else if (h == 256) {
        rows = h256;
        n = 4;
    } else if (h == 192) {
        rows = h192;
        n = 1;
    } else {
        throw std::runtime_error(
            "CKKSParams: secure fixed-hamming-weight secrets are only supported for h=192 and h=256; "
            "set secret_key_hamming_weight=0 to use standard uniform ternary validation");
    }
    for (size_t i = 0; i < n; ++i)
        if (rows[i].n == N) return rows[i].bits;
    throw std::runtime_error("CKKSParams: no 128-bit log(PQ) bound for N=" + std::to_string(N));
}

}  // namespace

CKKSParams::CKKSParams(CKKSParamsConfig config) {
    if (!ckks_params_detail::is_power_of_two(config.N))
        throw std::invalid_argument("CKKSParams: N must be a nonzero power of two");
    if (config.slots != 0 && config.slots * 2 != config.N) throw std::invalid_argument("CKKSParams: slots must equal N / 2");
    if (config.q_bits.empty() && config.q_bit == 0)
        throw std::invalid_argument("CKKSParams: q_bit must be positive when q_bits is empty");
    for (uint64_t b : config.p_bits)
        if (b == 0) throw std::invalid_argument("CKKSParams: p_bits entries must be positive");
    if (config.p_bits.empty() && config.pmoduli_count > 0 && config.p_bit == 0)
        throw std::invalid_argument("CKKSParams: p_bit must be positive when P limbs are requested");
    if (config.dnum == 0) throw std::invalid_argument("CKKSParams: dnum must be positive");
    if (!config.q_bits.empty() && !config.q_mult_bits.empty())
        throw std::invalid_argument("CKKSParams: q_bits and q_mult_bits are mutually exclusive");
    if (!config.q_mult_bits.empty()) {
        if (config.q_mult_bits.size() != config.mult_depth)
            throw std::invalid_argument("CKKSParams: q_mult_bits size must equal mult_depth");
        for (uint64_t b : config.q_mult_bits)
            if (b == 0) throw std::invalid_argument("CKKSParams: q_mult_bits entries must be positive");
    }
    secure = config.secure;
    bts_keys = config.bts_keys;
    s2c_ptxt = config.s2c_ptxt.value_or(bts_keys);
    c2s_ptxt = config.c2s_ptxt.value_or(bts_keys);
    fold_hybrid_keyswitch = config.fold_hybrid_keyswitch;
    montgomery = config.montgomery;
    aes_walsh_params = config.aes_walsh_params;
    N = config.N;
    slots = config.slots == 0 ? N / 2 : config.slots;
    mult_depth = config.mult_depth;
    q0_bit = config.q0_bit;
    q_bit = config.q_bit;
    q_mult_bits = std::move(config.q_mult_bits);
    dnum = config.dnum;
    p_bits = config.p_bits.empty() ? std::vector<uint64_t>(config.pmoduli_count, (uint64_t)config.p_bit)
                                   : std::move(config.p_bits);
    secret_key_hamming_weight = config.secret_key_hamming_weight;
    sigma = config.sigma;
    scale = config.scale > 0.0 ? config.scale : std::exp2((double)q_bit);
    rotate_values = std::move(config.rotate_values);
    bootstrap_params = std::move(config.bootstrap_params);
    if (!config.q_bits.empty()) {
        q_bits = std::move(config.q_bits);
        depth = q_bits.size() - 1;
        if (config.depth != 0 && config.depth != depth)
            throw std::invalid_argument("CKKSParams: depth must match q_bits.size() - 1");
        limbs_count = q_bits.size();
    } else {
        depth = config.depth == 0 ? calculateDepth() : config.depth;
        limbs_count = depth + 1;
        q_bits = defaultQBits();
    }
    if (q_bits.size() != limbs_count) throw std::runtime_error("CKKSParams: Q bit schedule must match limb count");
    if (depth != calculateDepth())
        throw std::runtime_error("CKKSParams: depth must equal mult_depth plus requested bootstrap/S2C depths");
    if (secure) {
        size_t log_pq = 0;
        for (uint64_t b : q_bits) log_pq += (size_t)b;
        for (uint64_t b : p_bits) log_pq += (size_t)b;
        const size_t bound = max_log_pq(N, secret_key_hamming_weight);
        if (log_pq > bound)
            throw std::runtime_error("CKKSParams : log(PQ) bit budget " + std::to_string(log_pq) +
                                     " exceeds 128-bit security bound " + std::to_string(bound) +
                                     " for N=" + std::to_string(N));
    }
    std::vector<uint64_t> p(p_bits.size()), q(q_bits.size());
    if (wg_find_primes(p_bits.data(), p_bits.size(), q_bits.data(), q_bits.size(), N, p.data(), q.data()) != WG_OK)
        throw std::runtime_error(std::string("CKKSParams: prime search failed: ") + wg_last_error());
    moduli.assign(q.begin(), q.end());
    pmoduli.assign(p.begin(), p.end());
}

size_t CKKSParams::bootstrapDepth(const CKKSBootstrapParams& p) const {
    return linear_transform_depth(p, 0) + linear_transform_depth(p, 1) + p.evalmod_depth;
}

std::vector<uint64_t> CKKSParams::defaultQBits() const {
    std::vector<uint64_t> bits;
    bits.push_back((uint64_t)q0_bit);
    auto mult = [&] {
        if (q_mult_bits.empty())
            bits.insert(bits.end(), mult_depth, (uint64_t)q_bit);
        else
            bits.insert(bits.end(), q_mult_bits.begin(), q_mult_bits.end());
    };
    if (bts_keys) {
        const auto& b = requireBootstrapParams();
        append_group_bits(bits, b.linear_transform_log_plaintext_scales[0], q_bit, linear_transform_depth(b, 0));
        mult();
        bits.insert(bits.end(), b.evalmod_depth, b.evalmod_bit_size == 0 ? (uint64_t)q_bit : (uint64_t)b.evalmod_bit_size);
        append_group_bits(bits, b.linear_transform_log_plaintext_scales[1], q_bit, linear_transform_depth(b, 1));
    } else if (s2c_ptxt || c2s_ptxt) {
        const auto& b = requireBootstrapParams();
        if (s2c_ptxt) append_group_bits(bits, b.linear_transform_log_plaintext_scales[0], q_bit, linear_transform_depth(b, 0));
        mult();
        if (c2s_ptxt) append_group_bits(bits, b.linear_transform_log_plaintext_scales[1], q_bit, linear_transform_depth(b, 1));
    } else {
        mult();
    }
    return bits;
}

size_t CKKSParams::calculateDepth() const {
    size_t d = mult_depth;
    if (bts_keys) {
        d += bootstrapDepth(requireBootstrapParams());
    } else if (s2c_ptxt || c2s_ptxt) {
        const auto& b = requireBootstrapParams();
        if (s2c_ptxt) d += linear_transform_depth(b, 0);
        if (c2s_ptxt) d += linear_transform_depth(b, 1);
    }
    return d;
}

const CKKSBootstrapParams& CKKSParams::requireBootstrapParams() const {
    if (!bts_keys && !s2c_ptxt && !c2s_ptxt)
        throw std::runtime_error(
            "CKKSParams: bootstrap params are disabled because bts_keys, s2c_ptxt, and c2s_ptxt are false");
    if (!bootstrap_params.has_value()) throw std::runtime_error("CKKSParams: bootstrap parameters are required");
    return *bootstrap_params;
}

size_t CKKSParams::getN() const { return N; }
size_t CKKSParams::getSlots() const {
    if (slots == 0 || slots * 2 != N) throw std::runtime_error("CKKSParams: slots must equal N / 2");
    return slots;
}
double CKKSParams::getScale() const { return scale; }
double CKKSParams::getSigma() const { return sigma; }
size_t CKKSParams::getSecretKeyHammingWeight() const { return secret_key_hamming_weight; }
const MyVector<uint64_t>& CKKSParams::getModuli() const { return moduli; }
const std::vector<uint64_t>& CKKSParams::getQBits() const { return q_bits; }
size_t CKKSParams::getQ0Bit() const { return q0_bit; }
size_t CKKSParams::getDefaultQBit() const { return q_bit; }
size_t CKKSParams::getDnum() const { return dnum; }
size_t CKKSParams::getMaxLevel() const {
    if (limbs_count == 0 || depth + 1 != limbs_count) throw std::runtime_error("CKKSParams: inconsistent limb count");
    if (depth != calculateDepth())
        throw std::runtime_error("CKKSParams: depth must equal mult_depth plus requested bootstrap/S2C depths");
    return depth;
}
size_t CKKSParams::getDepth() const { return getMaxLevel(); }
const MyVector<uint64_t>& CKKSParams::getPModuli() const { return pmoduli; }
const MyVector<int64_t>& CKKSParams::getRotateValues() const { return rotate_values; }
bool CKKSParams::usesAesWalsh() const { return aes_walsh_params.enabled; }
size_t CKKSParams::getAesWalshBlockCount() const { return aes_walsh_params.block_count; }
size_t CKKSParams::getAesWalshPackedSegmentCount() const {
    if (aes_walsh_params.packed_segment_count != 0) return aes_walsh_params.packed_segment_count;
    const size_t bc = getAesWalshBlockCount();
    return bc == 0 ? 0 : getSlots() / bc;
}
bool CKKSParams::hasBootstrapParams() const {
    if (!bts_keys && !s2c_ptxt && !c2s_ptxt) return false;
    requireBootstrapParams();
    return true;
}
const CKKSBootstrapParams& CKKSParams::getBootstrapParams() const { return requireBootstrapParams(); }
size_t CKKSParams::getBootstrapActiveSlotCount() const {
    const size_t full = getSlots();
    const size_t a = requireBootstrapParams().active_slot_count;
    if (a == 0) return full;
    if (!ckks_params_detail::is_power_of_two(a))
        throw std::runtime_error("CKKSParams: bootstrap active slot count must be a power of two");
    if (a > full || full % a) throw std::runtime_error("CKKSParams: bootstrap active slot count must divide N/2 slots");
    return a;
}
bool CKKSParams::usesSparseBootstrapSlots() const { return getBootstrapActiveSlotCount() != getSlots(); }
size_t CKKSParams::getBootstrapSparseSecretHammingWeight() const {
    return requireBootstrapParams().sparse_secret_hamming_weight;
}
size_t CKKSParams::getBootstrapS2CDepth() const { return linear_transform_depth(requireBootstrapParams(), 0); }
size_t CKKSParams::getBootstrapC2SDepth() const { return linear_transform_depth(requireBootstrapParams(), 1); }
const CKKSBootstrapDftScaleSchedule& CKKSParams::getBootstrapS2CLogPlaintextScales() const {
    return requireBootstrapParams().linear_transform_log_plaintext_scales[0];
}
const CKKSBootstrapDftScaleSchedule& CKKSParams::getBootstrapC2SLogPlaintextScales() const {
    return requireBootstrapParams().linear_transform_log_plaintext_scales[1];
}
size_t CKKSParams::getBootstrapEvalModDepth() const { return requireBootstrapParams().evalmod_depth; }
size_t CKKSParams::getBootstrapEvalModK() const {
    const auto& b = requireBootstrapParams();
    if (b.evalmod_k != 0) return b.evalmod_k;
    const long double f = b.evalmod_k_failure_probability_log2;
    if (!std::isfinite(f) || f >= 0.0L)
        throw std::runtime_error("CKKSParams: automatic EvalMod K failure probability log2 must be finite and negative");
    return required_binboot_k_bound(N, getBootstrapSparseSecretHammingWeight(), std::exp2(f)).evalmod_k;
}
size_t CKKSParams::getBootstrapEvalModPolynomialDegree() const {
    const size_t d = requireBootstrapParams().evalmod_polynomial_degree;
    if (d == 0) throw std::runtime_error("CKKSParams: EvalMod polynomial degree must be positive");
    return d;
}
size_t CKKSParams::getBootstrapEvalModDoubleAngle() const { return requireBootstrapParams().evalmod_double_angle; }
size_t CKKSParams::getBootstrapEvalModLogMessageRatio() const {
    return requireBootstrapParams().evalmod_log_message_ratio;
}
double CKKSParams::getBootstrapEvalModCoefficientPruneThreshold() const {
    const double t = requireBootstrapParams().evalmod_coefficient_prune_threshold;
    if (!std::isfinite(t) || t < 0.0) throw std::runtime_error("CKKSParams: invalid EvalMod prune threshold");
    return t;
}
double CKKSParams::getBootstrapEvalModDiscreteIntervalRadius() const {
    const double r = requireBootstrapParams().evalmod_discrete_interval_radius;
    if (!std::isfinite(r) || r < 0.0 || r >= 0.25)
        throw std::runtime_error("CKKSParams: EvalMod discrete interval radius must be in [0, 0.25)");
    return r > 0.0 ? r : automatic_binboot_discrete_interval_radius(getBootstrapEvalModLogMessageRatio());
}
size_t CKKSParams::getBootstrapEvalModDiscreteValidationPointsPerInterval() const {
    const size_t p = requireBootstrapParams().evalmod_discrete_validation_points_per_interval;
    if (p == 0) return kAutoEvalModDiscreteValidationPointsPerInterval;
    if (p < 2) throw std::runtime_error("CKKSParams: EvalMod validation points per interval must be at least 2");
    return p;
}
const std::array<size_t, 2>& CKKSParams::getBootstrapLinearTransformBsgsBabyStepCounts() const {
    return requireBootstrapParams().linear_transform_bsgs_baby_step_counts;
}
int CKKSParams::getBootstrapS2CLogBsgsRatio() const { return requireBootstrapParams().linear_transform_log_bsgs_ratios[0]; }
int CKKSParams::getBootstrapC2SLogBsgsRatio() const { return requireBootstrapParams().linear_transform_log_bsgs_ratios[1]; }
const std::vector<size_t>& CKKSParams::getBootstrapS2CMergeDepths() const {
    return requireBootstrapParams().linear_transform_merge_depths[0];
}
const std::vector<size_t>& CKKSParams::getBootstrapC2SMergeDepths() const {
    return requireBootstrapParams().linear_transform_merge_depths[1];
}
bool CKKSParams::getBootstrapS2CUseQpLinearTransform() const { return requireBootstrapParams().linear_transform_use_qp[0]; }
bool CKKSParams::getBootstrapC2SUseQpLinearTransform() const { return requireBootstrapParams().linear_transform_use_qp[1]; }

BinBootKBound required_binboot_k_bound(size_t coefficient_count, size_t hamming_weight,
                                       long double target_failure_probability) {
    if (!(target_failure_probability > 0.0L) || !(target_failure_probability < 1.0L))
        throw std::invalid_argument("binboot K bound: invalid failure probability");
    size_t k = 0;
    if (wg_evalmod_k_bound(coefficient_count, hamming_weight, (double)std::log2(target_failure_probability), &k) != WG_OK)
        throw std::invalid_argument(wg_last_error());
    BinBootKBound out;
    out.evalmod_k = k;
    out.mathematical_k = k - 1;
    return out;
}

PolynomialApproximation binboot_han_ki_discrete_multi_interval_approximate(double K, size_t degree,
                                                                           size_t double_angle, double interval_radius,
                                                                           size_t points, double prune) {
    PolynomialApproximation a;
    a.chebyshev_coeffs.resize(degree + 1);
    size_t n = 0;
    double iv[2] = {0.0, 0.0};
    if (wg_evalmod_fit(K, degree, double_angle, interval_radius, points, prune, a.chebyshev_coeffs.data(), &n,
                       &a.max_error, iv) != WG_OK)
        throw std::invalid_argument(wg_last_error());
    a.chebyshev_coeffs.resize(n);
    a.interval_min = iv[0];
    a.interval_max = iv[1];
    a.degree = n == 0 ? 0 : n - 1;
    return a;
}
