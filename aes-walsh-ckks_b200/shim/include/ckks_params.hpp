// CKKS parameter sets, as the reference declares them (src/ckks/parameters/ckks_params.hpp):
// the same configuration records and CKKSParams interface, so code written against the
// reference builds unchanged.  The modulus chain, depth and bootstrap schedule are derived by
// the same rules (ckks_params.cpp in the reference); the primes come from the device library's
// prime search (wg_find_primes), which is the reference's.
#ifndef CKKS_PARAMS_HPP
#define CKKS_PARAMS_HPP

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "aligned_vector.hpp"

using CKKSBootstrapDftScaleSchedule = std::vector<std::vector<size_t>>;

inline constexpr size_t kAutoEvalModDiscreteValidationPointsPerInterval = 64;
inline constexpr double kAutoBinBootDiscreteIntervalRadius = 1.0 / 32.0;

inline double automatic_binboot_discrete_interval_radius(size_t log_message_ratio) {
    if (log_message_ratio == 0) return kAutoBinBootDiscreteIntervalRadius;
    if (log_message_ratio >= static_cast<size_t>(std::numeric_limits<double>::max_exponent))
        return std::numeric_limits<double>::min();
    const double radius = std::ldexp(1.0, -static_cast<int>(log_message_ratio));
    return radius < std::nextafter(0.25, 0.0) ? radius : std::nextafter(0.25, 0.0);
}

struct CKKSBootstrapParams {
    size_t sparse_secret_hamming_weight = 0;
    // Logical slot count of sparse bootstrap DFTs; 0 means N/2.
    size_t active_slot_count = 0;
    std::array<size_t, 2> linear_transform_depths{0, 0};
    std::array<CKKSBootstrapDftScaleSchedule, 2> linear_transform_log_plaintext_scales;
    size_t evalmod_depth = 0;
    size_t evalmod_bit_size = 0;
    // 0 means derived from the sparse-secret overflow bound.
    size_t evalmod_k = 0;
    long double evalmod_k_failure_probability_log2 = -128.0L;
    size_t evalmod_polynomial_degree = 120;
    size_t evalmod_double_angle = 0;
    size_t evalmod_log_message_ratio = 0;
    double evalmod_coefficient_prune_threshold = 1e-10;
    double evalmod_discrete_interval_radius = 0.0;
    size_t evalmod_discrete_validation_points_per_interval = 0;
    std::array<size_t, 2> linear_transform_bsgs_baby_step_counts{0, 0};
    std::array<int, 2> linear_transform_log_bsgs_ratios{1, 1};
    std::array<std::vector<size_t>, 2> linear_transform_merge_depths;
    std::array<bool, 2> linear_transform_use_qp{false, false};
};

struct CKKSAesWalshParams {
    bool enabled = false;
    // Active AES blocks per bit ciphertext (also the packed segment stride).
    size_t block_count = 0;
    // Packed segments to provision rotation keys for; 0 means slots / block_count.
    size_t packed_segment_count = 0;
};

struct CKKSParamsConfig {
    double scale = 0.0;
    double sigma = 3.19;
    size_t N = size_t{1} << 15;
    size_t slots = 0;
    size_t depth = 0;
    size_t mult_depth = 0;
    size_t q0_bit = 33;
    size_t q_bit = 32;
    std::vector<uint64_t> q_mult_bits;
    size_t dnum = 3;
    size_t p_bit = 61;
    size_t pmoduli_count = 1;
    std::vector<uint64_t> p_bits;
    size_t secret_key_hamming_weight = 256;
    std::optional<CKKSBootstrapParams> bootstrap_params;
    std::vector<uint64_t> q_bits;
    MyVector<int64_t> rotate_values;
    bool bts_keys = false;
    std::optional<bool> s2c_ptxt;
    std::optional<bool> c2s_ptxt;
    bool secure = true;
    bool fold_hybrid_keyswitch = true;
    bool montgomery = true;
    CKKSAesWalshParams aes_walsh_params;
};

namespace ckks_params_detail {

inline bool is_power_of_two(size_t value) { return value != 0 && (value & (value - 1)) == 0; }

inline CKKSBootstrapParams make_evalmod_bootstrap_params(
    size_t sparse_secret_hamming_weight,
    std::array<CKKSBootstrapDftScaleSchedule, 2> linear_transform_log_plaintext_scales, size_t evalmod_depth,
    size_t evalmod_bit_size = 0, std::array<size_t, 2> linear_transform_bsgs_baby_step_counts = {0, 0}) {
    CKKSBootstrapParams params;
    params.sparse_secret_hamming_weight = sparse_secret_hamming_weight;
    params.linear_transform_log_plaintext_scales = std::move(linear_transform_log_plaintext_scales);
    params.linear_transform_depths = {params.linear_transform_log_plaintext_scales[0].size(),
                                      params.linear_transform_log_plaintext_scales[1].size()};
    params.evalmod_depth = evalmod_depth;
    params.evalmod_bit_size = evalmod_bit_size;
    params.linear_transform_bsgs_baby_step_counts = linear_transform_bsgs_baby_step_counts;
    return params;
}

}  // namespace ckks_params_detail

class CKKSParams {
public:
    explicit CKKSParams(CKKSParamsConfig config);
    static CKKSParams AESWalsh15();
    static CKKSParams XBootParamAes13Reference();
    static CKKSParams AESXBoot14Secure();
    static CKKSParams AESXBoot14SecureSparse1024();
    static CKKSParams AESXBoot15();
    static CKKSParams AESXBoot15Sparse1024();
    bool bts_keys = false;
    bool s2c_ptxt = false;
    bool c2s_ptxt = false;
    bool secure = true;
    bool fold_hybrid_keyswitch = true;
    bool montgomery = true;
    CKKSAesWalshParams aes_walsh_params;
    size_t getN() const;
    size_t getSlots() const;
    double getScale() const;
    double getSigma() const;
    size_t getSecretKeyHammingWeight() const;
    const MyVector<uint64_t>& getModuli() const;
    const std::vector<uint64_t>& getQBits() const;
    size_t getQ0Bit() const;
    size_t getDefaultQBit() const;
    size_t getDnum() const;
    size_t getDepth() const;
    size_t getMaxLevel() const;
    const MyVector<uint64_t>& getPModuli() const;
    const MyVector<int64_t>& getRotateValues() const;
    bool usesAesWalsh() const;
    size_t getAesWalshBlockCount() const;
    size_t getAesWalshPackedSegmentCount() const;
    bool hasBootstrapParams() const;
    const CKKSBootstrapParams& getBootstrapParams() const;
    size_t getBootstrapActiveSlotCount() const;
    bool usesSparseBootstrapSlots() const;
    size_t getBootstrapSparseSecretHammingWeight() const;
    size_t getBootstrapS2CDepth() const;
    size_t getBootstrapC2SDepth() const;
    const CKKSBootstrapDftScaleSchedule& getBootstrapS2CLogPlaintextScales() const;
    const CKKSBootstrapDftScaleSchedule& getBootstrapC2SLogPlaintextScales() const;
    size_t getBootstrapEvalModDepth() const;
    size_t getBootstrapEvalModK() const;
    size_t getBootstrapEvalModPolynomialDegree() const;
    size_t getBootstrapEvalModDoubleAngle() const;
    size_t getBootstrapEvalModLogMessageRatio() const;
    double getBootstrapEvalModCoefficientPruneThreshold() const;
    double getBootstrapEvalModDiscreteIntervalRadius() const;
    size_t getBootstrapEvalModDiscreteValidationPointsPerInterval() const;
    const std::array<size_t, 2>& getBootstrapLinearTransformBsgsBabyStepCounts() const;
    int getBootstrapS2CLogBsgsRatio() const;
    int getBootstrapC2SLogBsgsRatio() const;
    const std::vector<size_t>& getBootstrapS2CMergeDepths() const;
    const std::vector<size_t>& getBootstrapC2SMergeDepths() const;
    bool getBootstrapS2CUseQpLinearTransform() const;
    bool getBootstrapC2SUseQpLinearTransform() const;

private:
    double scale = 0.0;
    double sigma = 3.19;
    size_t N = 0;
    size_t slots = 0;
    size_t limbs_count = 0;
    size_t depth = 0;
    size_t mult_depth = 0;
    size_t q0_bit = 0;
    size_t q_bit = 0;
    std::vector<uint64_t> q_mult_bits;
    size_t dnum = 0;
    size_t secret_key_hamming_weight = 0;
    std::optional<CKKSBootstrapParams> bootstrap_params;
    MyVector<uint64_t> pmoduli;
    MyVector<uint64_t> moduli;
    std::vector<uint64_t> q_bits;
    std::vector<uint64_t> p_bits;
    MyVector<int64_t> rotate_values;

    size_t bootstrapDepth(const CKKSBootstrapParams& params) const;
    std::vector<uint64_t> defaultQBits() const;
    size_t calculateDepth() const;
    const CKKSBootstrapParams& requireBootstrapParams() const;
};

#endif  // CKKS_PARAMS_HPP
