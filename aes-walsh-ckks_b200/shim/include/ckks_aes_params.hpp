// The AES benchmark's parameter sets (the reference's src/ckks/parameters/ckks_aes_params.hpp):
// the same configurations, value for value, behind the same CKKSParams presets.
#ifndef CKKS_AES_PARAMS_HPP
#define CKKS_AES_PARAMS_HPP

#include <cmath>
#include <cstddef>

#include "binboot_k_bound.hpp"
#include "ckks_params.hpp"

namespace ckks_aes_params_detail {

// EvalMod settings every XBOOT set shares: cosine-discrete fit, no double angle, message ratio
// 2, radius just below 1/4, 64 validation points, no pruning, QP linear transforms.
inline void xboot_evalmod(CKKSBootstrapParams& p, size_t K, size_t degree, std::array<int, 2> log_bsgs) {
    p.evalmod_k = K;
    p.evalmod_polynomial_degree = degree;
    p.evalmod_double_angle = 0;
    p.evalmod_log_message_ratio = 1;
    p.evalmod_coefficient_prune_threshold = 0.0;
    p.evalmod_discrete_interval_radius = std::nextafter(0.25, 0.0);
    p.evalmod_discrete_validation_points_per_interval = 64;
    p.linear_transform_log_bsgs_ratios = log_bsgs;
    p.linear_transform_use_qp = {true, true};
}

inline CKKSBootstrapParams XBootParamAes13ReferenceBootstrapParams() {
    auto p = ckks_params_detail::make_evalmod_bootstrap_params(
        16, {CKKSBootstrapDftScaleSchedule{{28}}, CKKSBootstrapDftScaleSchedule{{28}, {28}}}, 6, 32, {0, 0});
    xboot_evalmod(p, 7, 60, {1, 2});
    return p;
}

inline CKKSBootstrapParams AESWalsh15BootstrapParams() {
    auto p = ckks_params_detail::make_evalmod_bootstrap_params(
        32,
        {CKKSBootstrapDftScaleSchedule{{18, 20, 23}}, CKKSBootstrapDftScaleSchedule{{25, 25}, {25, 25}}}, 7, 38,
        {0, 0});
    p.evalmod_k = required_binboot_k_bound(size_t{1} << 15, p.sparse_secret_hamming_weight, std::exp2(-16.0L)).evalmod_k;
    p.evalmod_polynomial_degree = 100;
    p.evalmod_double_angle = 0;
    p.evalmod_coefficient_prune_threshold = 1e-10;
    p.evalmod_discrete_interval_radius = std::nextafter(0.25, 0.0);
    p.evalmod_discrete_validation_points_per_interval = 128;
    p.linear_transform_log_bsgs_ratios = {1, 1};
    p.linear_transform_use_qp = {true, true};
    return p;
}

inline CKKSParamsConfig AESWalsh15Config() {
    CKKSParamsConfig c;
    c.secure = true;
    c.bts_keys = true;
    c.N = size_t{1} << 15;
    c.mult_depth = 2;
    c.q0_bit = 36;
    c.q_mult_bits = {42, 42};
    c.scale = std::exp2(35);
    c.dnum = 3;
    c.pmoduli_count = 4;
    c.p_bits = {61, 61, 61, 61};
    c.secret_key_hamming_weight = 256;
    c.aes_walsh_params.enabled = true;
    c.aes_walsh_params.block_count = 512;
    c.aes_walsh_params.packed_segment_count = 32;
    c.bootstrap_params = AESWalsh15BootstrapParams();
    return c;
}

inline CKKSParamsConfig XBootParamAes13ReferenceConfig() {
    CKKSParamsConfig c;
    c.secure = false;  // log(PQ) = 433 is above the fixed-h = 256 bound of 422 at N = 2^14
    c.bts_keys = true;
    c.N = size_t{1} << 14;
    c.mult_depth = 3;
    c.q0_bit = 32;
    c.q_bit = 32;
    // base | SlotsToCoeffs | AES round circuit | EvalMod | CoeffsToSlots
    c.q_bits = {32, 28, 31, 31, 31, 32, 32, 32, 32, 32, 32, 28, 28};
    c.scale = std::exp2(31);
    c.dnum = 13;
    c.pmoduli_count = 1;
    c.p_bits = {32};
    c.secret_key_hamming_weight = 256;
    c.bootstrap_params = XBootParamAes13ReferenceBootstrapParams();
    return c;
}

inline CKKSBootstrapParams AESXBoot14SecureBootstrapParams() {
    auto p = ckks_params_detail::make_evalmod_bootstrap_params(
        16, {CKKSBootstrapDftScaleSchedule{{27}}, CKKSBootstrapDftScaleSchedule{{27}, {27}}}, 6, 31, {0, 0});
    xboot_evalmod(p, 7, 60, {1, 2});
    return p;
}

inline CKKSParamsConfig AESXBoot14SecureConfig() {
    auto c = XBootParamAes13ReferenceConfig();
    c.secure = true;
    c.q0_bit = 31;
    c.q_bit = 31;
    c.q_bits = {31, 27, 30, 30, 30, 31, 31, 31, 31, 31, 31, 27, 27};  // each limb one bit below Param-AES-13
    c.scale = std::exp2(30);
    c.bootstrap_params = AESXBoot14SecureBootstrapParams();
    return c;
}

inline CKKSParamsConfig AESXBoot14SecureSparse1024Config() {
    auto c = AESXBoot14SecureConfig();
    c.bootstrap_params->active_slot_count = 1024;
    return c;
}

inline CKKSBootstrapParams AESXBoot15BootstrapParams() {
    auto p = ckks_params_detail::make_evalmod_bootstrap_params(
        32,
        {CKKSBootstrapDftScaleSchedule{{36}, {36}}, CKKSBootstrapDftScaleSchedule{{38}, {38}, {38}, {38}}}, 7, 38,
        {0, 0});
    xboot_evalmod(p, 12, 120, {2, 1});
    return p;
}

inline CKKSParamsConfig AESXBoot15Config() {
    CKKSParamsConfig c;
    c.secure = true;
    c.bts_keys = true;
    c.N = size_t{1} << 15;
    c.mult_depth = 3;
    c.q0_bit = 38;
    c.q_bit = 38;
    c.q_bits = {38, 36, 36, 37, 37, 37, 38, 38, 38, 38, 38, 38, 38, 38, 38, 38, 38};
    c.scale = std::exp2(37);
    c.dnum = 5;
    c.pmoduli_count = 5;
    c.p_bits = {38, 38, 38, 38, 38};
    c.secret_key_hamming_weight = 256;
    c.bootstrap_params = AESXBoot15BootstrapParams();
    return c;
}

inline CKKSParamsConfig AESXBoot15Sparse1024Config() {
    auto c = AESXBoot15Config();
    c.bootstrap_params->active_slot_count = 1024;
    return c;
}

}  // namespace ckks_aes_params_detail

inline CKKSParams CKKSParams::AESWalsh15() { return CKKSParams(ckks_aes_params_detail::AESWalsh15Config()); }
inline CKKSParams CKKSParams::XBootParamAes13Reference() {
    return CKKSParams(ckks_aes_params_detail::XBootParamAes13ReferenceConfig());
}
inline CKKSParams CKKSParams::AESXBoot14Secure() {
    return CKKSParams(ckks_aes_params_detail::AESXBoot14SecureConfig());
}
inline CKKSParams CKKSParams::AESXBoot14SecureSparse1024() {
    return CKKSParams(ckks_aes_params_detail::AESXBoot14SecureSparse1024Config());
}
inline CKKSParams CKKSParams::AESXBoot15() { return CKKSParams(ckks_aes_params_detail::AESXBoot15Config()); }
inline CKKSParams CKKSParams::AESXBoot15Sparse1024() {
    return CKKSParams(ckks_aes_params_detail::AESXBoot15Sparse1024Config());
}

#endif  // CKKS_AES_PARAMS_HPP
