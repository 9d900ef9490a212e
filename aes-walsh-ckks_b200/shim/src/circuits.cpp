// The AES circuit entries of the reference API, evaluated by the device library:
// ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks / ckks_aes_ctr_walsh_sbox_
// complex_blocks (src/ckks/operations/circuits/aes/ckks_aes_ctr_walsh_sbox.cpp:981-1051) and
// ckks_aes128_encrypt_expanded_round_key_bits / ckks_aes_ctr (ckks_aes_ctr.cpp:687-779).  Each
// call returns when the device has finished (the reference's calls are synchronous).
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "aes/ckks_aes_ctr.hpp"
#include "aes/ckks_aes_ctr_walsh_sbox.hpp"
#include "context_engine.hpp"

namespace {

constexpr size_t kKeyBits = 1408;
constexpr size_t kStateBits = 128;

void ok(int rc, const char* what) {
    if (rc == WG_OK) return;
    const std::string msg = std::string(what) + ": " + wg_last_error();
    if (rc == WG_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

void finish(const char* what) {
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

struct Ptrs {
    std::vector<uint64_t*> b, a;
};

Ptrs device_ptrs(MyVector<CKKSCiphertext>& cts) {
    Ptrs p;
    for (auto& c : cts) {
        p.b.push_back(c.devicePoly(0));
        p.a.push_back(c.devicePoly(1));
    }
    return p;
}

struct KeyView {
    std::vector<const uint64_t*> b, a;
    std::vector<double> scales;
    std::vector<size_t> levels;
};

KeyView key_view(const MyVector<CKKSCiphertext>& keys) {
    if (keys.size() != kKeyBits) throw std::invalid_argument("ckks_aes_ctr: expected 1408 encrypted round-key bits");
    KeyView v;
    for (const auto& k : keys) {
        v.b.push_back(k.devicePoly(0));
        v.a.push_back(k.devicePoly(1));
        v.scales.push_back((double)k.getScale());
        v.levels.push_back(k.getLevel());
    }
    return v;
}

MyVector<CKKSCiphertext> make_outputs(const CKKSContext::Engine& e, size_t count, const std::vector<size_t>& levels) {
    MyVector<CKKSCiphertext> out;
    out.reserve(count);
    const size_t N = e.params.getN();
    for (size_t i = 0; i < count; ++i) out.emplace_back(N, e.params.getScale(), levels[i], 2, levels[i] + 1);
    return out;
}

void label(MyVector<CKKSCiphertext>& cts, const std::vector<size_t>& levels, const std::vector<double>& scales) {
    for (size_t i = 0; i < cts.size(); ++i) {
        cts[i].markDeviceWritten();
        cts[i].setLevel(levels[i]);
        cts[i].setScale(scales[i]);
    }
}

std::vector<const wg_lt_stage*> cview(const std::vector<wg_lt_stage*>& v) { return {v.begin(), v.end()}; }

}  // namespace

MyVector<CKKSCiphertext> ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks(
    const CKKSContext& context, const std::array<uint8_t, 176>& expanded_round_keys, size_t active_complex_block_count) {
    CKKSContext::Engine& e = context.engine();
    if (!e.params.usesAesWalsh() || !e.has_plans)
        throw std::invalid_argument("ckks_aes_walsh: the context is not an AES-Walsh bootstrapping context");
    const wg_bootstrap_params bp = e.bootstrap_params();
    const std::vector<size_t> levels(kKeyBits, bp.s2c_depth + 1);
    auto out = make_outputs(e, kKeyBits, levels);
    Ptrs p = device_ptrs(out);
    std::vector<double> sc(kKeyBits);
    std::vector<size_t> lv(kKeyBits);
    ok(wg_aes_walsh_encrypt_round_key_bits(e.ctx, &bp, expanded_round_keys.data(), active_complex_block_count,
                                           e.secret.data(), e.next_seed(), e.params.getSigma(), p.b.data(), p.a.data(),
                                           sc.data(), lv.data(), nullptr),
       "ckks_aes_walsh");
    finish("ckks_aes_walsh");
    label(out, lv, sc);
    return out;
}

MyVector<CKKSCiphertext> ckks_aes_ctr_walsh_sbox_complex_blocks(
    CKKSContext& context, const MyVector<CKKSCiphertext>& keys, std::span<const std::array<uint8_t, 16>> counter_blocks,
    std::span<const std::array<uint8_t, 16>> ciphertext_blocks, const CKKSAesCtrWalshSboxOptions&) {
    CKKSContext::Engine& e = context.engine();
    if (!e.params.usesAesWalsh() || !e.has_plans || !e.has_evalmod)
        throw std::invalid_argument("ckks_aes_walsh: the context is not an AES-Walsh bootstrapping context");
    if (counter_blocks.size() != ciphertext_blocks.size() || counter_blocks.empty() || counter_blocks.size() % 2)
        throw std::invalid_argument("ckks_aes_walsh: counter and ciphertext spans must hold 2 * active blocks each");
    const size_t active = counter_blocks.size() / 2;
    const KeyView k = key_view(keys);
    for (size_t l : k.levels)
        if (l != k.levels[0]) throw std::invalid_argument("ckks_aes_walsh: round-key bits must share one level");
    const wg_bootstrap_params bp = e.bootstrap_params();
    auto out = make_outputs(e, kStateBits, std::vector<size_t>(kStateBits, bp.depth));
    Ptrs p = device_ptrs(out);
    std::vector<size_t> lv(kStateBits);
    std::vector<double> sc(kStateBits);
    const auto s2c = cview(e.s2c), s2c2 = cview(e.s2c_x2), c2s = cview(e.c2s);
    ok(wg_aes_ctr_walsh(e.ctx, &bp, s2c.data(), s2c.size(), s2c2.data(), s2c2.size(), c2s.data(), c2s.size(),
                        e.evalmod.chebyshev_coeffs.data(), e.evalmod.chebyshev_coeffs.size(),
                        e.params.getAesWalshBlockCount(), e.params.getAesWalshPackedSegmentCount(), k.b.data(),
                        k.a.data(), k.scales.data(), k.levels[0], counter_blocks.data()->data(),
                        ciphertext_blocks.data()->data(), active, p.b.data(), p.a.data(), lv.data(), sc.data(), nullptr),
       "ckks_aes_ctr_walsh_sbox_complex_blocks");
    finish("ckks_aes_ctr_walsh_sbox_complex_blocks");
    label(out, lv, sc);
    return out;
}

MyVector<CKKSCiphertext> ckks_aes128_encrypt_expanded_round_key_bits(const CKKSContext& context,
                                                                     const std::array<uint8_t, 176>& expanded_round_keys,
                                                                     size_t first_round_key_level) {
    CKKSContext::Engine& e = context.engine();
    if (!e.has_plans) throw std::invalid_argument("ckks_aes_ctr: the context is not a bootstrapping context");
    const wg_bootstrap_params bp = e.bootstrap_params();
    if (bp.s2c_depth + first_round_key_level > bp.depth)
        throw std::invalid_argument("ckks_aes_ctr: first round-key level exceeds the modulus chain");
    std::vector<size_t> levels(kKeyBits, bp.s2c_depth);
    for (size_t i = 0; i < kStateBits; ++i) levels[i] = bp.s2c_depth + first_round_key_level;
    auto out = make_outputs(e, kKeyBits, levels);
    Ptrs p = device_ptrs(out);
    std::vector<double> sc(kKeyBits);
    std::vector<size_t> lv(kKeyBits);
    ok(wg_aes_xboot_encrypt_round_key_bits(e.ctx, &bp, expanded_round_keys.data(), first_round_key_level,
                                           e.secret.data(), e.next_seed(), e.params.getSigma(), p.b.data(), p.a.data(),
                                           sc.data(), lv.data(), nullptr),
       "ckks_aes128_encrypt_expanded_round_key_bits");
    finish("ckks_aes128_encrypt_expanded_round_key_bits");
    label(out, lv, sc);
    return out;
}

MyVector<CKKSCiphertext> ckks_aes_ctr(CKKSContext& context, const MyVector<CKKSCiphertext>& keys,
                                      std::span<const std::array<uint8_t, 16>> counter_blocks,
                                      std::span<const std::array<uint8_t, 16>> ciphertext_blocks,
                                      const CKKSAes128CtrOptions&) {
    CKKSContext::Engine& e = context.engine();
    if (!e.has_plans || !e.has_evalmod) throw std::invalid_argument("ckks_aes_ctr: the context is not a bootstrapping context");
    if (counter_blocks.size() != ciphertext_blocks.size() || counter_blocks.empty())
        throw std::invalid_argument("ckks_aes_ctr: counter and ciphertext block counts must match");
    const KeyView k = key_view(keys);
    const wg_bootstrap_params bp = e.bootstrap_params();
    auto out = make_outputs(e, kStateBits, std::vector<size_t>(kStateBits, bp.depth));
    Ptrs p = device_ptrs(out);
    std::vector<size_t> lv(kStateBits);
    std::vector<double> sc(kStateBits);
    const auto s2c = cview(e.s2c), c2s = cview(e.c2s);
    ok(wg_aes_ctr_xboot(e.ctx, &bp, s2c.data(), s2c.size(), c2s.data(), c2s.size(), e.evalmod.chebyshev_coeffs.data(),
                        e.evalmod.chebyshev_coeffs.size(), k.b.data(), k.a.data(), k.scales.data(), k.levels.data(),
                        counter_blocks.data()->data(), ciphertext_blocks.data()->data(), counter_blocks.size(), p.b.data(),
                        p.a.data(), lv.data(), sc.data(), nullptr),
       "ckks_aes_ctr");
    finish("ckks_aes_ctr");
    label(out, lv, sc);
    return out;
}
