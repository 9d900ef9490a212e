// Homomorphic AES-128-CTR with the XBOOT S-box (the reference's
// src/ckks/operations/circuits/aes/ckks_aes_ctr.hpp), evaluated on the device.
#ifndef CKKS_AES_CTR_HPP
#define CKKS_AES_CTR_HPP

#include <array>
#include <cstddef>
#include <cstdint>
#include <span>
#include <vector>

#include "aligned_vector.hpp"
#include "ckks_ciphertext.hpp"
#include "ckks_context.hpp"

struct CKKSAes128CtrOptions {
    // Kept for source compatibility; the device batches the independent work of a round anyway.
    bool parallelize_independent_work = true;
};

// The 1408 bits of the expanded key, each the constant slot value at the parameter scale,
// encrypted on the device (wg_aes_xboot_encrypt_round_key_bits); round-0 bits
// first_round_key_level levels above the others.
MyVector<CKKSCiphertext> ckks_aes128_encrypt_expanded_round_key_bits(
    const CKKSContext& context, const std::array<uint8_t, 176>& expanded_round_keys, size_t first_round_key_level);

// 128 bit ciphertexts of the CTR plaintext of `ciphertext_blocks` (block b in slot b, repeated
// every active-slot count), evaluated by wg_aes_ctr_xboot.
MyVector<CKKSCiphertext> ckks_aes_ctr(CKKSContext& context,
                                      const MyVector<CKKSCiphertext>& encrypted_expanded_round_key_bits,
                                      std::span<const std::array<uint8_t, 16>> counter_blocks,
                                      std::span<const std::array<uint8_t, 16>> ciphertext_blocks,
                                      const CKKSAes128CtrOptions& options = {});

#endif  // CKKS_AES_CTR_HPP
