// Homomorphic AES-128-CTR with the Walsh S-box on lazy bits, complex-packed (the reference's
// src/ckks/operations/circuits/aes/ckks_aes_ctr_walsh_sbox.hpp), evaluated on the device.
#ifndef CKKS_AES_CTR_WALSH_SBOX_HPP
#define CKKS_AES_CTR_WALSH_SBOX_HPP

#include <array>
#include <cstddef>
#include <cstdint>
#include <span>

#include "aligned_vector.hpp"
#include "ckks_ciphertext.hpp"
#include "ckks_context.hpp"

struct CKKSAesCtrWalshSboxOptions {
    // Kept for source compatibility; the device runs all S-box pairs of a round as one batch.
    bool parallelize_sbox_pairs = true;
};

// The 1408 expanded-key bits, each (v, v) in the first active_complex_block_count slots,
// encrypted on the device (wg_aes_walsh_encrypt_round_key_bits).
MyVector<CKKSCiphertext> ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks(
    const CKKSContext& context, const std::array<uint8_t, 176>& expanded_round_keys,
    size_t active_complex_block_count);

// 128 bit ciphertexts: slot s carries block s in its real part and block
// active_complex_block_count + s in its imaginary part (wg_aes_ctr_walsh); the block spans hold
// 2 * active_complex_block_count blocks.
MyVector<CKKSCiphertext> ckks_aes_ctr_walsh_sbox_complex_blocks(
    CKKSContext& context, const MyVector<CKKSCiphertext>& encrypted_expanded_round_key_bits,
    std::span<const std::array<uint8_t, 16>> counter_blocks, std::span<const std::array<uint8_t, 16>> ciphertext_blocks,
    const CKKSAesCtrWalshSboxOptions& options = {});

#endif  // CKKS_AES_CTR_WALSH_SBOX_HPP
