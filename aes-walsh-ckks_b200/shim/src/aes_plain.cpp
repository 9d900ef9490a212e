// Plain AES-128 (FIPS-197): S-box from the multiplicative inverse in GF(2^8) (modulus
// x^8 + x^4 + x^3 + x + 1) followed by the affine map, key expansion, the ten rounds, and CTR
// mode as XOR with the encrypted counter block.
#include <array>
#include <cstdint>

#include "aes/aes.hpp"

namespace {

uint8_t gmul(uint8_t a, uint8_t b) {
    uint8_t r = 0;
    while (b) {
        if (b & 1) r ^= a;
        a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
        b >>= 1;
    }
    return r;
}

const std::array<uint8_t, 256>& sbox() {
    static const std::array<uint8_t, 256> t = [] {
        std::array<uint8_t, 256> s{};
        for (int x = 0; x < 256; ++x) {
            uint8_t inv = 0;
            for (int y = 1; y < 256 && x; ++y)
                if (gmul((uint8_t)x, (uint8_t)y) == 1) {
                    inv = (uint8_t)y;
                    break;
                }
            uint8_t v = inv;
            uint8_t out = 0x63;
            for (int k = 0; k < 5; ++k) {
                out ^= v;
                v = (uint8_t)((v << 1) | (v >> 7));
            }
            s[x] = out;
        }
        return s;
    }();
    return t;
}

}  // namespace

std::array<uint8_t, 176> aes128_expand_key(const std::array<uint8_t, 16>& key) {
    const auto& S = sbox();
    std::array<uint8_t, 176> w{};
    for (int i = 0; i < 16; ++i) w[i] = key[i];
    uint8_t rcon = 1;
    for (int i = 4; i < 44; ++i) {
        uint8_t t[4] = {w[4 * (i - 1)], w[4 * (i - 1) + 1], w[4 * (i - 1) + 2], w[4 * (i - 1) + 3]};
        if (i % 4 == 0) {
            const uint8_t t0 = t[0];
            t[0] = (uint8_t)(S[t[1]] ^ rcon);
            t[1] = S[t[2]];
            t[2] = S[t[3]];
            t[3] = S[t0];
            rcon = gmul(rcon, 2);
        }
        for (int k = 0; k < 4; ++k) w[4 * i + k] = (uint8_t)(w[4 * (i - 4) + k] ^ t[k]);
    }
    return w;
}

std::array<uint8_t, 16> aes128_encrypt_block(const std::array<uint8_t, 16>& key,
                                             const std::array<uint8_t, 16>& in) {
    const auto& S = sbox();
    const auto w = aes128_expand_key(key);
    std::array<uint8_t, 16> s{};
    for (int i = 0; i < 16; ++i) s[i] = (uint8_t)(in[i] ^ w[i]);
    for (int round = 1; round <= 10; ++round) {
        std::array<uint8_t, 16> t{};
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) t[4 * c + r] = S[s[4 * ((c + r) % 4) + r]];  // SubBytes + ShiftRows
        if (round != 10)
            for (int c = 0; c < 4; ++c) {  // MixColumns
                const uint8_t a0 = t[4 * c], a1 = t[4 * c + 1], a2 = t[4 * c + 2], a3 = t[4 * c + 3];
                t[4 * c] = (uint8_t)(gmul(a0, 2) ^ gmul(a1, 3) ^ a2 ^ a3);
                t[4 * c + 1] = (uint8_t)(a0 ^ gmul(a1, 2) ^ gmul(a2, 3) ^ a3);
                t[4 * c + 2] = (uint8_t)(a0 ^ a1 ^ gmul(a2, 2) ^ gmul(a3, 3));
                t[4 * c + 3] = (uint8_t)(gmul(a0, 3) ^ a1 ^ a2 ^ gmul(a3, 2));
            }
        for (int i = 0; i < 16; ++i) s[i] = (uint8_t)(t[i] ^ w[16 * round + i]);
    }
    return s;
}

std::array<uint8_t, 16> aes128_ctr_crypt_block(const std::array<uint8_t, 16>& key,
                                               const std::array<uint8_t, 16>& counter_block,
                                               const std::array<uint8_t, 16>& input_block) {
    const auto ks = aes128_encrypt_block(key, counter_block);
    std::array<uint8_t, 16> out{};
    for (int i = 0; i < 16; ++i) out[i] = (uint8_t)(ks[i] ^ input_block[i]);
    return out;
}
