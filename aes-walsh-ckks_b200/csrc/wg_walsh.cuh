// Per-residue steps of the fused Walsh S-box products: for one output pair (real bit rb,
// imaginary bit ib) and one limb, the constant-term combination (hm = 0) and the sum over the
// 15 nonzero high masks of (low combination for hm) x (high sign ciphertext hm), unrelinearised.
//
// Reference: build_low_sign_multiples, linear_combination_with_constant,
// linear_combination_pair_with_constant and walsh_sum_for_output_pair,
// src/ckks/operations/circuits/ckks_walsh_sbox.cpp:770-1032.  The reference forms each low
// combination c0 + sum_m c_m s_m from precomputed multiples |c| s_m (repeated additions) with
// modular additions and subtractions of canonical residues, so the combination is the canonical
// residue of the exact integer sum; here the sum is formed exactly (one signed word below 2^55,
// 32-bit halves for wider moduli) and reduced once.  The imaginary half is multiplied by the encoded i and added, then each
// product with a high sign follows the tensor formulas and the products are summed in mask
// order, as the reference's multiply and add sequence does.
#pragma once
#include <cstdint>

#include "wg_arith.cuh"

namespace wg {

constexpr int kWalshMasks = 16;     // nibble masks 0..15
constexpr int kWalshLimbs = 16;     // limbs a combination can span

constexpr int kWalshBias = 8;   // coefficients are stored as c + 8 in [0, 16] (|c| <= 8)

struct WalshCoefs {
    // [real|imag][hm]: the 16 coefficients c[lm] stored as bytes c + kWalshBias, packed
    // little-endian (c[0] unused: the constant term is c0), one 16-byte vector per combination
    uint32_t cw[2][kWalshMasks][4];
    uint64_t c0[2][kWalshMasks][kWalshLimbs];   // rounded c[.][hm][0] * scale mod q_limb
};

// the stored (biased) coefficient byte t, and the signed coefficient
WG_HD uint32_t walsh_coef_biased(const uint32_t* w, int t) { return (w[t >> 2] >> (8 * (t & 3))) & 0xffu; }
WG_HD int walsh_coef(const uint32_t* w, int t) { return (int)walsh_coef_biased(w, t) - kWalshBias; }

WG_HD void walsh_coef_words(const WalshCoefs& cf, int r, int hm, uint32_t* w) {
#if defined(__CUDA_ARCH__)
    const uint4 v = *reinterpret_cast<const uint4*>(cf.cw[r][hm]);
    w[0] = v.x;
    w[1] = v.y;
    w[2] = v.z;
    w[3] = v.w;
#else
    for (int i = 0; i < 4; ++i) w[i] = cf.cw[r][hm][i];
#endif
}

WG_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// canonical residue of sum_{lm=1..15} c[lm] s_lm for |c| <= 8 and canonical s; s_sum is
// sum_lm s_lm (used by the narrow path)
WG_HD uint64_t walsh_small_sum(const uint64_t* s, uint64_t s_sum, const uint32_t* w, const Modulus& m) {
    if (m.q < (1ull << 55)) {
        // sum (c + 8) s < 15 * 16 * 2^55 < 2^63 as an unsigned product of a small factor (two
        // 32-bit multiply-adds per term); minus 8 sum s gives the exact signed sum, |sum| <
        // 120 * 2^55 < 2^62, and adding q 2^sh in [2^62, 2^63) makes it a value in [0, 2^64)
        uint64_t acc = 0;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
        for (int t = 1; t < kWalshMasks; ++t) acc += (uint64_t)walsh_coef_biased(w, t) * s[t];
        return reduce64(acc - (uint64_t)kWalshBias * s_sum + (m.q << (clz64(m.q) - 1)), m);
    }
    // wide moduli: 32-bit halves, R = ah 2^32 + al with |R| < 2^70; q 2^15 >= 2^70 lifts it
    int64_t al = 0, ah = 0;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int t = 1; t < kWalshMasks; ++t) {
        const int64_t k = walsh_coef(w, t);
        al += k * (int64_t)(uint32_t)s[t];
        ah += k * (int64_t)(s[t] >> 32);
    }
    const unsigned __int128 v = (unsigned __int128)(((__int128)ah << 32) + (__int128)al + ((__int128)m.q << 15));
    return reduce128((uint64_t)(v >> 64), (uint64_t)v, m);
}

// (c0r + sum cr s) + pt_i (c0i + sum ci s) for mask hm; the constants only on the b polynomial
WG_HD uint64_t walsh_pair(const uint64_t* s, uint64_t s_sum, const WalshCoefs& cf, int hm, int limb, bool with_const,
                          uint64_t pt_i, const Modulus& m) {
    uint32_t wr[4], wi[4];
    walsh_coef_words(cf, 0, hm, wr);
    walsh_coef_words(cf, 1, hm, wi);
    uint64_t r = walsh_small_sum(s, s_sum, wr, m);
    uint64_t im = walsh_small_sum(s, s_sum, wi, m);
    if (with_const) {
        r = add_mod(cf.c0[0][hm][limb], r, m.q);
        im = add_mod(cf.c0[1][hm][limb], im, m.q);
    }
    return add_mod(r, barrett_mul(im, pt_i, m), m.q);
}

// The low signs of one residue position (masks 1..15 at their index; index 0 is zero).
struct WalshLow {
    uint64_t b[kWalshMasks], a[kWalshMasks];
    uint64_t sb, sa;  // sums of the 15 signs (below 15 q < 2^64 for q < 2^60)
};

WG_HD void walsh_load_low(const uint64_t* low_b, const uint64_t* low_a, WalshLow& w) {
    w.b[0] = w.a[0] = 0;
    w.sb = w.sa = 0;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int t = 1; t < kWalshMasks; ++t) {
        w.b[t] = low_b[t];
        w.a[t] = low_a[t];
        w.sb += low_b[t];
        w.sa += low_a[t];
    }
}

// the constant-term pair (hm = 0): (b, a)
WG_HD void walsh_constant_pair(const WalshLow& w, const WalshCoefs& cf, int limb, uint64_t pt_i, const Modulus& m,
                               uint64_t* acc_b, uint64_t* acc_a) {
    *acc_b = walsh_pair(w.b, w.sb, cf, 0, limb, true, pt_i, m);
    *acc_a = walsh_pair(w.a, w.sa, cf, 0, limb, false, pt_i, m);
}

// product hm of the raw sum, added to (rb, ra, rc) (the first product initialises them)
WG_HD void walsh_product(const WalshLow& w, const WalshCoefs& cf, int hm, int limb, uint64_t pt_i, const Modulus& m,
                         uint64_t yb, uint64_t ya, uint64_t* rb, uint64_t* ra, uint64_t* rc) {
    const uint64_t lb = walsh_pair(w.b, w.sb, cf, hm, limb, true, pt_i, m);
    const uint64_t la = walsh_pair(w.a, w.sa, cf, hm, limb, false, pt_i, m);
    const uint64_t c2 = barrett_mul(la, ya, m);
    const uint64_t tmp = barrett_mul(lb, ya, m);
    const uint64_t b = barrett_mul(lb, yb, m);
    const uint64_t a = add_mod(barrett_mul(la, yb, m), tmp, m.q);
    if (hm == 1) {
        *rb = b;
        *ra = a;
        *rc = c2;
    } else {
        *rb = add_mod(*rb, b, m.q);
        *ra = add_mod(*ra, a, m.q);
        *rc = add_mod(*rc, c2, m.q);
    }
}

}  // namespace wg
