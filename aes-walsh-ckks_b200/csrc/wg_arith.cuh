// Exact 64-bit modular arithmetic on the device.
//
// Every helper restates one scalar routine of the reference (src/math/modarith/modarith.hpp)
// with the same reduction steps, because several of them can legitimately leave a result in
// [q, 2q) (the 128-bit Barrett product keeps a single correction) and those representations
// flow into later operations.  Bit-exact parity therefore needs the same formulas, not just
// the same residues modulo q.  The 128-bit products are formed from __umul64hi and plain
// 64-bit multiplies.
#pragma once
#include <cmath>
#include <cstdint>

// Helpers are __host__ __device__ so the CPU emulation test (tests/emu) can run the very same
// kernel bodies against the oracle; the product library only uses them on the device.
#if defined(__CUDACC__)
#define WG_HD __host__ __device__ __forceinline__
#define WG_HDC __host__ __device__
#else
#define WG_HD inline
#define WG_HDC
#endif
#if defined(__CUDA_ARCH__)
#define WG_LDG(p) __ldg(p)
#else
#define WG_LDG(p) (*(p))
#endif

namespace wg {

// Per-modulus constants, one entry per Q modulus followed by the P moduli.
struct Modulus {
    uint64_t q;
    uint64_t mu_lo;      // floor((2^128-1)/q), low word   (barrett_const_computation)
    uint64_t mu_hi;      //                     high word
    uint64_t qninv;      // -q^{-1} mod 2^64               (ckks_montgomery_neg_inverse64)
    uint64_t n_inv;      // N^{-1} mod q
    uint64_t n_inv_shoup;
    double inv_q;        // 1.0 / (double)q
    uint64_t pad;
};

WG_HD uint64_t umulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// IEEE double helpers with explicit rounding, so no multiply-add is contracted unless asked.
WG_HD double u2d(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __ull2double_rn(x);
#else
    return (double)x;
#endif
}
WG_HD double dmul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
WG_HD double dadd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
WG_HD double dfma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
// (uint64_t)(x + 0.5) for x >= 0, truncating like the C conversion.
WG_HD uint64_t round_half_up(double x) {
#if defined(__CUDA_ARCH__)
    return __double2ull_rz(__dadd_rn(x, 0.5));
#else
    return (uint64_t)(x + 0.5);
#endif
}

// mul_mod_shoup (modarith.hpp:93-99): result canonical for any a < 2^64.
WG_HD uint64_t mul_shoup(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
    const uint64_t u = umulhi(a, ws);
    uint64_t r = a * w - u * q;
    return r >= q ? r - q : r;
}

// Shoup product without the final correction: result in [0, 2q) (the NTT butterfly form).
WG_HD uint64_t mul_shoup_lazy(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
    return a * w - umulhi(a, ws) * q;
}

// barrett_reduce (modarith.hpp:16-32), including its truncated carry handling.
WG_HD uint64_t barrett_mul(uint64_t a, uint64_t b, const Modulus& m) {
    const uint64_t z_lo = a * b;
    const uint64_t z_hi = umulhi(a, b);
    const uint64_t t_lo = z_hi * m.mu_lo;
    const uint64_t t_hi = umulhi(z_hi, m.mu_lo);
    const uint64_t c = umulhi(z_lo, m.mu_lo);
    const uint64_t s_lo = t_lo + c;
    const uint64_t carry = t_hi + (s_lo < t_lo ? 1ull : 0ull);
    const uint64_t q_hat = z_hi * m.mu_hi + umulhi(z_lo, m.mu_hi) + carry;
    uint64_t r = z_lo - q_hat * m.q;
    return r >= m.q ? r - m.q : r;
}

// Canonical residue of a 128-bit value z = z_hi 2^64 + z_lo.  The quotient estimate is the one
// barrett_mul forms; for any z < 2^128 it is at most two below floor(z / q) (mu = floor((2^128-1)/q)
// costs less than one, the middle carry left out at most one) and never above it, so z - q_hat q
// lies in [0, 3q) and two corrections make it canonical.  Requires q < 2^62.
WG_HD uint64_t reduce128(uint64_t z_hi, uint64_t z_lo, const Modulus& m) {
    const uint64_t t_lo = z_hi * m.mu_lo;
    const uint64_t t_hi = umulhi(z_hi, m.mu_lo);
    const uint64_t c = umulhi(z_lo, m.mu_lo);
    const uint64_t s_lo = t_lo + c;
    const uint64_t carry = t_hi + (s_lo < t_lo ? 1ull : 0ull);
    const uint64_t q_hat = z_hi * m.mu_hi + umulhi(z_lo, m.mu_hi) + carry;
    uint64_t r = z_lo - q_hat * m.q;
    if (r >= m.q) r -= m.q;
    return r >= m.q ? r - m.q : r;
}

// Canonical residue of any a < 2^64: the estimate umulhi(a, mu_hi), mu_hi = floor(mu / 2^64)
// >= 2^64 / q - 1, is at most one below floor(a / q) and never above it.
WG_HD uint64_t reduce64(uint64_t a, const Modulus& m) {
    uint64_t r = a - umulhi(a, m.mu_hi) * m.q;
    if (r >= m.q) r -= m.q;
    return r >= m.q ? r - m.q : r;
}

// barrett_reduce_u64 (modarith.hpp:53-58).
WG_HD uint64_t barrett_u64(uint64_t a, uint64_t q, uint64_t mu_hi) {
    const uint64_t q_hat = umulhi(a, mu_hi);
    uint64_t r = a - q_hat * q;
    return r >= q ? r - q : r;
}

// ckks_montgomery_mul_normal_by_montgomery (modarith.hpp:116-130).
// qninv = -q^-1 mod 2^64, so m q = -t_lo (mod 2^64): the low words of t + m q sum to 0, with a
// carry exactly when t_lo != 0, and the low product m q need not be formed.
WG_HD uint64_t mont_mul(uint64_t normal, uint64_t mont, uint64_t q, uint64_t qninv) {
    const uint64_t t_lo = normal * mont;
    const uint64_t t_hi = umulhi(normal, mont);
    const uint64_t m = t_lo * qninv;
    const uint64_t mq_hi = umulhi(m, q);
    uint64_t u = t_hi + mq_hi + (t_lo != 0 ? 1ull : 0ull);
    return u >= q ? u - q : u;
}

// reduce_mod_4q, add_mod_q, sub_mod_q (modarith.hpp:43-81).
WG_HD uint64_t red4q(uint64_t x, uint64_t q) {
    const uint64_t two_q = q << 1;
    if (x >= two_q) x -= two_q;
    return x >= q ? x - q : x;
}
WG_HD uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) {
    const uint64_t r = a + b;
    return r >= q ? r - q : r;
}
WG_HD uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
    const uint64_t r = a - b;
    return a < b ? r + q : r;
}

// reduce_u64_mod_q_shoup (modarith.hpp:34-41).
WG_HD uint64_t reduce_shoup(uint64_t x, uint64_t q, uint64_t one_shoup) {
    const uint64_t u = umulhi(x, one_shoup);
    uint64_t r = x - u * q;
    if (r >= q) r -= q;
    return r >= q ? r - q : r;
}

}  // namespace wg
