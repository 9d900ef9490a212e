// Per-coefficient bodies of the hybrid key switch, shared by the device kernels
// (wg_keyswitch.cu) and the CPU emulation test.
//
// Reference: src/ckks/operations/keyswitch/ckks_keyswitch.cpp
//   HPS ModUp             apply_hps_crt_base_change                         :278-332
//   key inner product     ckks_pointwise_multiply_accumulate_montgomery_key  :445-463
//   folded ModDown        ckks_apply_folded_approx_crt_moddown_pair_eval_q   :521-607
//   combine               ckks_hybrid_key_switch_inplace                     :1624-1640
// The HPS alpha estimates are FP64 sums in the reference's order.  The reference build
// rounds the ModUp sum as multiply-then-add and contracts the ModDown sum into an FMA; the
// kernels do the same with explicitly rounded intrinsics.
#pragma once
#include <cstddef>
#include <cstdint>

#include "wg_arith.cuh"

namespace wg {

constexpr int kMaxDigitWidth = 16;  // largest alpha (Q limbs per digit) the kernels support
constexpr int kMaxPLimbs = 16;

// Galois automorphism on the bit-reversed evaluation layout
// (build_ntt_automorphism_map, src/ckks/context/rotation_key_generation.cpp:80-90):
// output slot i reads input slot src_index(i).
WG_HD uint32_t bitrev32(uint32_t x, int bits) {
#if defined(__CUDA_ARCH__)
    return __brev(x) >> (32 - bits);
#else
    uint32_t r = 0;
    for (int k = 0; k < bits; ++k) r = (r << 1) | ((x >> k) & 1u);
    return r;
#endif
}
WG_HD uint32_t automorphism_src(uint32_t i, uint64_t galois, int logN) {
    const uint64_t mask2n = (uint64_t{2} << logN) - 1;  // 2N - 1 (2N is a power of two)
    const uint64_t dst_nat = bitrev32(i, logN);
    const uint64_t src_exp = ((2 * dst_nat + 1) * galois) & mask2n;
    return bitrev32((uint32_t)((src_exp - 1) >> 1), logN);
}

// HPS ModUp of one coefficient for one digit, digit width at most W (the scaled residues stay
// in registers: every index below is a compile-time constant after unrolling).
//   src:   coefficient-domain key term, limb-major (Q limb k at src + k*N)
//   digit: QP digit buffer of this part (limb t at digit + t*N)
template <int W, class Desc>
WG_HD void modup_coeff_w(const Desc& d, const Modulus* __restrict__ mods, const uint64_t* __restrict__ src,
                         uint64_t* __restrict__ digit, size_t N, size_t coeff) {
    uint64_t scaled[W];
    double alpha = 0.0;
    const int n = d.src_count;
#pragma unroll
    for (int i = 0; i < W; ++i) {
        scaled[i] = 0;
        if (i < n) {
            const uint64_t qi = mods[d.src_first + i].q;
            const uint64_t x = red4q(src[(size_t)(d.src_first + i) * N + coeff], qi);
            const uint64_t s = mul_shoup(x, WG_LDG(d.qhat_inv + i), WG_LDG(d.qhat_inv_s + i), qi);
            scaled[i] = s;
            alpha = dadd(alpha, dmul(u2d(s), WG_LDG(d.src_inv + i)));
        }
    }
    uint64_t hps = round_half_up(alpha);
    if (hps > (uint64_t)n) hps = (uint64_t)n;
    for (int t = 0; t < d.dst_count; ++t) {
        const uint64_t m = mods[WG_LDG(d.dst_mod + t)].q;
        const uint64_t* row = d.qhat + (size_t)t * n;
        const uint64_t* row_s = d.qhat_s + (size_t)t * n;
        uint64_t acc = 0;
#pragma unroll
        for (int i = 0; i < W; ++i)
            if (i < n) acc = add_mod(acc, mul_shoup(scaled[i], WG_LDG(row + i), WG_LDG(row_s + i), m), m);
        const uint64_t corr = WG_LDG(d.corr + (size_t)t * (n + 1) + hps);
        digit[(size_t)WG_LDG(d.dst_limb + t) * N + coeff] = sub_mod(acc, corr, m);
    }
}

template <class Desc>
WG_HD void modup_coeff(const Desc& d, const Modulus* __restrict__ mods, const uint64_t* __restrict__ src,
                       uint64_t* __restrict__ digit, size_t N, size_t coeff) {
    if (d.src_count <= 4)
        modup_coeff_w<4>(d, mods, src, digit, N, coeff);
    else if (d.src_count <= 8)
        modup_coeff_w<8>(d, mods, src, digit, N, coeff);
    else
        modup_coeff_w<kMaxDigitWidth>(d, mods, src, digit, N, coeff);
}

// moddown_all_limbs for at most KW P limbs (the P residues stay in registers).
template <bool FUSED, int KW>
WG_HD void moddown_all_limbs_k(const Modulus* __restrict__ mods, int nq, int L, int K,
                               const uint64_t* __restrict__ src_p, size_t N, size_t coeff,
                               const uint64_t* __restrict__ inv, const uint64_t* __restrict__ inv_s,
                               uint64_t* __restrict__ out) {
    uint64_t s[KW];
    double alpha = 0.0;
#pragma unroll
    for (int pi = 0; pi < KW; ++pi) {
        s[pi] = 0;
        if (pi < K) {
            const Modulus& mp = mods[nq + pi];
            s[pi] = red4q(src_p[(size_t)pi * N + coeff], mp.q);
            alpha = FUSED ? dfma(u2d(s[pi]), mp.inv_q, alpha) : dadd(alpha, dmul(u2d(s[pi]), mp.inv_q));
        }
    }
    uint64_t hps = round_half_up(alpha);
    if (hps > (uint64_t)K) hps = (uint64_t)K;
    for (int qi = 0; qi < L; ++qi) {
        const Modulus& mq = mods[qi];
        const uint64_t q = mq.q;
        const uint64_t* iv = inv + (size_t)qi * K;
        const uint64_t* ivs = inv_s + (size_t)qi * K;
        uint64_t acc = 0;
        // s[pi] mod q need not be formed: the Shoup product is canonical for any 64-bit input
#pragma unroll
        for (int pi = 0; pi < KW; ++pi)
            if (pi < K) acc = add_mod(acc, mul_shoup(s[pi], WG_LDG(iv + pi), WG_LDG(ivs + pi), q), q);
        out[(size_t)qi * N + coeff] = sub_mod(acc, hps, q);
    }
}

// Folded ModDown of one coefficient for Q limbs [0, L):
//   contribution_qi = (sum_j [x_j mod q_i] inv_ij) - round(sum_j x_j / p_j)   (mod q_i)
// The P residues are read and the FP64 alpha estimate formed once, then each limb gets its Shoup
// dot product (the reference reduces x_j mod q_i first with barrett_reduce_u64; the Shoup product
// is the canonical residue of x_j inv_ij for any 64-bit x_j, so that reduction cannot change a
// word).  out[qi * N + coeff] = contribution.
// FUSED selects how the alpha sum is rounded: the reference's pair ModDown
// (ckks_keyswitch.cpp:521-607) is compiled into an FMA, its single-polynomial ModDown
// (ckks_keyswitch.cpp:609-673, used by the QP linear transform) into a multiply and an add.
template <bool FUSED = true>
WG_HD void moddown_all_limbs(const Modulus* __restrict__ mods, int nq, int L, int K,
                             const uint64_t* __restrict__ src_p, size_t N, size_t coeff,
                             const uint64_t* __restrict__ inv, const uint64_t* __restrict__ inv_s,
                             uint64_t* __restrict__ out) {
    if (K <= 4)
        moddown_all_limbs_k<FUSED, 4>(mods, nq, L, K, src_p, N, coeff, inv, inv_s, out);
    else if (K <= 8)
        moddown_all_limbs_k<FUSED, 8>(mods, nq, L, K, src_p, N, coeff, inv, inv_s, out);
    else
        moddown_all_limbs_k<FUSED, kMaxPLimbs>(mods, nq, L, K, src_p, N, coeff, inv, inv_s, out);
}

// Key inner product for QP limb i at one coefficient, added digit by digit onto (acc_a,
// acc_b) with canonical modular additions (ckks_pointwise_multiply_accumulate_montgomery_key_lazy,
// ckks_keyswitch.cpp:445-463).  Source limbs of a digit use the evaluation-form key term itself.
WG_HD void mac_accumulate(const Modulus& m, int L, int K, int parts, int alpha, const uint64_t* __restrict__ key,
                          int key_level, const uint64_t* __restrict__ key_term, const uint64_t* __restrict__ digits,
                          size_t part_stride, size_t N, int i, size_t coeff, uint64_t& acc_a, uint64_t& acc_b) {
    const bool is_p = i >= L;
    const uint64_t q = m.q, qninv = m.qninv;
    const size_t key_limbs = (size_t)key_level + 1 + K;
    const size_t klimb = is_p ? (size_t)key_level + 1 + (i - L) : (size_t)i;
#pragma unroll 4
    for (int j = 0; j < parts; ++j) {
        const int s0 = j * alpha, s1 = s0 + alpha < L ? s0 + alpha : L;
        const uint64_t d = (!is_p && i >= s0 && i < s1) ? key_term[(size_t)i * N + coeff]
                                                         : digits[j * part_stride + (size_t)i * N + coeff];
        const uint64_t ka = key[(((size_t)j * 2 + 0) * key_limbs + klimb) * N + coeff];
        const uint64_t kb = key[(((size_t)j * 2 + 1) * key_limbs + klimb) * N + coeff];
        acc_a = add_mod(acc_a, mont_mul(d, ka, q, qninv), q);
        acc_b = add_mod(acc_b, mont_mul(d, kb, q, qninv), q);
    }
}

// Key inner product for QP limb i at one coefficient:
//   acc_{a,b}[i] = sum_parts REDC(digit_part[i] * key_part_{a,b}[i]).
// Source limbs of a digit use the evaluation-form key term itself (as the reference does).
WG_HD void mac_coeff(const Modulus* __restrict__ mods, int nq, int L, int K, int parts, int alpha,
                     const uint64_t* __restrict__ key, int key_level, const uint64_t* __restrict__ key_term,
                     const uint64_t* __restrict__ digits, size_t part_stride, uint64_t* __restrict__ acc,
                     size_t N, int i, size_t coeff) {
    const int T = L + K;
    const Modulus& m = mods[i >= L ? nq + (i - L) : i];
    uint64_t acc_a = 0, acc_b = 0;
    mac_accumulate(m, L, K, parts, alpha, key, key_level, key_term, digits, part_stride, N, i, coeff, acc_a, acc_b);
    acc[(size_t)i * N + coeff] = acc_a;
    acc[(size_t)(T + i) * N + coeff] = acc_b;
}

// Final combine for Q limb qi: v = acc - contrib; out = add ? in + v : v (a and b).
WG_HD void combine_coeff(uint64_t q, int L, int K, const uint64_t* acc, const uint64_t* contrib,
                         const uint64_t* b_in, const uint64_t* a_in, uint64_t* b_out, uint64_t* a_out,
                         int b_add, int a_add, size_t N, int qi, size_t coeff) {
    const int T = L + K;
    const size_t k = (size_t)qi * N + coeff;
    const uint64_t va = sub_mod(acc[k], contrib[k], q);
    const uint64_t vb = sub_mod(acc[(size_t)T * N + k], contrib[(size_t)L * N + k], q);
    b_out[k] = b_add ? add_mod(b_in[k], vb, q) : vb;
    a_out[k] = a_add ? add_mod(a_in[k], va, q) : va;
}

}  // namespace wg
