// Per-thread steps of the fused key-switch and rescale kernels (wg_ksfuse.cu), shared with the CPU
// emulation test, which runs them thread by thread between the same barriers.
//
// The fused kernels work on one column tile of the two-phase NTT (wg_ntt.cu): the TILE
// coefficients {(h << NB2) + tile * SUBS + c : h < 2^NB1, c < SUBS}, i.e. SUBS whole columns.
// The inverse transform ends with the column phase and the forward transform starts with it,
// and both phases cover exactly these coefficients, so a CTA can finish the inverse transform
// of some limbs, combine them coefficient by coefficient, and start the forward transform of
// the results without a pass through device memory in between:
//
//   ModUp:   inverse column phase of the digit's alpha source limbs (their row phase ran as one
//            batched launch), N^-1 scaling, the HPS base change of modup_coeff_w
//            (wg_keyswitch.cuh; apply_hps_crt_base_change, ckks_keyswitch.cpp:278-332), then the
//            forward column phase of every destination limb;
//   ModDown: inverse column phase of the K P limbs of one accumulator, N^-1 scaling, the folded
//            ModDown of moddown_all_limbs (ckks_apply_folded_approx_crt_moddown_pair_eval_q,
//            ckks_keyswitch.cpp:521-607), then the forward column phase of every Q limb;
//   Rescale: inverse column phase of the dropped limb, N^-1 scaling, the rounded remainder
//            for every lower limb, then the forward column phase of each remainder (the row
//            phase that follows finishes the rescale in its epilogue, k_ntt_rows_epi).
//
// The butterflies, reductions and FP64 sums are those of the unfused kernels in the same
// order, so the words written equal the ones the separate launches write.  Thread t owns tile
// elements t + k * THREADS (k < 8) in every element-wise step, so those steps need no barrier
// between them; the column rounds are separated by barriers as in k_ntt_phase.
#pragma once
#include <cstddef>
#include <cstdint>

#include "wg_keyswitch.cuh"
#include "wg_ntt.cuh"

namespace wg {
namespace ksf {

// Column tile of the fused kernels: 1024 elements (8 per thread, 128 threads), so the
// source tiles of a digit or of the P limbs fit in shared memory several CTAs per SM.
constexpr int kTile = 1024;

template <int LOGN>
struct Geom {
    using Fwd = ntt::Phase<LOGN, true, true, 3, false, kTile>;
    using Inv = ntt::Phase<LOGN, false, true, 3, false, kTile>;
    static constexpr int N = 1 << LOGN;
    static constexpr int TILE = Fwd::TILE;
    static constexpr int THREADS = Fwd::THREADS;
    static constexpr int E = 8;
    static constexpr int SUBS = Fwd::SUBS;
    static constexpr int PAD = TILE + TILE / 16;  // words of one padded tile
    static constexpr int TILES = N / TILE;
    static constexpr int ROUNDS = Fwd::ROUNDS;
    static_assert(Fwd::TILE == Inv::TILE && Fwd::THREADS == Inv::THREADS, "one tile shape for both directions");
};

template <int LOGN>
WG_HD size_t col_offset(int tile, int e) {
    return ntt::tile_offset<LOGN, true, true, 3, false, kTile>(tile, e);
}

// Load thread t's elements of one limb's column tile.
template <int LOGN>
WG_HD void load_tile(uint64_t* sm, const uint64_t* __restrict__ limb, int tile, int t) {
    using G = Geom<LOGN>;
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        const int e = t + k * G::THREADS;
        sm[ntt::pad16(e)] = limb[col_offset<LOGN>(tile, e)];
    }
}

#if defined(__CUDACC__)
// The same load as an asynchronous copy (cp.async, 8 bytes per element) that lands in shared
// memory without passing through registers, so a CTA can have all its source tiles in flight at
// once; completion is awaited per commit group (cp_async_wait_upto) before a barrier.
template <int LOGN>
__device__ __forceinline__ void load_tile_async(uint64_t* sm, const uint64_t* __restrict__ limb, int tile, int t) {
    using G = Geom<LOGN>;
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        const int e = t + k * G::THREADS;
        const unsigned dst = (unsigned)__cvta_generic_to_shared(sm + ntt::pad16(e));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(limb + col_offset<LOGN>(tile, e))
                     : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int P>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(P) : "memory");
}
// wait until at most `pending` of this thread's commit groups are still in flight
__device__ __forceinline__ void cp_async_wait_upto(int pending) {
    switch (pending) {
        case 0: cp_async_wait<0>(); break;
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        case 3: cp_async_wait<3>(); break;
        case 4: cp_async_wait<4>(); break;
        case 5: cp_async_wait<5>(); break;
        case 6: cp_async_wait<6>(); break;
        default: cp_async_wait<7>(); break;
    }
}
#endif

// Store thread t's elements of the tile to one limb (no reduction: the forward transform's row
// phase continues from these words).
template <int LOGN>
WG_HD void store_tile(const uint64_t* sm, uint64_t* __restrict__ limb, int tile, int t) {
    using G = Geom<LOGN>;
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        const int e = t + k * G::THREADS;
        limb[col_offset<LOGN>(tile, e)] = sm[ntt::pad16(e)];
    }
}

// Round RD of the column phase for thread t (a barrier must follow each round).
template <int LOGN, bool FWD, int RD, bool LAZY>
WG_HD void col_round(uint64_t* sm, int tile, int t, uint64_t q, const ntt::TwPair* __restrict__ tw) {
    using P = ntt::Phase<LOGN, FWD, true, 3, false, kTile>;
    ntt::ntt_round<LOGN, FWD, true, 3, false, RD, LAZY, kTile>(sm, t % P::SUBS, t / P::SUBS, tile, q, tw);
}

// Last step of the inverse transform for thread t's elements: multiply by N^-1 (canonical).
template <int LOGN>
WG_HD void scale_n_inv(uint64_t* sm, int t, const Modulus& m) {
    using G = Geom<LOGN>;
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        uint64_t& v = sm[ntt::pad16(t + k * G::THREADS)];
        v = mul_shoup(v, m.n_inv, m.n_inv_shoup, m.q);
    }
}

// ModUp, source limb i of the digit (coefficients in tile sm_i, canonical): scale by
// qhat_inv_i in place and add the FP64 estimate term to thread t's alpha sums, in the order of
// modup_coeff_w.  (modup_coeff_w first reduces its input below q; the inverse transform's
// N^-1 step already leaves it canonical, so that reduction is the identity here.)
template <int LOGN, class Desc>
WG_HD void modup_scale(uint64_t* sm_i, int t, const Desc& d, int i, uint64_t qi, double* alpha) {
    using G = Geom<LOGN>;
    const uint64_t w = WG_LDG(d.qhat_inv + i), ws = WG_LDG(d.qhat_inv_s + i);
    const double inv = WG_LDG(d.src_inv + i);
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        uint64_t& v = sm_i[ntt::pad16(t + k * G::THREADS)];
        const uint64_t s = mul_shoup(v, w, ws, qi);
        v = s;
        alpha[k] = dadd(alpha[k], dmul(u2d(s), inv));
    }
}

WG_HD uint32_t hps_count(double alpha, int n) {
    uint64_t h = round_half_up(alpha);
    return (uint32_t)(h > (uint64_t)n ? (uint64_t)n : h);
}

// ModUp destination dst of the digit: thread t's coefficients into the work tile.
// src_tiles holds the n scaled source tiles (stride PAD); W >= n bounds the digit width so the
// dst row of constants stays in registers.
template <int LOGN, int W, class Desc>
WG_HD void modup_value(uint64_t* work, const uint64_t* src_tiles, int t, const Desc& d, int dst, uint64_t m,
                       const uint32_t* hps) {
    using G = Geom<LOGN>;
    const int n = d.src_count;
    const uint64_t* row = d.qhat + (size_t)dst * n;
    const uint64_t* row_s = d.qhat_s + (size_t)dst * n;
    const uint64_t* corr = d.corr + (size_t)dst * (n + 1);
    uint64_t w[W], ws[W];
#pragma unroll
    for (int i = 0; i < W; ++i) {
        w[i] = i < n ? WG_LDG(row + i) : 0;
        ws[i] = i < n ? WG_LDG(row_s + i) : 0;
    }
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        const int pe = ntt::pad16(t + k * G::THREADS);
        uint64_t acc = 0;
#pragma unroll
        for (int i = 0; i < W; ++i)
            if (i < n) acc = add_mod(acc, mul_shoup(src_tiles[(size_t)i * G::PAD + pe], w[i], ws[i], m), m);
        work[pe] = sub_mod(acc, WG_LDG(corr + hps[k]), m);
    }
}

// ModDown: FP64 estimate of thread t's coefficients over the K P tiles, in the order of
// moddown_all_limbs_k; FMA: rounded as a fused multiply-add (the pair ModDown's compiled form)
// or as a multiply then an add (the single-polynomial ModDown's).  The tiles hold canonical
// residues (the inverse transform's N^-1 step), so moddown_all_limbs_k's reduction of its input
// below p is the identity here and is left out.  KW >= K keeps the constants in registers.
template <int LOGN, int KW, bool FMA = true>
WG_HD void moddown_hps(const uint64_t* p_tiles, int t, const Modulus* __restrict__ pmods, int K, uint32_t* hps) {
    using G = Geom<LOGN>;
    double inv[KW];
#pragma unroll
    for (int pi = 0; pi < KW; ++pi) inv[pi] = pi < K ? pmods[pi].inv_q : 0.0;
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        const int pe = ntt::pad16(t + k * G::THREADS);
        double alpha = 0.0;
#pragma unroll
        for (int pi = 0; pi < KW; ++pi)
            if (pi < K) {
                const uint64_t s = p_tiles[(size_t)pi * G::PAD + pe];
                alpha = FMA ? dfma(u2d(s), inv[pi], alpha) : dadd(alpha, dmul(u2d(s), inv[pi]));
            }
        hps[k] = hps_count(alpha, K);
    }
}

// ModDown contribution for Q limb qi: thread t's coefficients into the work tile (canonical P
// residues as for moddown_hps; KW >= K).
template <int LOGN, int KW>
WG_HD void moddown_value(uint64_t* work, const uint64_t* p_tiles, int t, int K, uint64_t q,
                         const uint64_t* __restrict__ iv, const uint64_t* __restrict__ ivs, const uint32_t* hps) {
    using G = Geom<LOGN>;
    uint64_t w[KW], ws[KW];
#pragma unroll
    for (int pi = 0; pi < KW; ++pi) {
        w[pi] = pi < K ? WG_LDG(iv + pi) : 0;
        ws[pi] = pi < K ? WG_LDG(ivs + pi) : 0;
    }
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        const int pe = ntt::pad16(t + k * G::THREADS);
        uint64_t acc = 0;
#pragma unroll
        for (int pi = 0; pi < KW; ++pi)
            if (pi < K) acc = add_mod(acc, mul_shoup(p_tiles[(size_t)pi * G::PAD + pe], w[pi], ws[pi], q), q);
        work[pe] = sub_mod(acc, (uint64_t)hps[k], q);
    }
}

// Rescale: thread t's rounded remainders of the dropped limb (coefficients in drop, canonical,
// modulus p) for target limb q into the work tile, as kb_rescale_prep forms them
// (ckks_rescale, src/ckks/operations/arith/ckks_rescale.cpp:68-148).
template <int LOGN>
WG_HD void rescale_value(uint64_t* work, const uint64_t* drop, int t, uint64_t p, uint64_t q, uint64_t one_s,
                         uint64_t half) {
    using G = Geom<LOGN>;
#pragma unroll
    for (int k = 0; k < G::E; ++k) {
        const int pe = ntt::pad16(t + k * G::THREADS);
        uint64_t shift = drop[pe] + (p >> 1);
        if (shift >= p) shift -= p;
        work[pe] = sub_mod(reduce_shoup(shift, q, one_s), half, q);
    }
}

}  // namespace ksf
}  // namespace wg
