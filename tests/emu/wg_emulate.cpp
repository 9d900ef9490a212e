// CPU emulation of the device kernels (test infrastructure).
//
// Compiles the product's kernel bodies (wg_ntt.cuh, wg_keyswitch.cuh) and host table builder
// (wg_tables.cpp, wg_host.cpp) with the host compiler and runs them CTA by CTA and thread by
// thread, so the index logic, butterflies, HPS base changes and tables can be checked against
// the oracle without a GPU.  Shared-memory rounds are separated exactly where the kernels put
// __syncthreads().  Not part of the product library.
#include <cstring>
#include <utility>
#include <stdexcept>
#include <vector>

#include "wg_keyswitch.cuh"
#include "wg_ksfuse.cuh"
#include "wg_ntt.cuh"
#include "wg_tables.hpp"
#include "wg_walsh.cuh"
#include "wg_ring.hpp"
#include "wg_bundle.hpp"
#include "wg_batching.hpp"
#include <deque>
#include <random>

using namespace wg;

namespace {

struct HostModUp {
    int src_count, dst_count, src_first, pad;
    const uint64_t *qhat_inv, *qhat_inv_s;
    const double* src_inv;
    const uint64_t *qhat, *qhat_s, *corr;
    const int *dst_limb, *dst_mod;
};

struct Emu {
    HostTables H;
    int logN;
    std::vector<std::vector<HostModUp>> modup;
    std::vector<ntt::TwPair> tw;  // interleaved table of every modulus: [mod][fwd N, inv N]
};

template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, bool LAZY, int... RD>
void rounds(std::integer_sequence<int, RD...>, uint64_t* sm, int tile, uint64_t q, const ntt::TwPair* tw) {
    using P = ntt::Phase<LOGN, FWD, COLS, EB, STAGED>;
    auto one = [&](auto rd_const) {
        constexpr int R = decltype(rd_const)::value;
        for (int t = 0; t < P::THREADS; ++t) {
            const int sub = COLS ? t % P::SUBS : t >> P::OB;
            const int o = COLS ? t / P::SUBS : t & ((1 << P::OB) - 1);
            ntt::ntt_round<LOGN, FWD, COLS, EB, STAGED, R, LAZY>(sm, sub, o, tile, q, tw);
        }
    };
    (one(std::integral_constant<int, RD>{}), ...);
}

// NTT geometry the emulated phases use (the device's kNttGeometries order: 0 = 8 residues per
// thread, staged twiddles; 1 = 8, table; 2 = 16, staged; 3 = 16, table).
int g_geometry = 0;

template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED>
void phase(const Emu& E, uint64_t* x, int mi) {
    using P = ntt::Phase<LOGN, FWD, COLS, EB, STAGED>;
    const size_t N = P::N;
    std::vector<ntt::TwPair> table(2 * N);
    ntt::interleave_twiddles(N, E.H.tw.data() + (size_t)mi * 4 * N, table.data());
    const ntt::TwPair* tw = table.data() + (FWD ? 0 : N);
    const Modulus& md = E.H.mods[mi];
    std::vector<uint64_t> sm(P::TILE + P::TILE / 16);
    std::vector<ntt::TwPair> tw_s(P::TW);
    for (int tile = 0; tile < (int)(N / P::TILE); ++tile) {
        for (int e = 0; e < P::TILE; ++e) sm[ntt::pad16(e)] = x[ntt::tile_offset<LOGN, FWD, COLS, EB, STAGED>(tile, e)];
        if (STAGED)
            for (int e = 0; e < P::TW; ++e) tw_s[e] = tw[ntt::twiddle_src<LOGN, FWD, COLS, EB, STAGED>(tile, e)];
        const ntt::TwPair* twr = STAGED ? tw_s.data() : tw;
        const bool lazy = FWD && md.q < ntt::kLazyForwardLimit;
        if (lazy)
            rounds<LOGN, FWD, COLS, EB, STAGED, true>(std::make_integer_sequence<int, P::ROUNDS>{}, sm.data(), tile, md.q,
                                                      twr);
        else
            rounds<LOGN, FWD, COLS, EB, STAGED, false>(std::make_integer_sequence<int, P::ROUNDS>{}, sm.data(), tile,
                                                       md.q, twr);
        for (int e = 0; e < P::TILE; ++e) {
            uint64_t v = sm[ntt::pad16(e)];
            if (P::LAST) v = FWD ? (lazy ? reduce64(v, md) : red4q(v, md.q)) : mul_shoup(v, md.n_inv, md.n_inv_shoup, md.q);
            x[ntt::tile_offset<LOGN, FWD, COLS, EB, STAGED>(tile, e)] = v;
        }
    }
}

template <int LOGN, bool FWD, bool COLS>
void phase_geom(const Emu& E, uint64_t* x, int mi) {
    switch (g_geometry) {
        case 0: phase<LOGN, FWD, COLS, 3, true>(E, x, mi); break;
        case 1: phase<LOGN, FWD, COLS, 3, false>(E, x, mi); break;
        case 2: phase<LOGN, FWD, COLS, 4, true>(E, x, mi); break;
        default: phase<LOGN, FWD, COLS, 4, false>(E, x, mi); break;
    }
}

template <int LOGN>
void ntt_limb(const Emu& E, uint64_t* x, int mi, bool fwd) {
    if (fwd) {
        phase_geom<LOGN, true, true>(E, x, mi);
        phase_geom<LOGN, true, false>(E, x, mi);
    } else {
        phase_geom<LOGN, false, false>(E, x, mi);
        phase_geom<LOGN, false, true>(E, x, mi);
    }
}

void ntt_one(const Emu& E, uint64_t* x, int mi, bool fwd) {
    switch (E.logN) {
        case 10: ntt_limb<10>(E, x, mi, fwd); break;
        case 11: ntt_limb<11>(E, x, mi, fwd); break;
        case 12: ntt_limb<12>(E, x, mi, fwd); break;
        case 13: ntt_limb<13>(E, x, mi, fwd); break;
        case 14: ntt_limb<14>(E, x, mi, fwd); break;
        case 15: ntt_limb<15>(E, x, mi, fwd); break;
        case 16: ntt_limb<16>(E, x, mi, fwd); break;
        default: throw std::invalid_argument("emu: unsupported ring degree");
    }
}

// Key switches and rescales run the fused sequences of wg_ksfuse.cu (Context::ntt_fusion).
int g_fused = 0;

template <int LOGN, bool FWD, bool LAZY, int... RD>
void col_rounds(std::integer_sequence<int, RD...>, uint64_t* sm, int tile, uint64_t q, const ntt::TwPair* tw) {
    using G = ksf::Geom<LOGN>;
    auto one = [&](auto rd_const) {
        constexpr int R = decltype(rd_const)::value;
        for (int t = 0; t < G::THREADS; ++t) ksf::col_round<LOGN, FWD, R, LAZY>(sm, tile, t, q, tw);
    };
    (one(std::integral_constant<int, RD>{}), ...);
}

template <int LOGN>
void inverse_cols(const Emu& E, uint64_t* sm, int tile, int mi) {
    using G = ksf::Geom<LOGN>;
    const Modulus& m = E.H.mods[mi];
    col_rounds<LOGN, false, false>(std::make_integer_sequence<int, G::ROUNDS>{}, sm, tile, m.q,
                                   E.tw.data() + (size_t)mi * 2 * G::N + G::N);
    for (int t = 0; t < G::THREADS; ++t) ksf::scale_n_inv<LOGN>(sm, t, m);
}

template <int LOGN>
void forward_cols(const Emu& E, uint64_t* sm, int tile, int mi) {
    using G = ksf::Geom<LOGN>;
    const uint64_t q = E.H.mods[mi].q;
    const ntt::TwPair* tw = E.tw.data() + (size_t)mi * 2 * G::N;
    if (q < ntt::kLazyForwardLimit)
        col_rounds<LOGN, true, true>(std::make_integer_sequence<int, G::ROUNDS>{}, sm, tile, q, tw);
    else
        col_rounds<LOGN, true, false>(std::make_integer_sequence<int, G::ROUNDS>{}, sm, tile, q, tw);
}

// k_modup_ntt over every column tile of one digit.
template <int LOGN>
void modup_fused(const Emu& E, const HostModUp& d, const uint64_t* src, uint64_t* digit) {
    using G = ksf::Geom<LOGN>;
    const int n = d.src_count;
    std::vector<uint64_t> smem((size_t)(n + 1) * G::PAD);
    uint64_t* work = smem.data() + (size_t)n * G::PAD;
    for (int tile = 0; tile < G::TILES; ++tile) {
        std::vector<double> alpha((size_t)G::THREADS * G::E, 0.0);
        for (int i = 0; i < n; ++i) {
            const int mi = d.src_first + i;
            uint64_t* sm = smem.data() + (size_t)i * G::PAD;
            for (int t = 0; t < G::THREADS; ++t) ksf::load_tile<LOGN>(sm, src + (size_t)mi * G::N, tile, t);
            inverse_cols<LOGN>(E, sm, tile, mi);
            for (int t = 0; t < G::THREADS; ++t)
                ksf::modup_scale<LOGN>(sm, t, d, i, E.H.mods[mi].q, alpha.data() + (size_t)t * G::E);
        }
        std::vector<uint32_t> hps((size_t)G::THREADS * G::E);
        for (size_t k = 0; k < hps.size(); ++k) hps[k] = ksf::hps_count(alpha[k], n);
        for (int dst = 0; dst < d.dst_count; ++dst) {
            const int mi = d.dst_mod[dst];
            for (int t = 0; t < G::THREADS; ++t)
                ksf::modup_value<LOGN, 16>(work, smem.data(), t, d, dst, E.H.mods[mi].q, hps.data() + (size_t)t * G::E);
            forward_cols<LOGN>(E, work, tile, mi);
            for (int t = 0; t < G::THREADS; ++t)
                ksf::store_tile<LOGN>(work, digit + (size_t)d.dst_limb[dst] * G::N, tile, t);
        }
    }
}

// k_moddown_ntt over every column tile of one accumulator polynomial.
template <int LOGN>
void moddown_fused(const Emu& E, const uint64_t* src_p, uint64_t* out, int L, const uint64_t* inv,
                   const uint64_t* inv_s) {
    using G = ksf::Geom<LOGN>;
    const int K = (int)E.H.np, nq = (int)E.H.nq;
    const Modulus* pmods = E.H.mods.data() + nq;
    std::vector<uint64_t> smem((size_t)(K + 1) * G::PAD);
    uint64_t* work = smem.data() + (size_t)K * G::PAD;
    for (int tile = 0; tile < G::TILES; ++tile) {
        for (int pi = 0; pi < K; ++pi) {
            uint64_t* sm = smem.data() + (size_t)pi * G::PAD;
            for (int t = 0; t < G::THREADS; ++t) ksf::load_tile<LOGN>(sm, src_p + (size_t)pi * G::N, tile, t);
            inverse_cols<LOGN>(E, sm, tile, nq + pi);
        }
        std::vector<uint32_t> hps((size_t)G::THREADS * G::E);
        for (int t = 0; t < G::THREADS; ++t)
            ksf::moddown_hps<LOGN, 16>(smem.data(), t, pmods, K, hps.data() + (size_t)t * G::E);
        for (int qi = 0; qi < L; ++qi) {
            for (int t = 0; t < G::THREADS; ++t)
                ksf::moddown_value<LOGN, 16>(work, smem.data(), t, K, E.H.mods[qi].q, inv + (size_t)qi * K,
                                             inv_s + (size_t)qi * K, hps.data() + (size_t)t * G::E);
            forward_cols<LOGN>(E, work, tile, qi);
            for (int t = 0; t < G::THREADS; ++t) ksf::store_tile<LOGN>(work, out + (size_t)qi * G::N, tile, t);
        }
    }
}

// k_ntt_rows_epi for one job: the forward row phase of a copy of the job's limb (the kernel
// reads it and stores nothing back) with the emulated geometry, then the epilogue per word.
template <int LOGN>
void rows_epi(const Emu& E, const ntt::NttEpiJob& j) {
    const size_t N = (size_t)1 << LOGN;
    std::vector<uint64_t> v(j.data, j.data + N);
    phase_geom<LOGN, true, false>(E, v.data(), j.mod);
    for (size_t off = 0; off < N; ++off) ntt::ntt_epilogue(j, off, v[off], E.H.mods[j.mod].q);
}

// k_rescale_ntt over every column tile of one polynomial (dropped limb after the inverse row
// phase); rc: the rescale constants of level lv (one_s, inv_p, inv_p_s, half).
template <int LOGN>
void rescale_fused(const Emu& E, const uint64_t* drop, uint64_t* rem, int lv, const uint64_t* rc) {
    using G = ksf::Geom<LOGN>;
    std::vector<uint64_t> smem((size_t)2 * G::PAD);
    uint64_t* dl = smem.data();
    uint64_t* work = smem.data() + G::PAD;
    const uint64_t p = E.H.mods[lv].q;
    for (int tile = 0; tile < G::TILES; ++tile) {
        for (int t = 0; t < G::THREADS; ++t) ksf::load_tile<LOGN>(dl, drop, tile, t);
        inverse_cols<LOGN>(E, dl, tile, lv);
        for (int qi = 0; qi < lv; ++qi) {
            for (int t = 0; t < G::THREADS; ++t)
                ksf::rescale_value<LOGN>(work, dl, t, p, E.H.mods[qi].q, rc[qi], rc[3 * lv + qi]);
            forward_cols<LOGN>(E, work, tile, qi);
            for (int t = 0; t < G::THREADS; ++t) ksf::store_tile<LOGN>(work, rem + (size_t)qi * G::N, tile, t);
        }
    }
}

// One phase of one limb with the emulated geometry (cols: the high-bit phase).
template <int LOGN>
void phase_one(const Emu& E, uint64_t* x, int mi, bool fwd, bool cols) {
    if (fwd) {
        if (cols) phase_geom<LOGN, true, true>(E, x, mi);
        else phase_geom<LOGN, true, false>(E, x, mi);
    } else {
        if (cols) phase_geom<LOGN, false, true>(E, x, mi);
        else phase_geom<LOGN, false, false>(E, x, mi);
    }
}

#define EMU_LOGN_SWITCH(logN, CALL)                                        \
    do switch (logN) {                                                     \
        case 10: { constexpr int LG = 10; CALL; } break;                   \
        case 11: { constexpr int LG = 11; CALL; } break;                   \
        case 12: { constexpr int LG = 12; CALL; } break;                   \
        case 13: { constexpr int LG = 13; CALL; } break;                   \
        case 14: { constexpr int LG = 14; CALL; } break;                   \
        case 15: { constexpr int LG = 15; CALL; } break;                   \
        case 16: { constexpr int LG = 16; CALL; } break;                   \
        default: throw std::invalid_argument("emu: unsupported ring degree"); \
    } while (0)

}  // namespace

extern "C" {

void* emu_create(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np, size_t dnum) {
    Emu* E = new Emu;
    E->H = build_tables(N, q, nq, p, np, dnum);
    E->logN = __builtin_ctzll(N);
    const uint64_t* T = E->H.words.data();
    E->modup.resize(nq);
    for (size_t l = 0; l < nq; ++l)
        for (const auto& o : E->H.modup[l]) {
            HostModUp d;
            d.src_count = o.src_count;
            d.dst_count = o.dst_count;
            d.src_first = o.src_first;
            d.pad = 0;
            d.qhat_inv = T + o.qhat_inv;
            d.qhat_inv_s = T + o.qhat_inv_s;
            d.src_inv = reinterpret_cast<const double*>(T + o.src_inv);
            d.qhat = T + o.qhat;
            d.qhat_s = T + o.qhat_s;
            d.corr = T + o.corr;
            d.dst_limb = reinterpret_cast<const int*>(T + o.dst_limb);
            d.dst_mod = reinterpret_cast<const int*>(T + o.dst_mod);
            E->modup[l].push_back(d);
        }
    E->tw.resize((nq + np) * 2 * N);
    for (size_t m = 0; m < nq + np; ++m)
        ntt::interleave_twiddles(N, E->H.tw.data() + m * 4 * N, E->tw.data() + m * 2 * N);
    return E;
}

void emu_destroy(void* h) { delete static_cast<Emu*>(h); }

void emu_set_ntt_geometry(int geometry) { g_geometry = geometry; }
void emu_set_keyswitch_fusion(int fused) { g_fused = fused; }

// limbs consecutive limbs using modulus index first.. (basis 0 = Q, 1 = P)
void emu_ntt(void* h, uint64_t* poly, size_t limbs, size_t first, int basis, int inverse) {
    const Emu& E = *static_cast<Emu*>(h);
    for (size_t l = 0; l < limbs; ++l)
        ntt_one(E, poly + l * E.H.N, (int)((basis ? E.H.nq : 0) + first + l), !inverse);
}

// The device keyswitch() sequence, stage by stage, with the same buffers.
void emu_keyswitch(void* h, size_t level, const uint64_t* key_term, const uint64_t* key, size_t key_level,
                   uint64_t* b, uint64_t* a, int b_add, int a_add, uint64_t galois) {
    const Emu& E = *static_cast<Emu*>(h);
    const size_t N = E.H.N, L = level + 1, K = E.H.np, T = L + K, nq = E.H.nq;
    const size_t alpha = E.H.alpha;
    const size_t B = parts_at(level, nq, alpha, E.H.dnum);
    std::vector<uint64_t> ws(N * (L + B * T + 2 * T + 2 * L));
    uint64_t* coeff = ws.data();
    uint64_t* digits = coeff + L * N;
    uint64_t* acc = digits + B * T * N;
    uint64_t* contrib = acc + 2 * T * N;
    const Modulus* mods = E.H.mods.data();
    std::memcpy(coeff, key_term, L * N * 8);
    if (g_fused) {
        // inverse row phase, fused [inverse columns, ModUp, forward columns], forward row phase
        for (size_t l = 0; l < L; ++l) EMU_LOGN_SWITCH(E.logN, phase_one<LG>(E, coeff + l * N, (int)l, false, false));
        for (size_t j = 0; j < B; ++j)
            EMU_LOGN_SWITCH(E.logN, modup_fused<LG>(E, E.modup[level][j], coeff, digits + j * T * N));
    } else {
        for (size_t l = 0; l < L; ++l) ntt_one(E, coeff + l * N, (int)l, false);
        for (size_t j = 0; j < B; ++j)
            for (size_t c = 0; c < N; ++c) modup_coeff(E.modup[level][j], mods, coeff, digits + j * T * N, N, c);
    }
    for (size_t j = 0; j < B; ++j) {
        const size_t s0 = j * alpha, s1 = std::min(s0 + alpha, L);
        for (size_t l = 0; l < T; ++l) {
            if (l >= s0 && l < s1) continue;
            const int mi = (int)(l < L ? l : nq + (l - L));
            if (g_fused)
                EMU_LOGN_SWITCH(E.logN, phase_one<LG>(E, digits + j * T * N + l * N, mi, true, false));
            else
                ntt_one(E, digits + j * T * N + l * N, mi, true);
        }
    }
    for (size_t i = 0; i < T; ++i)
        for (size_t c = 0; c < N; ++c)
            mac_coeff(mods, (int)nq, (int)L, (int)K, (int)B, (int)alpha, key, (int)key_level, key_term, digits, T * N,
                      acc, N, (int)i, c);
    const uint64_t* W = E.H.words.data();
    if (g_fused) {
        for (int poly = 0; poly < 2; ++poly)
            for (size_t pi = 0; pi < K; ++pi)
                EMU_LOGN_SWITCH(E.logN, phase_one<LG>(E, acc + (poly * T + L + pi) * N, (int)(nq + pi), false, false));
        for (int poly = 0; poly < 2; ++poly)
            EMU_LOGN_SWITCH(E.logN, moddown_fused<LG>(E, acc + (poly * T + L) * N, contrib + poly * L * N, (int)L,
                                                      W + E.H.fold_inv[level], W + E.H.fold_inv_s[level]));
        // forward row phase of the contributions with the combine as its epilogue (outputs over
        // the accumulators' Q limbs when an automorphism follows)
        const bool gal = galois != 0;
        for (size_t qi = 0; qi < L; ++qi) {
            const ntt::NttEpiJob ja{contrib + qi * N, acc + qi * N, a + qi * N, (gal ? acc : a) + qi * N,
                                    (uint64_t)a_add, 0, (int)qi, ntt::kEpiCombine};
            const ntt::NttEpiJob jb{contrib + (L + qi) * N, acc + (T + qi) * N, b + qi * N,
                                    (gal ? acc + T * N : b) + qi * N, (uint64_t)b_add, 0, (int)qi, ntt::kEpiCombine};
            EMU_LOGN_SWITCH(E.logN, rows_epi<LG>(E, ja));
            EMU_LOGN_SWITCH(E.logN, rows_epi<LG>(E, jb));
        }
        if (gal)
            for (size_t qi = 0; qi < L; ++qi)
                for (uint32_t i = 0; i < N; ++i) {
                    const uint32_t s = automorphism_src(i, galois, E.logN);
                    b[qi * N + i] = acc[(T + qi) * N + s];
                    a[qi * N + i] = acc[qi * N + s];
                }
        return;
    } else {
        for (int poly = 0; poly < 2; ++poly)
            for (size_t pi = 0; pi < K; ++pi) ntt_one(E, acc + (poly * T + L + pi) * N, (int)(nq + pi), false);
        for (int poly = 0; poly < 2; ++poly)
            for (size_t c = 0; c < N; ++c)
                moddown_all_limbs(mods, (int)nq, (int)L, (int)K, acc + (poly * T + L) * N, N, c,
                                  W + E.H.fold_inv[level], W + E.H.fold_inv_s[level], contrib + poly * L * N);
        for (int poly = 0; poly < 2; ++poly)
            for (size_t qi = 0; qi < L; ++qi) ntt_one(E, contrib + (poly * L + qi) * N, (int)qi, true);
    }
    if (galois == 0) {
        for (size_t qi = 0; qi < L; ++qi)
            for (size_t c = 0; c < N; ++c)
                combine_coeff(mods[qi].q, (int)L, (int)K, acc, contrib, b, a, b, a, b_add, a_add, N, (int)qi, c);
    } else {
        uint64_t* tb = acc + T * N;
        uint64_t* ta = acc;
        for (size_t qi = 0; qi < L; ++qi)
            for (size_t c = 0; c < N; ++c)
                combine_coeff(mods[qi].q, (int)L, (int)K, acc, contrib, b, a, tb, ta, b_add, a_add, N, (int)qi, c);
        for (size_t qi = 0; qi < L; ++qi)
            for (uint32_t i = 0; i < N; ++i) {
                const uint32_t s = automorphism_src(i, galois, E.logN);
                b[qi * N + i] = tb[qi * N + s];
                a[qi * N + i] = ta[qi * N + s];
            }
    }
}

// The device rescale sequence (wg_batch_kernels.cuh RescaleJobs) on one polynomial at level lv:
// x holds lv + 1 limbs; afterwards its first lv limbs are the rescaled polynomial.
void emu_rescale(void* h, size_t lv, uint64_t* x) {
    const Emu& E = *static_cast<Emu*>(h);
    const size_t N = E.H.N;
    const uint64_t* rc = E.H.words.data() + E.H.rescale[lv];
    std::vector<uint64_t> rem(lv * N);
    uint64_t* dl = x + lv * N;
    if (g_fused) {
        EMU_LOGN_SWITCH(E.logN, phase_one<LG>(E, dl, (int)lv, false, false));
        EMU_LOGN_SWITCH(E.logN, rescale_fused<LG>(E, dl, rem.data(), (int)lv, rc));
        for (size_t q = 0; q < lv; ++q) {
            const ntt::NttEpiJob j{rem.data() + q * N, nullptr, x + q * N, x + q * N, rc[lv + q], rc[2 * lv + q],
                                   (int)q, ntt::kEpiRescale};
            EMU_LOGN_SWITCH(E.logN, rows_epi<LG>(E, j));
        }
        return;
    }
    ntt_one(E, dl, (int)lv, false);
    const Modulus& mp = E.H.mods[lv];
    for (size_t q = 0; q < lv; ++q) {
        const Modulus& mq = E.H.mods[q];
        uint64_t* r = rem.data() + q * N;
        for (size_t k = 0; k < N; ++k) {  // kb_rescale_prep
            uint64_t shift = dl[k] + (mp.q >> 1);
            if (shift >= mp.q) shift -= mp.q;
            r[k] = sub_mod(reduce_shoup(shift, mq.q, rc[q]), rc[3 * lv + q], mq.q);
        }
        ntt_one(E, r, (int)q, true);
        for (size_t k = 0; k < N; ++k) {  // kb_rescale_finish
            uint64_t v = x[q * N + k];
            if (v >= mq.q) v -= mq.q;
            x[q * N + k] = mul_shoup(sub_mod(v, r[k], mq.q), rc[lv + q], rc[2 * lv + q], mq.q);
        }
    }
}

static Modulus emu_modulus(uint64_t q) {
    Modulus m{};
    const unsigned __int128 mu = ~(unsigned __int128)0 / q;
    m.q = q;
    m.mu_lo = (uint64_t)mu;
    m.mu_hi = (uint64_t)(mu >> 64);
    return m;
}

// mont_mul (the Montgomery product of the key inner products) on n pairs: out[i] = x[i] y[i] 2^-64
// mod q for odd q, qninv = -q^-1 mod 2^64 by Newton iteration.
void emu_mont_mul(uint64_t q, const uint64_t* x, const uint64_t* y, size_t n, uint64_t* out) {
    uint64_t inv = q;  // q q = 1 (mod 8): three correct bits, doubled by each step
    for (int k = 0; k < 5; ++k) inv *= 2 - q * inv;
    for (size_t i = 0; i < n; ++i) out[i] = mont_mul(x[i], y[i], q, 0 - inv);
}

// reduce128 on n values (hi[i], lo[i]) modulo q
void emu_reduce128(uint64_t q, const uint64_t* hi, const uint64_t* lo, size_t n, uint64_t* out) {
    const Modulus m = emu_modulus(q);
    for (size_t i = 0; i < n; ++i) out[i] = reduce128(hi[i], lo[i], m);
}

// The fused Walsh products at n residue positions of one limb (limb index 0, modulus q).
// low_b, low_a, high_b, high_a: [n][16] (mask 0 ignored); coefs: [2][16][16] int8; c0: [2][16];
// out: [n][5] = acc b, acc a, raw b, raw a, raw c2.
void emu_walsh_products(uint64_t q, size_t n, const uint64_t* low_b, const uint64_t* low_a, const uint64_t* high_b,
                        const uint64_t* high_a, const uint64_t* pt_i, const int8_t* coefs, const uint64_t* c0,
                        uint64_t* out) {
    const Modulus m = emu_modulus(q);
    WalshCoefs cf{};
    // [2][16][16] signed coefficients, stored biased as in the device table
    uint8_t biased[2 * 16 * 16];
    for (int i = 0; i < 2 * 16 * 16; ++i) biased[i] = (uint8_t)(coefs[i] + kWalshBias);
    std::memcpy(cf.cw, biased, sizeof(cf.cw));
    for (int r = 0; r < 2; ++r)
        for (int hm = 0; hm < kWalshMasks; ++hm) cf.c0[r][hm][0] = c0[r * kWalshMasks + hm];
    for (size_t i = 0; i < n; ++i) {
        WalshLow w;
        walsh_load_low(low_b + i * 16, low_a + i * 16, w);
        uint64_t* o = out + i * 5;
        walsh_constant_pair(w, cf, 0, pt_i[i], m, o, o + 1);
        for (int hm = 1; hm < kWalshMasks; ++hm)
            walsh_product(w, cf, hm, 0, pt_i[i], m, high_b[i * 16 + hm], high_a[i * 16 + hm], o + 2, o + 3, o + 4);
    }
}

// The staging ring's placement (wg_ring.hpp) over `steps` seeded uploads of mixed sizes (1 in 100
// a large one), with no upload ever completing on its own (the host arbitrarily far ahead of the
// device): returns how many regions overlapped an upload the placement did not wait for.
size_t emu_ring_violations(uint64_t seed, size_t steps) {
    struct F {
        size_t begin, end;
    };
    std::mt19937_64 g(seed);
    std::deque<F> flights;
    size_t ring = 0, head = 0, bad = 0;
    for (size_t i = 0; i < steps; ++i) {
        const size_t bytes = (g() % 100 == 0) ? (size_t{100} << 20) : (size_t)(1024 + g() % (128 * 1024));
        const size_t need = (bytes + 255) & ~size_t{255};
        if (need > ring) {  // growth: everything in flight completes first
            flights.clear();
            ring = std::max<size_t>(2 * need, size_t{64} << 20);
            head = 0;
        }
        size_t wait = 0;
        const size_t begin = wg::ring_place(head, ring, need, flights, &wait);
        for (size_t k = 0; k < wait; ++k) flights.pop_front();
        for (const F& f : flights)
            if (f.begin < begin + need && begin < f.end) ++bad;
        flights.push_back({begin, begin + need});
        head = begin + need;
    }
    return bad;
}

// The bundle file format (wg_bundle.hpp): a seeded random bundle survives encode + decode
// unchanged (returns 0), and the reader rejects every damaged variant tried: each single flipped
// byte at `trials` seeded positions, every truncation length tried, a wrong magic and a wrong
// version (returns how many damaged variants it accepted).
int emu_bundle_roundtrip(uint64_t seed) {
    std::mt19937_64 g(seed);
    Bundle b;
    b.N = 1u << 10;
    b.dnum = 3;
    for (int i = 0; i < 5; ++i) b.q.push_back(g());
    for (int i = 0; i < 2; ++i) b.p.push_back(g());
    for (int k = 0; k < 3; ++k) {
        BundleKey key;
        key.kind = (int64_t)(g() % 5);
        key.rotation = (int64_t)(g() % 1000) - 500;
        key.parts = 1 + g() % 3;
        key.key_level = g() % 5;
        key.data.resize(1 + g() % 5000);
        for (auto& w : key.data) w = g();
        b.keys.push_back(key);
    }
    for (int k = 0; k < 2; ++k) {
        BundleStage st;
        st.level = g() % 5;
        st.baby = 1 + g() % 16;
        st.slots = 512;
        st.rescale = g() & 1;
        st.indices.resize(1 + g() % 40);
        for (auto& w : st.indices) w = g() % 512;
        st.diagonals.resize(st.indices.size() * 7);
        for (auto& w : st.diagonals) w = g();
        b.stages.push_back(st);
    }
    const auto bytes = bundle_encode(b);
    const Bundle r = bundle_decode(bytes.data(), bytes.size());
    bool same = r.N == b.N && r.dnum == b.dnum && r.q == b.q && r.p == b.p && r.keys.size() == b.keys.size() &&
                r.stages.size() == b.stages.size();
    for (size_t k = 0; same && k < b.keys.size(); ++k)
        same = r.keys[k].kind == b.keys[k].kind && r.keys[k].rotation == b.keys[k].rotation &&
               r.keys[k].parts == b.keys[k].parts && r.keys[k].key_level == b.keys[k].key_level &&
               r.keys[k].data == b.keys[k].data;
    for (size_t k = 0; same && k < b.stages.size(); ++k)
        same = r.stages[k].level == b.stages[k].level && r.stages[k].baby == b.stages[k].baby &&
               r.stages[k].slots == b.stages[k].slots && r.stages[k].rescale == b.stages[k].rescale &&
               r.stages[k].indices == b.stages[k].indices && r.stages[k].diagonals == b.stages[k].diagonals;
    return same ? 0 : 1;
}

size_t emu_bundle_damage_accepted(uint64_t seed, size_t trials) {
    std::mt19937_64 g(seed);
    Bundle b;
    b.N = 64;
    b.dnum = 2;
    b.q = {g(), g()};
    b.p = {g()};
    BundleKey key;
    key.data.resize(100);
    for (auto& w : key.data) w = g();
    b.keys.push_back(key);
    BundleStage st;
    st.indices = {1, 2};
    st.diagonals.resize(10);
    b.stages.push_back(st);
    const auto good = bundle_encode(b);
    size_t accepted = 0;
    auto accepts = [&](const std::vector<uint8_t>& v) {
        try {
            bundle_decode(v.data(), v.size());
            return true;
        } catch (const std::invalid_argument&) {
            return false;
        }
    };
    for (size_t t = 0; t < trials; ++t) {
        auto v = good;
        v[g() % v.size()] ^= (uint8_t)(1u << (g() % 8));
        accepted += accepts(v);
    }
    for (size_t len = 0; len < good.size(); len += 1 + good.size() / 97)
        accepted += accepts(std::vector<uint8_t>(good.begin(), good.begin() + len));
    auto magic = good;
    magic[0] = 'X';
    accepted += accepts(magic);
    auto version = good;
    version[4] = 2;
    accepted += accepts(version);
    return accepted;
}

// The service's request packing (wg_batching.hpp) on `trials` seeded queues of 0..12 requests of
// 1..max_blocks blocks: returns how many queues broke a property of first fit — positions
// ascending, the oldest request taken, the taken blocks within the slots, every skipped request
// too large for the slots left at its turn — or of batch_full (some request skipped, or the
// slots used up exactly).
size_t emu_first_fit_violations(uint64_t seed, size_t trials) {
    std::mt19937_64 g(seed);
    size_t bad = 0;
    for (size_t t = 0; t < trials; ++t) {
        const size_t max_blocks = 1 + g() % 64;
        std::deque<size_t> q(g() % 13);
        for (auto& n : q) n = 1 + g() % max_blocks;
        const auto id = [](size_t n) { return n; };
        const std::vector<size_t> take = wg::first_fit(q, max_blocks, id);
        bool ok = q.empty() ? take.empty() : (!take.empty() && take[0] == 0);
        size_t used = 0, ti = 0;
        bool skipped = false;
        for (size_t k = 0; k < q.size(); ++k) {
            if (ti < take.size() && take[ti] == k) {
                used += q[k];
                ++ti;
            } else {
                skipped = true;
                ok = ok && used + q[k] > max_blocks;
            }
        }
        ok = ok && ti == take.size() && used <= max_blocks;
        for (size_t k = 1; k < take.size(); ++k) ok = ok && take[k] > take[k - 1];
        ok = ok && wg::batch_full(q, max_blocks, id) == (skipped || used == max_blocks);
        bad += ok ? 0 : 1;
    }
    return bad;
}

}  // extern "C"
