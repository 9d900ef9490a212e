// Index logic and butterflies of the two-phase NTT (see wg_ntt.cu), shared by the device
// kernels and the CPU emulation test.
#pragma once
#include <cstddef>
#include <cstdint>
#include <utility>

#include "wg_arith.cuh"

namespace wg {
namespace ntt {

constexpr int kMaxTile = 2048;

WG_HD int pad16(int e) { return e + (e >> 4); }
WG_HD int floor_log2(unsigned x) {
#if defined(__CUDA_ARCH__)
    return 31 - __clz(x);
#else
    return 31 - __builtin_clz(x);
#endif
}
WG_HD int insert_zero(int v, int g) {
    return ((v >> g) << (g + 1)) | (v & ((1 << g) - 1));
}

// Bits handled by one round: up to three stage bits (in processing order) plus filler bits
// (the lowest free bits) so every thread always owns 8 elements.
struct RoundPlan {
    int ns;
    int sb[3];  // stage bits, processing order
    int jb[3];  // position of each stage bit inside the 3-bit element index j
    int g[3];   // group bits ascending
};

template <int MB, bool FWD>
WG_HDC constexpr RoundPlan make_plan(int rd) {
    RoundPlan p{0, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int k = 0; k < 3; ++k) {
        const int b = FWD ? MB - 1 - 3 * rd - k : 3 * rd + k;
        if (b >= 0 && b < MB) p.sb[p.ns++] = b;
    }
    int mask = 0;
    for (int k = 0; k < p.ns; ++k) mask |= 1 << p.sb[k];
    int filled = p.ns;
    for (int b = 0; filled < 3; ++b)
        if (!((mask >> b) & 1)) {
            mask |= 1 << b;
            ++filled;
        }
    int k = 0;
    for (int b = 0; b < 32 && k < 3; ++b)
        if ((mask >> b) & 1) p.g[k++] = b;
    for (int s = 0; s < p.ns; ++s) p.jb[s] = p.sb[s] == p.g[0] ? 0 : (p.sb[s] == p.g[1] ? 1 : 2);
    return p;
}

template <int LOGN, bool FWD, bool COLS>
struct Phase {
    static constexpr int N = 1 << LOGN;
    static constexpr int NB1 = LOGN / 2;
    static constexpr int NB2 = LOGN - NB1;
    static constexpr int MB = COLS ? NB1 : NB2;
    static constexpr int TILE = N < kMaxTile ? N : kMaxTile;
    static constexpr int THREADS = TILE / 8;
    static constexpr int SUBS = TILE >> MB;  // sub-transforms per tile
    static constexpr int OB = MB - 3;
    static constexpr int ROUNDS = (MB + 2) / 3;
    static constexpr bool LAST = FWD ? !COLS : COLS;
    // Twiddles one CTA reads, staged in shared memory: the column phase reads table entries
    // [0, 2^NB1); the row phase reads, for row-stage k, SUBS * 2^k contiguous entries.
    static constexpr int TW = COLS ? (1 << NB1) : (TILE - SUBS);
    static_assert(MB >= 3, "transform too small");
};

// Table index of staged twiddle t (see Phase::TW).  Row-stage k occupies staged entries
// [SUBS (2^k - 1), SUBS (2^(k+1) - 1)) and maps to table entries starting at
// 2^(NB1 + k) + tile * SUBS * 2^k.
template <int LOGN, bool FWD, bool COLS>
WG_HD size_t twiddle_src(int tile, int t) {
    using P = Phase<LOGN, FWD, COLS>;
    if (COLS) return (size_t)t;
    const int k = floor_log2((unsigned)(t / P::SUBS + 1));
    const int off = P::SUBS * ((1 << k) - 1);
    return ((size_t)1 << (P::NB1 + k)) + (size_t)tile * P::SUBS * ((size_t)1 << k) + (size_t)(t - off);
}

// Bits of element j (0..7) of a round placed at the plan's group positions.
WG_HDC int round_bits(const RoundPlan& p, int j) {
    return ((j & 1) << p.g[0]) | (((j >> 1) & 1) << p.g[1]) | (((j >> 2) & 1) << p.g[2]);
}

// Moduli for which the forward transform may skip the per-butterfly reduction of its upper
// input: each stage then adds at most 2q to a value's bound, so the at most 16 stages of
// N <= 2^16 take inputs below 4q to values below (4 + 2 x 16) q = 36 q < 2^64, and the Shoup
// lazy product accepts any 64-bit input.  The last phase then reduces the full word (reduce64)
// instead of a value below 4q.
constexpr uint64_t kLazyForwardLimit = uint64_t{1} << 58;
static_assert((4 + 2 * 16) < (1 << (64 - 58)), "lazy forward bound: 36 q < 2^64 for q < 2^58");

// One round (up to three radix-2 stages) for thread (sub, o); tw / tws are the staged
// twiddles of this CTA (twiddle_src order).  LAZY (forward only, q < kLazyForwardLimit) keeps
// the upper value unreduced through the round.
//
// The thread's 8 elements are base | round_bits(j), with base's bits disjoint from the group
// positions, so every index splits into a runtime part (one per round, or one per stage for
// twiddles) plus a compile-time offset: pad16 and shifts distribute over disjoint bit sets.
// Loads then use immediate offsets, and butterflies of a stage that share a twiddle load it
// once (same address).
template <int LOGN, bool FWD, bool COLS, int RD, bool LAZY = false>
WG_HD void ntt_round(uint64_t* sm, int sub, int o, uint64_t q, const uint64_t* __restrict__ tw,
                     const uint64_t* __restrict__ tws) {
    using P = Phase<LOGN, FWD, COLS>;
    constexpr RoundPlan plan = make_plan<P::MB, FWD>(RD);
    const uint64_t two_q = q << 1;
    int base = o;
    base = insert_zero(base, plan.g[0]);
    base = insert_zero(base, plan.g[1]);
    base = insert_zero(base, plan.g[2]);
    // element index e = COLS ? h * SUBS + sub : (sub << MB) | h, with h = base | round_bits(j)
    const int e_base = COLS ? base * P::SUBS + sub : (sub << P::MB) | base;
    uint64_t* row = sm + pad16(e_base);
    uint64_t v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = COLS ? round_bits(plan, j) * P::SUBS : round_bits(plan, j);
        v[j] = row[pad16(c)];
    }
#pragma unroll
    for (int s = 0; s < plan.ns; ++s) {
        const int b = plan.sb[s];
        const int jb = plan.jb[s];
        // The table index of a pair is (1 << (n-1-gb)) + (x >> (gb+1)) for its global index x
        // and stage bit gb; relative to the staged block it is:
        const int base_idx = COLS ? (1 << (P::NB1 - 1 - b)) : P::SUBS * ((1 << (P::NB2 - 1 - b)) - 1) + (sub << (P::NB2 - 1 - b));
        const uint64_t* tw_st = tw + base_idx + (base >> (b + 1));
        const uint64_t* tws_st = tws + base_idx + (base >> (b + 1));
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if ((j >> jb) & 1) continue;
            const int j1 = j | (1 << jb);
            const int k = round_bits(plan, j) >> (b + 1);
            const uint64_t w = tw_st[k], ws = tws_st[k];
            if (FWD) {
                uint64_t t = v[j];
                if (!LAZY && t >= two_q) t -= two_q;
                const uint64_t u = mul_shoup_lazy(v[j1], w, ws, q);
                v[j] = t + u;
                v[j1] = t + two_q - u;
            } else {
                const uint64_t t = v[j], u = v[j1];
                uint64_t sum = t + u;
                if (sum >= two_q) sum -= two_q;
                v[j] = sum;
                v[j1] = mul_shoup_lazy(t - u + two_q, w, ws, q);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = COLS ? round_bits(plan, j) * P::SUBS : round_bits(plan, j);
        row[pad16(c)] = v[j];
    }
}

// Global offset (within one limb) of tile element e.
template <int LOGN, bool FWD, bool COLS>
WG_HD size_t tile_offset(int tile, int e) {
    using P = Phase<LOGN, FWD, COLS>;
    if (COLS) {
        const int hh = e / P::SUBS, c = e % P::SUBS;
        return ((size_t)hh << P::NB2) + (size_t)tile * P::SUBS + c;
    }
    return (size_t)tile * P::TILE + e;
}

}  // namespace ntt
}  // namespace wg
