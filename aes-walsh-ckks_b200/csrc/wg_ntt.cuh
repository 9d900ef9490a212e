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

// One entry of the interleaved twiddle table: the twiddle and its Shoup constant side by side,
// so a butterfly fetches both with one 16-byte load.  Table layout per modulus:
// [forward pairs (N)][inverse pairs (N)].
struct alignas(16) TwPair {
    uint64_t w, ws;
};

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

// Bits handled by one round: up to EB stage bits (in processing order) plus filler bits (the
// lowest free bits) so every thread always owns 2^EB elements.
struct RoundPlan {
    int ns;
    int sb[4];  // stage bits, processing order
    int jb[4];  // position of each stage bit inside the EB-bit element index j
    int g[4];   // group bits ascending
};

template <int MB, bool FWD, int EB>
WG_HDC constexpr RoundPlan make_plan(int rd) {
    RoundPlan p{0, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
    for (int k = 0; k < EB; ++k) {
        const int b = FWD ? MB - 1 - EB * rd - k : EB * rd + k;
        if (b >= 0 && b < MB) p.sb[p.ns++] = b;
    }
    int mask = 0;
    for (int k = 0; k < p.ns; ++k) mask |= 1 << p.sb[k];
    int filled = p.ns;
    for (int b = 0; filled < EB; ++b)
        if (!((mask >> b) & 1)) {
            mask |= 1 << b;
            ++filled;
        }
    int k = 0;
    for (int b = 0; b < 32 && k < EB; ++b)
        if ((mask >> b) & 1) p.g[k++] = b;
    for (int s = 0; s < p.ns; ++s)
        for (int x = 0; x < EB; ++x)
            if (p.sb[s] == p.g[x]) p.jb[s] = x;
    return p;
}

// Geometry of one phase of an N = 2^LOGN transform.
//   EB:     a thread carries 2^EB residues through each round (3: radix-8 rounds of up to three
//           stages; 4: radix-16 rounds of up to four), so a round is one shared-memory round trip;
//   STAGED: the CTA first copies the twiddle pairs it will read into shared memory; otherwise
//           the rounds read them from the (L2-resident) global table directly, which leaves
//           shared memory to the data tile and admits more CTAs per SM.
//   TL:     largest tile (elements per CTA); a column-phase tile holds TL >> NB1 whole columns.
template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, int TL = kMaxTile>
struct Phase {
    static constexpr int N = 1 << LOGN;
    static constexpr int NB1 = LOGN / 2;
    static constexpr int NB2 = LOGN - NB1;
    static constexpr int MB = COLS ? NB1 : NB2;
    static constexpr int E = 1 << EB;
    static constexpr int TILE = N < TL ? N : TL;
    static constexpr int THREADS = TILE / E;
    static constexpr int SUBS = TILE >> MB;  // sub-transforms per tile
    static constexpr int OB = MB - EB;
    static constexpr int ROUNDS = (MB + EB - 1) / EB;
    static constexpr bool LAST = FWD ? !COLS : COLS;
    // Twiddle pairs one CTA reads (staged in shared memory when STAGED): the column phase reads
    // table entries [0, 2^NB1); the row phase reads, for row-stage k, SUBS * 2^k contiguous
    // entries.
    static constexpr int TW = COLS ? (1 << NB1) : (TILE - SUBS);
    static_assert(MB >= EB, "transform too small for this round radix");
    static_assert(EB == 3 || EB == 4, "rounds of 8 or 16 residues per thread");
};

// Table index of staged twiddle t (see Phase::TW).  Row-stage k occupies staged entries
// [SUBS (2^k - 1), SUBS (2^(k+1) - 1)) and maps to table entries starting at
// 2^(NB1 + k) + tile * SUBS * 2^k.
template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, int TL = kMaxTile>
WG_HD size_t twiddle_src(int tile, int t) {
    using P = Phase<LOGN, FWD, COLS, EB, STAGED, TL>;
    if (COLS) return (size_t)t;
    const int k = floor_log2((unsigned)(t / P::SUBS + 1));
    const int off = P::SUBS * ((1 << k) - 1);
    return ((size_t)1 << (P::NB1 + k)) + (size_t)tile * P::SUBS * ((size_t)1 << k) + (size_t)(t - off);
}

// Bits of element j (0 .. 2^EB - 1) of a round placed at the plan's group positions.
template <int EB>
WG_HDC constexpr int round_bits(const RoundPlan& p, int j) {
    int r = 0;
    for (int k = 0; k < EB; ++k) r |= ((j >> k) & 1) << p.g[k];
    return r;
}

// Moduli for which the forward transform may skip the per-butterfly reduction of its upper
// input: each stage then adds at most 2q to a value's bound, so the at most 16 stages of
// N <= 2^16 take inputs below 4q to values below (4 + 2 x 16) q = 36 q < 2^64, and the Shoup
// lazy product accepts any 64-bit input.  The last phase then reduces the full word (reduce64)
// instead of a value below 4q.
constexpr uint64_t kLazyForwardLimit = uint64_t{1} << 58;
static_assert((4 + 2 * 16) < (1 << (64 - 58)), "lazy forward bound: 36 q < 2^64 for q < 2^58");

// One round (up to EB radix-2 stages) for thread (sub, o) of tile `tile`.  `tw` is the CTA's
// staged block (STAGED, twiddle_src order) or the modulus's table of this direction.  LAZY
// (forward only, q < kLazyForwardLimit) keeps the upper value unreduced through the round.
//
// The thread's elements are base | round_bits(j), with base's bits disjoint from the group
// positions, so every index splits into a runtime part (one per round, or one per stage for
// twiddles) plus a compile-time offset: pad16 and shifts distribute over disjoint bit sets.
// Loads then use immediate offsets, and butterflies of a stage that share a twiddle load it
// once (same address).
template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, int RD, bool LAZY = false, int TL = kMaxTile>
WG_HD void ntt_round(uint64_t* sm, int sub, int o, int tile, uint64_t q, const TwPair* __restrict__ tw) {
    using P = Phase<LOGN, FWD, COLS, EB, STAGED, TL>;
    constexpr int E = P::E;
    constexpr RoundPlan plan = make_plan<P::MB, FWD, EB>(RD);
    const uint64_t two_q = q << 1;
    int base = o;
#pragma unroll
    for (int k = 0; k < EB; ++k) base = insert_zero(base, plan.g[k]);
    // element index e = COLS ? h * SUBS + sub : (sub << MB) | h, with h = base | round_bits(j)
    const int e_base = COLS ? base * P::SUBS + sub : (sub << P::MB) | base;
    uint64_t* row = sm + pad16(e_base);
    uint64_t v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int c = COLS ? round_bits<EB>(plan, j) * P::SUBS : round_bits<EB>(plan, j);
        v[j] = row[pad16(c)];
    }
#pragma unroll
    for (int s = 0; s < plan.ns; ++s) {
        const int b = plan.sb[s];
        const int jb = plan.jb[s];
        // The table index of a pair is (1 << (n-1-gb)) + (x >> (gb+1)) for its global index x
        // and stage bit gb; relative to the staged block (or to the table) it is:
        const int kr = P::NB2 - 1 - b;  // row-stage of bit b
        const size_t base_idx =
            COLS ? (size_t)(1 << (P::NB1 - 1 - b))
                 : (STAGED ? (size_t)(P::SUBS * ((1 << kr) - 1) + (sub << kr))
                           : ((size_t)1 << (P::NB1 + kr)) + (size_t)tile * P::SUBS * ((size_t)1 << kr) +
                                 (size_t)(sub << kr));
        const TwPair* tw_st = tw + base_idx + (base >> (b + 1));
#pragma unroll
        for (int j = 0; j < E; ++j) {
            if ((j >> jb) & 1) continue;
            const int j1 = j | (1 << jb);
            const int k = round_bits<EB>(plan, j) >> (b + 1);
#if defined(__CUDA_ARCH__)
            uint64_t w, ws;
            if (STAGED) {
                const TwPair tp = tw_st[k];
                w = tp.w;
                ws = tp.ws;
            } else {
                const ulonglong2 tp = __ldg(reinterpret_cast<const ulonglong2*>(tw_st + k));
                w = tp.x;
                ws = tp.y;
            }
#else
            const uint64_t w = tw_st[k].w, ws = tw_st[k].ws;
#endif
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
    for (int j = 0; j < E; ++j) {
        const int c = COLS ? round_bits<EB>(plan, j) * P::SUBS : round_bits<EB>(plan, j);
        row[pad16(c)] = v[j];
    }
}

// The forward row phase of one limb (data: after the forward column phase, read only) with an
// element-wise epilogue on the finished canonical words v instead of storing them:
//   kEpiRescale: out = (in - v) * p^-1 mod q  (in reduced below q first; c0, c1 = p^-1 and its
//                Shoup constant: the rescale finish step, as kb_rescale_finish);
//   kEpiCombine: out = c0 ? in + (acc - v) : acc - v  (the key switch's final combine, as
//                combine_coeff).
// out may alias in or acc (each word is read and written by the same thread).
enum NttEpilogue : int { kEpiRescale = 1, kEpiCombine = 2 };
struct NttEpiJob {
    const uint64_t* data;
    const uint64_t* acc;
    const uint64_t* in;
    uint64_t* out;
    uint64_t c0, c1;
    int mod;
    int kind;
};

// The epilogue's word for the finished canonical word v and the operands acc, in (each used
// only where the kind needs it).
WG_HD uint64_t epilogue_value(const NttEpiJob& j, uint64_t acc, uint64_t in, uint64_t v, uint64_t q) {
    if (j.kind == kEpiRescale) {
        if (in >= q) in -= q;
        return mul_shoup(sub_mod(in, v, q), j.c0, j.c1, q);
    }
    const uint64_t d = sub_mod(acc, v, q);
    return j.c0 ? add_mod(in, d, q) : d;
}

// The epilogue at word off of the job's limbs, operands read from their arrays.
WG_HD void ntt_epilogue(const NttEpiJob& j, size_t off, uint64_t v, uint64_t q) {
    const uint64_t acc = j.kind == kEpiCombine ? j.acc[off] : 0;
    const uint64_t in = (j.kind == kEpiRescale || j.c0) ? j.in[off] : 0;
    j.out[off] = epilogue_value(j, acc, in, v, q);
}

// Global offset (within one limb) of tile element e.
template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, int TL = kMaxTile>
WG_HD size_t tile_offset(int tile, int e) {
    using P = Phase<LOGN, FWD, COLS, EB, STAGED, TL>;
    if (COLS) {
        const int hh = e / P::SUBS, c = e % P::SUBS;
        return ((size_t)hh << P::NB2) + (size_t)tile * P::SUBS + c;
    }
    return (size_t)tile * P::TILE + e;
}

// Interleaved twiddle table (TwPair layout above) from the split one [fwd, fwd_shoup, inv,
// inv_shoup][N] of one modulus.
inline void interleave_twiddles(size_t N, const uint64_t* split, TwPair* out) {
    for (size_t d = 0; d < 2; ++d)
        for (size_t i = 0; i < N; ++i) out[d * N + i] = TwPair{split[2 * d * N + i], split[(2 * d + 1) * N + i]};
}

}  // namespace ntt
}  // namespace wg
