// Negacyclic NTT / inverse NTT over batches of RNS limbs.
//
// Same transform as the reference's ntt_forward_dit2 / ntt_inverse_dif2 (src/math/ntt/ntt.cpp:
// 235-386): forward Cooley-Tukey with psi-folded bit-reversed twiddles (natural order in,
// bit-reversed out), inverse Gentleman-Sande with the mirrored table followed by N^-1.
// Outputs are canonical ([0, q)).
//
// Device organisation (N = 2^n, n = n1 + n2, n1 = floor(n/2)):
//   * the transform runs as two phases; the "column" phase owns the n1 high index bits, the
//     "row" phase the n2 low bits.  Forward = columns then rows, inverse = rows then columns.
//   * a CTA stages a 2048-element tile (or the whole limb for N < 2048) in shared memory with
//     one pad word every 16 words, so strided 64-bit accesses stay at two wavefronts per warp;
//   * each thread carries 8 elements through up to three radix-2 stages in registers per
//     round (one shared-memory round trip per three stages);
//   * grid.y indexes limbs and grid.z polynomials, so one launch covers a whole ciphertext
//     batch; each limb picks its modulus through a LimbMap (Q limbs, P limbs or a mix).
// Butterflies are Harvey/Shoup with lazy ranges: forward values stay in [0, 4q) (or, for moduli
// below 2^58, grow by at most 2q per stage without reduction, see kLazyForwardLimit), inverse
// in [0, 2q); the last phase canonicalises (forward) or scales by N^-1 with Shoup (inverse).
#include <utility>

#include "wg_internal.hpp"
#include "wg_ntt.cuh"

namespace wg {
namespace {
using namespace ntt;

template <int LOGN, bool FWD, bool COLS, bool LAZY, int... RD>
__device__ __forceinline__ void ntt_rounds(std::integer_sequence<int, RD...>, uint64_t* sm, int sub,
                                           int o, uint64_t q, const uint64_t* tw, const uint64_t* tws) {
    ((ntt_round<LOGN, FWD, COLS, RD, LAZY>(sm, sub, o, q, tw, tws), __syncthreads()), ...);
}

template <int LOGN, bool FWD, bool COLS>
constexpr size_t smem_bytes() {
    using P = Phase<LOGN, FWD, COLS>;
    return 8 * (size_t)(P::TILE + P::TILE / 16 + 2 * P::TW);
}

// Addressing of one limb: either a strided batch (blockIdx.y = limb, blockIdx.z = polynomial,
// modulus from a LimbMap) or an entry of a job table (blockIdx.y + 65535 * blockIdx.z).  The
// first phase may read from a different buffer than it writes (src -> dst); the second phase
// works in place on dst.
template <int LOGN, bool FWD, bool COLS, bool TABLE>
__global__ void __launch_bounds__(Phase<LOGN, FWD, COLS>::THREADS, 4)
    k_ntt_phase(uint64_t* __restrict__ data, size_t poly_stride, LimbMap map, const NttJob* __restrict__ jobs,
                int njobs, const Modulus* __restrict__ mods, const uint64_t* __restrict__ tw_base) {
    using P = Phase<LOGN, FWD, COLS>;
    constexpr int N = P::N;
    constexpr bool FIRST = FWD ? COLS : !COLS;
    extern __shared__ uint64_t smem[];
    uint64_t* sm = smem;                                  // data tile, padded
    uint64_t* tw_s = smem + P::TILE + P::TILE / 16;       // staged twiddles
    uint64_t* tws_s = tw_s + P::TW;

    const uint64_t* __restrict__ xin;
    uint64_t* __restrict__ x;
    int mi;
    if (TABLE) {
        const int j = blockIdx.y + 65535 * blockIdx.z;
        if (j >= njobs) return;
        const NttJob job = jobs[j];
        x = job.dst;
        xin = FIRST ? job.src : job.dst;
        mi = job.mod;
    } else {
        const int limb = blockIdx.y;
        x = data + (size_t)blockIdx.z * poly_stride + (size_t)limb * N;
        xin = x;
        mi = map(limb);
    }
    const uint64_t q = mods[mi].q;
    const uint64_t* tw = tw_base + (size_t)mi * 4 * N + (FWD ? 0 : 2 * N);
    const uint64_t* tws = tw + N;
    const int tile = blockIdx.x;
    const int t = threadIdx.x;

#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int e = t + k * P::THREADS;
        sm[pad16(e)] = xin[tile_offset<LOGN, FWD, COLS>(tile, e)];
    }
    if (COLS) {
        for (int e = t; e < P::TW; e += P::THREADS) {
            tw_s[e] = __ldg(tw + e);
            tws_s[e] = __ldg(tws + e);
        }
    } else {
        // row-stage k: SUBS * 2^k contiguous table entries (twiddle_src order)
#pragma unroll
        for (int k = 0; k < P::MB; ++k) {
            const int cnt = P::SUBS << k;
            const int dst = P::SUBS * ((1 << k) - 1);
            const size_t src = ((size_t)1 << (P::NB1 + k)) + (size_t)tile * cnt;
            for (int e = t; e < cnt; e += P::THREADS) {
                tw_s[dst + e] = __ldg(tw + src + e);
                tws_s[dst + e] = __ldg(tws + src + e);
            }
        }
    }
    __syncthreads();

    const int sub = COLS ? t % P::SUBS : t >> P::OB;
    const int o = COLS ? t / P::SUBS : t & ((1 << P::OB) - 1);
    // forward transforms under kLazyForwardLimit skip the per-butterfly reduction (uniform per CTA)
    const bool lazy = FWD && q < kLazyForwardLimit;
    if (lazy)
        ntt_rounds<LOGN, FWD, COLS, true>(std::make_integer_sequence<int, P::ROUNDS>{}, sm, sub, o, q, tw_s, tws_s);
    else
        ntt_rounds<LOGN, FWD, COLS, false>(std::make_integer_sequence<int, P::ROUNDS>{}, sm, sub, o, q, tw_s, tws_s);

    uint64_t n_inv = 0, n_inv_s = 0;
    if (P::LAST && !FWD) {
        n_inv = mods[mi].n_inv;
        n_inv_s = mods[mi].n_inv_shoup;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int e = t + k * P::THREADS;
        uint64_t val = sm[pad16(e)];
        if (P::LAST) val = FWD ? (lazy ? reduce64(val, mods[mi]) : red4q(val, q)) : mul_shoup(val, n_inv, n_inv_s, q);
        x[tile_offset<LOGN, FWD, COLS>(tile, e)] = val;
    }
}

template <int LOGN, bool FWD, bool COLS, bool TABLE>
void enable_smem() {
    // opt in to more than 48 KiB of dynamic shared memory once per kernel instance
    static const bool done = [] {
        cudaFuncSetAttribute(k_ntt_phase<LOGN, FWD, COLS, TABLE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes<LOGN, FWD, COLS>());
        return true;
    }();
    (void)done;
}

template <int LOGN, bool FWD, bool COLS>
void launch_phase(const Context& c, uint64_t* data, int limbs, int polys, size_t stride, LimbMap map,
                  const NttJob* jobs, int njobs, cudaStream_t s) {
    using P = Phase<LOGN, FWD, COLS>;
    constexpr size_t sm = smem_bytes<LOGN, FWD, COLS>();
    if (jobs) {
        enable_smem<LOGN, FWD, COLS, true>();
        const dim3 grid(P::N / P::TILE, njobs < 65535 ? njobs : 65535, (njobs + 65534) / 65535);
        // algorithmic bytes: every residue read once and written once per transform, i.e. 8 B
        // per residue for each of the two phases (16 N B per limb-transform)
        Probe probe(kClsNtt, 8.0 * P::N * njobs, s);
        k_ntt_phase<LOGN, FWD, COLS, true><<<grid, P::THREADS, sm, s>>>(nullptr, 0, map, jobs, njobs, c.d_mod, c.d_tw);
    } else {
        enable_smem<LOGN, FWD, COLS, false>();
        const dim3 grid(P::N / P::TILE, limbs, polys);
        Probe probe(kClsNtt, 8.0 * P::N * limbs * polys, s);
        k_ntt_phase<LOGN, FWD, COLS, false><<<grid, P::THREADS, sm, s>>>(data, stride, map, nullptr, 0, c.d_mod,
                                                                         c.d_tw);
    }
}

template <int LOGN>
void run(const Context& c, uint64_t* data, int limbs, int polys, size_t stride, LimbMap map, const NttJob* jobs,
         int njobs, bool fwd, cudaStream_t s) {
    if (fwd) {
        launch_phase<LOGN, true, true>(c, data, limbs, polys, stride, map, jobs, njobs, s);
        launch_phase<LOGN, true, false>(c, data, limbs, polys, stride, map, jobs, njobs, s);
    } else {
        launch_phase<LOGN, false, false>(c, data, limbs, polys, stride, map, jobs, njobs, s);
        launch_phase<LOGN, false, true>(c, data, limbs, polys, stride, map, jobs, njobs, s);
    }
}

void dispatch(const Context& c, uint64_t* data, int limbs, int polys, size_t stride, LimbMap map,
              const NttJob* jobs, int njobs, bool fwd, cudaStream_t s) {
    if (jobs ? njobs <= 0 : (limbs <= 0 || polys <= 0)) return;
    if (!jobs && (polys > 65535 || limbs > 65535)) fail(kInvalid, "ntt: too many limbs or polynomials in one batch");
    switch (c.logN) {
        case 10: run<10>(c, data, limbs, polys, stride, map, jobs, njobs, fwd, s); break;
        case 11: run<11>(c, data, limbs, polys, stride, map, jobs, njobs, fwd, s); break;
        case 12: run<12>(c, data, limbs, polys, stride, map, jobs, njobs, fwd, s); break;
        case 13: run<13>(c, data, limbs, polys, stride, map, jobs, njobs, fwd, s); break;
        case 14: run<14>(c, data, limbs, polys, stride, map, jobs, njobs, fwd, s); break;
        case 15: run<15>(c, data, limbs, polys, stride, map, jobs, njobs, fwd, s); break;
        case 16: run<16>(c, data, limbs, polys, stride, map, jobs, njobs, fwd, s); break;
        default: fail(kInvalid, "ntt: ring degree must be 2^10 .. 2^16");
    }
    check_cuda(cudaGetLastError(), "ntt launch");
}

}  // namespace

void ntt_forward(const Context& c, uint64_t* data, int limbs, int polys, size_t poly_stride, LimbMap map,
                 cudaStream_t s) {
    dispatch(c, data, limbs, polys, poly_stride, map, nullptr, 0, true, s);
}

void ntt_inverse(const Context& c, uint64_t* data, int limbs, int polys, size_t poly_stride, LimbMap map,
                 cudaStream_t s) {
    dispatch(c, data, limbs, polys, poly_stride, map, nullptr, 0, false, s);
}

void ntt_jobs(const Context& c, const NttJob* d_jobs, int njobs, bool forward, cudaStream_t s) {
    dispatch(c, nullptr, 0, 0, 0, LimbMap{0, 0, 0}, d_jobs, njobs, forward, s);
}

}  // namespace wg
