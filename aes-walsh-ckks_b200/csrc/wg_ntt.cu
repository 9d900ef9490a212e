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
//   * each thread carries 8 or 16 elements (the geometry's EB) through up to three or four
//     radix-2 stages in registers per round (one shared-memory round trip per round);
//   * twiddles come as (w, Shoup w) pairs, one 16-byte load each, either staged in shared
//     memory per CTA or read from the L2-resident table directly (the geometry's STAGED);
//   * grid.y indexes limbs and grid.z polynomials, so one launch covers a whole ciphertext
//     batch; each limb picks its modulus through a LimbMap (Q limbs, P limbs or a mix).
// Butterflies are Harvey/Shoup with lazy ranges: forward values stay in [0, 4q) (or, for moduli
// below 2^58, grow by at most 2q per stage without reduction, see kLazyForwardLimit), inverse
// in [0, 2q); the last phase canonicalises (forward) or scales by N^-1 with Shoup (inverse).
// Every geometry performs the same butterflies on the same values, so all of them give the
// same words; which one runs is chosen per (direction, phase) by timing them on the device
// when a context is created (ntt_autotune).
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "wg_internal.hpp"
#include "wg_ntt.cuh"

namespace wg {
namespace {
using namespace ntt;

template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, bool LAZY, int... RD>
__device__ __forceinline__ void ntt_rounds(std::integer_sequence<int, RD...>, uint64_t* sm, int sub, int o, int tile,
                                           uint64_t q, const TwPair* tw) {
    ((ntt_round<LOGN, FWD, COLS, EB, STAGED, RD, LAZY>(sm, sub, o, tile, q, tw), __syncthreads()), ...);
}

template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED>
constexpr size_t smem_bytes() {
    using P = Phase<LOGN, FWD, COLS, EB, STAGED>;
    return 8 * (size_t)(P::TILE + P::TILE / 16) + (STAGED ? 16 * (size_t)P::TW : 0);
}

// Registers: 8-residue rounds fit 64 registers (4 CTAs of 256 threads per SM); 16-residue
// rounds get up to 128 (4 CTAs of 128 threads).
template <int EB>
constexpr int min_blocks() {
    return 4;
}

// Addressing of one limb: either a strided batch (blockIdx.y = limb, blockIdx.z = polynomial,
// modulus from a LimbMap) or an entry of a job table (blockIdx.y + 65535 * blockIdx.z).  The
// first phase may read from a different buffer than it writes (src -> dst); the second phase
// works in place on dst.
template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, bool TABLE>
__global__ void __launch_bounds__(Phase<LOGN, FWD, COLS, EB, STAGED>::THREADS, min_blocks<EB>())
    k_ntt_phase(uint64_t* __restrict__ data, size_t poly_stride, LimbMap map, const NttJob* __restrict__ jobs,
                int njobs, const Modulus* __restrict__ mods, const TwPair* __restrict__ tw_base) {
    using P = Phase<LOGN, FWD, COLS, EB, STAGED>;
    constexpr int N = P::N;
    constexpr int E = P::E;
    constexpr bool FIRST = FWD ? COLS : !COLS;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* sm = smem;                                                             // data tile, padded
    TwPair* tw_s = reinterpret_cast<TwPair*>(smem + P::TILE + P::TILE / 16);        // staged twiddles

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
    const TwPair* tw = tw_base + (size_t)mi * 2 * N + (FWD ? 0 : N);
    const int tile = blockIdx.x;
    const int t = threadIdx.x;

#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int e = t + k * P::THREADS;
        sm[pad16(e)] = xin[tile_offset<LOGN, FWD, COLS, EB, STAGED>(tile, e)];
    }
    if (STAGED) {
        const ulonglong2* src2 = reinterpret_cast<const ulonglong2*>(tw);
        ulonglong2* dst2 = reinterpret_cast<ulonglong2*>(tw_s);
        if (COLS) {
            for (int e = t; e < P::TW; e += P::THREADS) dst2[e] = __ldg(src2 + e);
        } else {
            // row-stage k: SUBS * 2^k contiguous table entries (twiddle_src order)
#pragma unroll
            for (int k = 0; k < P::MB; ++k) {
                const int cnt = P::SUBS << k;
                const int dst = P::SUBS * ((1 << k) - 1);
                const size_t src = ((size_t)1 << (P::NB1 + k)) + (size_t)tile * cnt;
                for (int e = t; e < cnt; e += P::THREADS) dst2[dst + e] = __ldg(src2 + src + e);
            }
        }
    }
    __syncthreads();

    const int sub = COLS ? t % P::SUBS : t >> P::OB;
    const int o = COLS ? t / P::SUBS : t & ((1 << P::OB) - 1);
    const TwPair* twr = STAGED ? tw_s : tw;
    // forward transforms under kLazyForwardLimit skip the per-butterfly reduction (uniform per CTA)
    const bool lazy = FWD && q < kLazyForwardLimit;
    if (lazy)
        ntt_rounds<LOGN, FWD, COLS, EB, STAGED, true>(std::make_integer_sequence<int, P::ROUNDS>{}, sm, sub, o, tile,
                                                      q, twr);
    else
        ntt_rounds<LOGN, FWD, COLS, EB, STAGED, false>(std::make_integer_sequence<int, P::ROUNDS>{}, sm, sub, o, tile,
                                                       q, twr);

    uint64_t n_inv = 0, n_inv_s = 0;
    if (P::LAST && !FWD) {
        n_inv = mods[mi].n_inv;
        n_inv_s = mods[mi].n_inv_shoup;
    }
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int e = t + k * P::THREADS;
        uint64_t val = sm[pad16(e)];
        if (P::LAST) val = FWD ? (lazy ? reduce64(val, mods[mi]) : red4q(val, q)) : mul_shoup(val, n_inv, n_inv_s, q);
        x[tile_offset<LOGN, FWD, COLS, EB, STAGED>(tile, e)] = val;
    }
}

// The forward row phase of one job-table limb with an element-wise epilogue (NttEpiJob): the
// same rounds and final reduction as k_ntt_phase<LOGN, true, false, ...>, then the epilogue in
// place of the store.  The epilogue's operands (acc, in: the tile's contiguous words) are
// copied into shared memory with cp.async when the block starts, so their loads overlap the
// rounds instead of stalling the final step; out may alias acc or in, since each word is read
// and written by this block only.
template <int LOGN, int EB, bool STAGED>
constexpr size_t rows_epi_smem() {
    using P = Phase<LOGN, true, false, EB, STAGED>;
    return smem_bytes<LOGN, true, false, EB, STAGED>() + 2 * 8 * (size_t)P::TILE;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem) : "memory");
}

template <int LOGN, int EB, bool STAGED>
__global__ void __launch_bounds__(Phase<LOGN, true, false, EB, STAGED>::THREADS, min_blocks<EB>())
    k_ntt_rows_epi(const NttEpiJob* __restrict__ jobs, int njobs, const Modulus* __restrict__ mods,
                   const TwPair* __restrict__ tw_base) {
    using P = Phase<LOGN, true, false, EB, STAGED>;
    constexpr int N = P::N;
    constexpr int E = P::E;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* sm = smem;
    TwPair* tw_s = reinterpret_cast<TwPair*>(smem + P::TILE + P::TILE / 16);
    uint64_t* acc_s = smem + smem_bytes<LOGN, true, false, EB, STAGED>() / 8;
    uint64_t* in_s = acc_s + P::TILE;
    const int j = blockIdx.y + 65535 * blockIdx.z;
    if (j >= njobs) return;
    const NttEpiJob job = jobs[j];
    const int mi = job.mod;
    const Modulus m = mods[mi];
    const TwPair* tw = tw_base + (size_t)mi * 2 * N;
    const int tile = blockIdx.x;
    const int t = threadIdx.x;
    // the row tile is P::TILE contiguous words at tile * TILE: 16-byte copies when the operand
    // limbs are 16-byte aligned (they start on a word; tile * TILE keeps any 16-byte alignment),
    // 8-byte copies otherwise
    const size_t base = (size_t)tile * P::TILE;
    const bool need_acc = job.kind == kEpiCombine;
    const bool need_in = job.kind == kEpiRescale || job.c0 != 0;
    const uintptr_t align = (need_acc ? reinterpret_cast<uintptr_t>(job.acc) : 0) |
                            (need_in ? reinterpret_cast<uintptr_t>(job.in) : 0);
    if ((align & 15) == 0) {
        for (int c = t; c < P::TILE / 2; c += P::THREADS) {
            if (need_acc) cp_async16(acc_s + 2 * c, job.acc + base + 2 * c);
            if (need_in) cp_async16(in_s + 2 * c, job.in + base + 2 * c);
        }
    } else {
        for (int e = t; e < P::TILE; e += P::THREADS) {
            if (need_acc) cp_async8(acc_s + e, job.acc + base + e);
            if (need_in) cp_async8(in_s + e, job.in + base + e);
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int e = t + k * P::THREADS;
        sm[pad16(e)] = job.data[tile_offset<LOGN, true, false, EB, STAGED>(tile, e)];
    }
    if (STAGED) {
        const ulonglong2* src2 = reinterpret_cast<const ulonglong2*>(tw);
        ulonglong2* dst2 = reinterpret_cast<ulonglong2*>(tw_s);
#pragma unroll
        for (int k = 0; k < P::MB; ++k) {
            const int cnt = P::SUBS << k;
            const int dst = P::SUBS * ((1 << k) - 1);
            const size_t src = ((size_t)1 << (P::NB1 + k)) + (size_t)tile * cnt;
            for (int e = t; e < cnt; e += P::THREADS) dst2[dst + e] = __ldg(src2 + src + e);
        }
    }
    __syncthreads();
    const int sub = t >> P::OB;
    const int o = t & ((1 << P::OB) - 1);
    const TwPair* twr = STAGED ? tw_s : tw;
    const bool lazy = m.q < kLazyForwardLimit;
    if (lazy)
        ntt_rounds<LOGN, true, false, EB, STAGED, true>(std::make_integer_sequence<int, P::ROUNDS>{}, sm, sub, o, tile,
                                                       m.q, twr);
    else
        ntt_rounds<LOGN, true, false, EB, STAGED, false>(std::make_integer_sequence<int, P::ROUNDS>{}, sm, sub, o,
                                                        tile, m.q, twr);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    const uint64_t q = m.q;
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int e = t + k * P::THREADS;
        const uint64_t raw = sm[pad16(e)];
        const uint64_t v = lazy ? reduce64(raw, m) : red4q(raw, q);
        job.out[base + e] = epilogue_value(job, need_acc ? acc_s[e] : 0, need_in ? in_s[e] : 0, v, q);
    }
}

template <int LOGN, int EB, bool STAGED>
void launch_rows_epi(const Context& c, const NttEpiJob* jobs, int njobs, cudaStream_t s) {
    using P = Phase<LOGN, true, false, EB, STAGED>;
    constexpr size_t sm = rows_epi_smem<LOGN, EB, STAGED>();
    static const bool opted = [] {
        cudaFuncSetAttribute(k_ntt_rows_epi<LOGN, EB, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        return true;
    }();
    (void)opted;
    const dim3 grid(P::N / P::TILE, njobs < 65535 ? njobs : 65535, (njobs + 65534) / 65535);
    k_ntt_rows_epi<LOGN, EB, STAGED><<<grid, P::THREADS, sm, s>>>(jobs, njobs, c.d_mod,
                                                                  reinterpret_cast<const TwPair*>(c.d_tw));
}

template <int LOGN>
void rows_epi_variant(const Context& c, int variant, const NttEpiJob* jobs, int njobs, cudaStream_t s) {
    switch (variant) {
        case 0: launch_rows_epi<LOGN, 3, true>(c, jobs, njobs, s); break;
        case 1: launch_rows_epi<LOGN, 3, false>(c, jobs, njobs, s); break;
        case 2: launch_rows_epi<LOGN, 4, true>(c, jobs, njobs, s); break;
        default: launch_rows_epi<LOGN, 4, false>(c, jobs, njobs, s); break;
    }
}

template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED, bool TABLE>
void enable_smem() {
    // opt in to more than 48 KiB of dynamic shared memory once per kernel instance
    static const bool done = [] {
        cudaFuncSetAttribute(k_ntt_phase<LOGN, FWD, COLS, EB, STAGED, TABLE>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<LOGN, FWD, COLS, EB, STAGED>());
        return true;
    }();
    (void)done;
}

template <int LOGN, bool FWD, bool COLS, int EB, bool STAGED>
void launch_geom(const Context& c, uint64_t* data, int limbs, int polys, size_t stride, LimbMap map,
                 const NttJob* jobs, int njobs, cudaStream_t s) {
    using P = Phase<LOGN, FWD, COLS, EB, STAGED>;
    constexpr size_t sm = smem_bytes<LOGN, FWD, COLS, EB, STAGED>();
    const TwPair* tw = reinterpret_cast<const TwPair*>(c.d_tw);
    if (jobs) {
        enable_smem<LOGN, FWD, COLS, EB, STAGED, true>();
        const dim3 grid(P::N / P::TILE, njobs < 65535 ? njobs : 65535, (njobs + 65534) / 65535);
        // algorithmic bytes: every residue read once and written once per transform, i.e. 8 B
        // per residue for each of the two phases (16 N B per limb-transform)
        Probe probe(kClsNtt, 8.0 * P::N * njobs, s);
        k_ntt_phase<LOGN, FWD, COLS, EB, STAGED, true><<<grid, P::THREADS, sm, s>>>(nullptr, 0, map, jobs, njobs,
                                                                                   c.d_mod, tw);
    } else {
        enable_smem<LOGN, FWD, COLS, EB, STAGED, false>();
        const dim3 grid(P::N / P::TILE, limbs, polys);
        Probe probe(kClsNtt, 8.0 * P::N * limbs * polys, s);
        k_ntt_phase<LOGN, FWD, COLS, EB, STAGED, false><<<grid, P::THREADS, sm, s>>>(data, stride, map, nullptr, 0,
                                                                                    c.d_mod, tw);
    }
}

// One phase with the geometry `variant` (kNttGeometries order).
template <int LOGN, bool FWD, bool COLS>
void launch_phase(const Context& c, int variant, uint64_t* data, int limbs, int polys, size_t stride, LimbMap map,
                  const NttJob* jobs, int njobs, cudaStream_t s) {
    switch (variant) {
        case 0: launch_geom<LOGN, FWD, COLS, 3, true>(c, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 1: launch_geom<LOGN, FWD, COLS, 3, false>(c, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 2: launch_geom<LOGN, FWD, COLS, 4, true>(c, data, limbs, polys, stride, map, jobs, njobs, s); break;
        default: launch_geom<LOGN, FWD, COLS, 4, false>(c, data, limbs, polys, stride, map, jobs, njobs, s); break;
    }
}

template <int LOGN>
void run_phase(const Context& c, bool fwd, bool cols, int variant, uint64_t* data, int limbs, int polys, size_t stride,
               LimbMap map, const NttJob* jobs, int njobs, cudaStream_t s) {
    if (fwd) {
        if (cols) launch_phase<LOGN, true, true>(c, variant, data, limbs, polys, stride, map, jobs, njobs, s);
        else launch_phase<LOGN, true, false>(c, variant, data, limbs, polys, stride, map, jobs, njobs, s);
    } else {
        if (cols) launch_phase<LOGN, false, true>(c, variant, data, limbs, polys, stride, map, jobs, njobs, s);
        else launch_phase<LOGN, false, false>(c, variant, data, limbs, polys, stride, map, jobs, njobs, s);
    }
}

void phase_dispatch(const Context& c, bool fwd, bool cols, int variant, uint64_t* data, int limbs, int polys,
                    size_t stride, LimbMap map, const NttJob* jobs, int njobs, cudaStream_t s) {
    switch (c.logN) {
        case 10: run_phase<10>(c, fwd, cols, variant, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 11: run_phase<11>(c, fwd, cols, variant, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 12: run_phase<12>(c, fwd, cols, variant, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 13: run_phase<13>(c, fwd, cols, variant, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 14: run_phase<14>(c, fwd, cols, variant, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 15: run_phase<15>(c, fwd, cols, variant, data, limbs, polys, stride, map, jobs, njobs, s); break;
        case 16: run_phase<16>(c, fwd, cols, variant, data, limbs, polys, stride, map, jobs, njobs, s); break;
        default: fail(kInvalid, "ntt: ring degree must be 2^10 .. 2^16");
    }
}

void dispatch(const Context& c, uint64_t* data, int limbs, int polys, size_t stride, LimbMap map,
              const NttJob* jobs, int njobs, bool fwd, cudaStream_t s) {
    if (jobs ? njobs <= 0 : (limbs <= 0 || polys <= 0)) return;
    if (!jobs && (polys > 65535 || limbs > 65535)) fail(kInvalid, "ntt: too many limbs or polynomials in one batch");
    const int d = fwd ? 0 : 1;
    // forward: columns then rows; inverse: rows then columns
    const bool first_cols = fwd;
    phase_dispatch(c, fwd, first_cols, c.ntt_variant[d][first_cols ? 1 : 0], data, limbs, polys, stride, map, jobs,
                   njobs, s);
    phase_dispatch(c, fwd, !first_cols, c.ntt_variant[d][first_cols ? 0 : 1], data, limbs, polys, stride, map, jobs,
                   njobs, s);
    check_cuda(cudaGetLastError(), "ntt launch");
}

// Tuned choices per (device, ring degree), shared by every context of the process.
struct TuneKey {
    int device, logN;
    bool operator<(const TuneKey& o) const { return device != o.device ? device < o.device : logN < o.logN; }
};
std::mutex g_tune_mutex;
std::map<TuneKey, NttTuning> g_tuned;

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

void ntt_jobs_phase(const Context& c, const NttJob* d_jobs, int njobs, bool forward, bool cols, cudaStream_t s) {
    if (njobs <= 0) return;
    phase_dispatch(c, forward, cols, c.ntt_variant[forward ? 0 : 1][cols ? 1 : 0], nullptr, 0, 0, 0, LimbMap{0, 0, 0},
                   d_jobs, njobs, s);
    check_cuda(cudaGetLastError(), "ntt launch");
}

void ntt_rows_epilogue_jobs(const Context& c, const NttEpiJob* d_jobs, int njobs, double bytes, cudaStream_t s) {
    if (njobs <= 0) return;
    // booked as NTT work: the phase's share plus the epilogue's words (ntt_epilogue_bytes)
    Probe probe(kClsNtt, bytes, s);
    // 8 residues per thread with twiddles from the table whatever the tuner chose for the plain
    // row phase: the prefetched operands take 32 KiB of shared memory, which leaves 4 blocks per
    // SM only in this geometry
    const int v = 1;
    switch (c.logN) {
        case 10: rows_epi_variant<10>(c, v, d_jobs, njobs, s); break;
        case 11: rows_epi_variant<11>(c, v, d_jobs, njobs, s); break;
        case 12: rows_epi_variant<12>(c, v, d_jobs, njobs, s); break;
        case 13: rows_epi_variant<13>(c, v, d_jobs, njobs, s); break;
        case 14: rows_epi_variant<14>(c, v, d_jobs, njobs, s); break;
        case 15: rows_epi_variant<15>(c, v, d_jobs, njobs, s); break;
        case 16: rows_epi_variant<16>(c, v, d_jobs, njobs, s); break;
        default: fail(kInvalid, "ntt: ring degree must be 2^10 .. 2^16");
    }
    check_cuda(cudaGetLastError(), "ntt epilogue launch");
}

void ntt_phase_geometry(const Context& c, bool forward, bool cols, int variant, uint64_t* data, int limbs, int polys,
                        size_t poly_stride, LimbMap map, cudaStream_t s) {
    if (variant < 0 || variant >= kNttGeometries) fail(kInvalid, "ntt: unknown geometry");
    if (limbs <= 0 || polys <= 0) return;
    phase_dispatch(c, forward, cols, variant, data, limbs, polys, poly_stride, map, nullptr, 0, s);
    check_cuda(cudaGetLastError(), "ntt launch");
}

// Time every geometry of every (direction, phase) the way the batched circuits launch the
// transform: job-table launches of 64 limbs over a scratch batch larger than the L2 cache (160 MB
// of limbs) cycling over the context's moduli, so lazy and full-reduction moduli are both
// represented; best of three passes after one warm-up.  A geometry replaces the default
// (8 residues per thread, staged twiddles) only when it is at least 5 % faster, so timing noise
// does not flip the choice.  Phases are timed on their own: each is one full pass over the
// batch whatever the other phase does, and every geometry computes the same words, so the
// choices combine freely.
void ntt_autotune(Context& c) {
    {
        std::lock_guard<std::mutex> g(g_tune_mutex);
        auto it = g_tuned.find({c.device, c.logN});
        if (it != g_tuned.end()) {
            c.tuning = it->second;
            for (int d = 0; d < 2; ++d)
                for (int p = 0; p < 2; ++p) c.ntt_variant[d][p] = it->second.chosen[d][p];
            return;
        }
    }
    const size_t N = c.N;
    const int kTuneLimbs = (int)((size_t{160} << 20) / (8 * N));
    const int kTuneBatch = 64;
    const int nm = (int)(c.nq + c.np);
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    uint64_t* buf = nullptr;
    NttJob* d_jobs = nullptr;
    if (cudaMalloc(&buf, (size_t)kTuneLimbs * N * 8) != cudaSuccess ||
        cudaMalloc(&d_jobs, (size_t)kTuneLimbs * sizeof(NttJob)) != cudaSuccess) {
        // no room for the timing batch: keep the default geometry (tuning.limbs = 0 says so)
        cudaGetLastError();
        cudaFree(buf);
        return;
    }
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NttTuning tn{};
    auto release = [&] {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
        cudaFree(buf);
        cudaFree(d_jobs);
    };
    try {
        check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "ntt autotune: stream");
        check_cuda(cudaEventCreate(&e0), "ntt autotune: event");
        check_cuda(cudaEventCreate(&e1), "ntt autotune: event");
        check_cuda(cudaMemsetAsync(buf, 0, (size_t)kTuneLimbs * N * 8, s), "ntt autotune: clear");
        std::vector<NttJob> jobs(kTuneLimbs);
        for (int l = 0; l < kTuneLimbs; ++l) jobs[l] = {buf + (size_t)l * N, buf + (size_t)l * N, l % nm, 0};
        check_cuda(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(NttJob), cudaMemcpyHostToDevice, s),
                   "ntt autotune: jobs");
        for (int d = 0; d < 2; ++d)
            for (int p = 0; p < 2; ++p) {
                for (int v = 0; v < kNttGeometries; ++v) {
                    float t_best = 1e30f;
                    for (int rep = 0; rep < 4; ++rep) {
                        check_cuda(cudaEventRecord(e0, s), "ntt autotune: record");
                        // launches of kTuneBatch limbs, the size of a batched key switch's NTT
                        // launch, so block tails and occupancy weigh as they do in the circuits
                        for (int l0 = 0; l0 < kTuneLimbs; l0 += kTuneBatch)
                            phase_dispatch(c, d == 0, p == 1, v, nullptr, 0, 0, 0, LimbMap{0, 0, 0}, d_jobs + l0,
                                           std::min(kTuneBatch, kTuneLimbs - l0), s);
                        check_cuda(cudaEventRecord(e1, s), "ntt autotune: record");
                        check_cuda(cudaEventSynchronize(e1), "ntt autotune: wait");
                        float ms = 0;
                        check_cuda(cudaEventElapsedTime(&ms, e0, e1), "ntt autotune: time");
                        if (rep > 0) t_best = std::min(t_best, ms);
                    }
                    tn.ms[d][p][v] = t_best;
                }
                int best_v = 0;
                for (int v = 1; v < kNttGeometries; ++v)
                    if (tn.ms[d][p][v] < 0.95f * tn.ms[d][p][0] && tn.ms[d][p][v] < tn.ms[d][p][best_v]) best_v = v;
                tn.chosen[d][p] = best_v;
            }
        tn.limbs = kTuneLimbs;
    } catch (...) {
        release();
        throw;
    }
    release();
    c.tuning = tn;
    for (int d = 0; d < 2; ++d)
        for (int p = 0; p < 2; ++p) c.ntt_variant[d][p] = tn.chosen[d][p];
    std::lock_guard<std::mutex> g(g_tune_mutex);
    g_tuned[{c.device, c.logN}] = tn;
}

}  // namespace wg
