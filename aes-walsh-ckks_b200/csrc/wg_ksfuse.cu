// Key-switch ModUp and ModDown, and the rescale's remainder step, fused with the NTT column
// phases around them.
//
// Unfused, a hybrid key switch (ckks_hybrid_key_switch_inplace,
// src/ckks/operations/keyswitch/ckks_keyswitch.cpp:1330-1641) moves every intermediate limb
// through device memory between separate launches: the inverse NTT of the key term writes its
// coefficients, ModUp reads them and writes the digits, the forward NTT reads and rewrites the
// digits twice (one pass per phase); after the key inner product the same happens around
// ModDown.  Here one CTA per (digit or accumulator, column tile) runs
//
//   inverse column phase of its source limbs -> N^-1 -> ModUp / ModDown -> forward column
//   phase of every output limb
//
// in shared memory (wg_ksfuse.cuh), so the coefficient-form source limbs and the un-transformed
// outputs never reach device memory.  Per switch at walsh15's top level (L = 13, K = 4, three
// digits of 5, 5 and 3 source limbs, 38 destination limbs) the NTT/ModUp/ModDown traffic falls
// from 425 to 255 limb passes of 8N bytes, with the same words written.
#include <utility>

#include "wg_internal.hpp"
#include "wg_ksfuse.cuh"

namespace wg {
namespace {
using namespace ksf;
using ntt::TwPair;

template <int LOGN, bool FWD, bool LAZY, int... RD>
__device__ __forceinline__ void col_rounds(std::integer_sequence<int, RD...>, uint64_t* sm, int tile, int t,
                                           uint64_t q, const TwPair* tw) {
    ((col_round<LOGN, FWD, RD, LAZY>(sm, tile, t, q, tw), __syncthreads()), ...);
}

template <int LOGN>
__device__ __forceinline__ void inverse_cols(uint64_t* sm, int tile, int t, const Modulus& m, const TwPair* tw) {
    col_rounds<LOGN, false, false>(std::make_integer_sequence<int, Geom<LOGN>::ROUNDS>{}, sm, tile, t, m.q, tw);
    scale_n_inv<LOGN>(sm, t, m);
}

template <int LOGN>
__device__ __forceinline__ void forward_cols(uint64_t* sm, int tile, int t, uint64_t q, const TwPair* tw) {
    // moduli below kLazyForwardLimit skip the per-butterfly reduction, as k_ntt_phase does
    if (q < ntt::kLazyForwardLimit)
        col_rounds<LOGN, true, true>(std::make_integer_sequence<int, Geom<LOGN>::ROUNDS>{}, sm, tile, t, q, tw);
    else
        col_rounds<LOGN, true, false>(std::make_integer_sequence<int, Geom<LOGN>::ROUNDS>{}, sm, tile, t, q, tw);
}

// Shared memory: the source tiles, then the work tile (PAD words each).  Resident blocks per SM
// (the launch bounds) follow from it: up to 4 source tiles of 8.5 KiB leave room for 5 blocks,
// the rescale's single tile for 6 (register-limited).
template <int LOGN>
constexpr size_t fused_smem(int tiles) {
    return 8 * (size_t)Geom<LOGN>::PAD * (size_t)(tiles + 1);
}

// Block (tile, job): one digit's column tile.  W >= every job's digit width.
template <int LOGN, int W>
__global__ void __launch_bounds__(Geom<LOGN>::THREADS, W <= 4 ? 5 : 4)
    k_modup_ntt(const ModUpNttJob* __restrict__ jobs, int njobs, const Modulus* __restrict__ mods,
                const TwPair* __restrict__ tw_base) {
    using G = Geom<LOGN>;
    const int j = blockIdx.y + 65535 * blockIdx.z;
    if (j >= njobs) return;
    extern __shared__ __align__(16) uint64_t smem[];
    const ModUpNttJob job = jobs[j];
    const ModUpDesc& d = *job.desc;
    const int n = d.src_count, first = d.src_first, nd = d.dst_count;
    const int tile = blockIdx.x, t = threadIdx.x;
    uint64_t* work = smem + (size_t)n * G::PAD;

    // every source tile in flight at once, each awaited just before its inverse column phase
    for (int i = 0; i < n; ++i) {
        load_tile_async<LOGN>(smem + (size_t)i * G::PAD, job.src + (size_t)(first + i) * G::N, tile, t);
        cp_async_commit();
    }
    double alpha[G::E];
#pragma unroll
    for (int k = 0; k < G::E; ++k) alpha[k] = 0.0;
    for (int i = 0; i < n; ++i) {
        const int mi = first + i;
        const Modulus m = mods[mi];
        uint64_t* sm = smem + (size_t)i * G::PAD;
        cp_async_wait_upto(n - 1 - i);
        __syncthreads();
        inverse_cols<LOGN>(sm, tile, t, m, tw_base + (size_t)mi * 2 * G::N + G::N);
        modup_scale<LOGN>(sm, t, d, i, m.q, alpha);
    }
    uint32_t hps[G::E];
#pragma unroll
    for (int k = 0; k < G::E; ++k) hps[k] = hps_count(alpha[k], n);
    for (int dst = 0; dst < nd; ++dst) {
        const int mi = __ldg(d.dst_mod + dst);
        const uint64_t q = mods[mi].q;
        modup_value<LOGN, W>(work, smem, t, d, dst, q, hps);
        __syncthreads();
        forward_cols<LOGN>(work, tile, t, q, tw_base + (size_t)mi * 2 * G::N);
        store_tile<LOGN>(work, job.digit + (size_t)__ldg(d.dst_limb + dst) * G::N, tile, t);
    }
}

// Block (tile, job): one accumulator polynomial's column tile.  FMA: the alpha sum's rounding
// (moddown_hps); KW >= K.
template <int LOGN, bool FMA, int KW>
__global__ void __launch_bounds__(Geom<LOGN>::THREADS, KW <= 4 ? 5 : 4)
    k_moddown_ntt(const ModDownNttJob* __restrict__ jobs, int njobs, const Modulus* __restrict__ mods, int nq, int K,
                  const TwPair* __restrict__ tw_base) {
    using G = Geom<LOGN>;
    const int j = blockIdx.y + 65535 * blockIdx.z;
    if (j >= njobs) return;
    extern __shared__ __align__(16) uint64_t smem[];
    const ModDownNttJob job = jobs[j];
    const int tile = blockIdx.x, t = threadIdx.x;
    uint64_t* work = smem + (size_t)K * G::PAD;
    const Modulus* pmods = mods + nq;

    for (int pi = 0; pi < K; ++pi) {
        load_tile_async<LOGN>(smem + (size_t)pi * G::PAD, job.src_p + (size_t)pi * G::N, tile, t);
        cp_async_commit();
    }
    for (int pi = 0; pi < K; ++pi) {
        const Modulus m = pmods[pi];
        uint64_t* sm = smem + (size_t)pi * G::PAD;
        cp_async_wait_upto(K - 1 - pi);
        __syncthreads();
        inverse_cols<LOGN>(sm, tile, t, m, tw_base + (size_t)(nq + pi) * 2 * G::N + G::N);
    }
    uint32_t hps[G::E];
    moddown_hps<LOGN, KW, FMA>(smem, t, pmods, K, hps);
    for (int qi = 0; qi < job.L; ++qi) {
        const uint64_t q = mods[qi].q;
        moddown_value<LOGN, KW>(work, smem, t, K, q, job.inv + (size_t)qi * K, job.inv_s + (size_t)qi * K, hps);
        __syncthreads();
        forward_cols<LOGN>(work, tile, t, q, tw_base + (size_t)qi * 2 * G::N);
        store_tile<LOGN>(work, job.out + (size_t)qi * G::N, tile, t);
    }
}

// Block (tile, job): one polynomial's column tile of a rescale.
template <int LOGN>
__global__ void __launch_bounds__(Geom<LOGN>::THREADS, 6)
    k_rescale_ntt(const RescaleNttJob* __restrict__ jobs, int njobs, const Modulus* __restrict__ mods,
                  const TwPair* __restrict__ tw_base) {
    using G = Geom<LOGN>;
    const int j = blockIdx.y + 65535 * blockIdx.z;
    if (j >= njobs) return;
    extern __shared__ __align__(16) uint64_t smem[];
    const RescaleNttJob job = jobs[j];
    const int tile = blockIdx.x, t = threadIdx.x, lv = job.lv;
    uint64_t* drop = smem;
    uint64_t* work = smem + G::PAD;
    const Modulus mp = mods[lv];
    load_tile<LOGN>(drop, job.drop, tile, t);
    __syncthreads();
    inverse_cols<LOGN>(drop, tile, t, mp, tw_base + (size_t)lv * 2 * G::N + G::N);
    for (int qi = 0; qi < lv; ++qi) {
        const uint64_t q = mods[qi].q;
        rescale_value<LOGN>(work, drop, t, mp.q, q, __ldg(job.rc + qi), __ldg(job.rc + 3 * lv + qi));
        __syncthreads();
        forward_cols<LOGN>(work, tile, t, q, tw_base + (size_t)qi * 2 * G::N);
        store_tile<LOGN>(work, job.rem + (size_t)qi * G::N, tile, t);
    }
}

template <int LOGN>
void launch_rescale(const Context& c, const RescaleNttJob* jobs, int njobs, cudaStream_t s) {
    using G = Geom<LOGN>;
    const dim3 grid(G::TILES, njobs < 65535 ? njobs : 65535, (njobs + 65534) / 65535);
    k_rescale_ntt<LOGN><<<grid, G::THREADS, fused_smem<LOGN>(1), s>>>(jobs, njobs, c.d_mod,
                                                                      reinterpret_cast<const TwPair*>(c.d_tw));
}

template <int LOGN, int W>
void launch_modup_w(const Context& c, const ModUpNttJob* jobs, int njobs, int max_src, cudaStream_t s) {
    using G = Geom<LOGN>;
    static const bool opted = [] {
        cudaFuncSetAttribute(k_modup_ntt<LOGN, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fused_smem<LOGN>(W));
        return true;
    }();
    (void)opted;
    const dim3 grid(G::TILES, njobs < 65535 ? njobs : 65535, (njobs + 65534) / 65535);
    k_modup_ntt<LOGN, W><<<grid, G::THREADS, fused_smem<LOGN>(max_src), s>>>(jobs, njobs, c.d_mod,
                                                                              reinterpret_cast<const TwPair*>(c.d_tw));
}

template <int LOGN>
void launch_modup(const Context& c, const ModUpNttJob* jobs, int njobs, int max_src, cudaStream_t s) {
    if (max_src <= 4)
        launch_modup_w<LOGN, 4>(c, jobs, njobs, max_src, s);
    else if (max_src <= 8)
        launch_modup_w<LOGN, 8>(c, jobs, njobs, max_src, s);
    else
        launch_modup_w<LOGN, kMaxDigitWidth>(c, jobs, njobs, max_src, s);
}

template <int LOGN, bool FMA, int KW>
void launch_moddown_k(const Context& c, const ModDownNttJob* jobs, int njobs, cudaStream_t s) {
    using G = Geom<LOGN>;
    static const bool opted = [] {
        cudaFuncSetAttribute(k_moddown_ntt<LOGN, FMA, KW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fused_smem<LOGN>(KW));
        return true;
    }();
    (void)opted;
    const dim3 grid(G::TILES, njobs < 65535 ? njobs : 65535, (njobs + 65534) / 65535);
    k_moddown_ntt<LOGN, FMA, KW><<<grid, G::THREADS, fused_smem<LOGN>((int)c.np), s>>>(
        jobs, njobs, c.d_mod, (int)c.nq, (int)c.np, reinterpret_cast<const TwPair*>(c.d_tw));
}

template <int LOGN, bool FMA>
void launch_moddown_f(const Context& c, const ModDownNttJob* jobs, int njobs, cudaStream_t s) {
    if (c.np <= 4)
        launch_moddown_k<LOGN, FMA, 4>(c, jobs, njobs, s);
    else if (c.np <= 8)
        launch_moddown_k<LOGN, FMA, 8>(c, jobs, njobs, s);
    else
        launch_moddown_k<LOGN, FMA, kMaxPLimbs>(c, jobs, njobs, s);
}

template <int LOGN>
void launch_moddown(const Context& c, const ModDownNttJob* jobs, int njobs, bool fma, cudaStream_t s) {
    if (fma)
        launch_moddown_f<LOGN, true>(c, jobs, njobs, s);
    else
        launch_moddown_f<LOGN, false>(c, jobs, njobs, s);
}

}  // namespace

void modup_ntt_jobs(const Context& c, const ModUpNttJob* d_jobs, int njobs, int max_src, double bytes,
                    cudaStream_t s) {
    if (njobs <= 0) return;
    if (max_src < 1 || max_src > kMaxDigitWidth) fail(kInvalid, "fused modup: digit width out of range");
    Probe probe(kClsModUp, bytes, s);
    switch (c.logN) {
        case 10: launch_modup<10>(c, d_jobs, njobs, max_src, s); break;
        case 11: launch_modup<11>(c, d_jobs, njobs, max_src, s); break;
        case 12: launch_modup<12>(c, d_jobs, njobs, max_src, s); break;
        case 13: launch_modup<13>(c, d_jobs, njobs, max_src, s); break;
        case 14: launch_modup<14>(c, d_jobs, njobs, max_src, s); break;
        case 15: launch_modup<15>(c, d_jobs, njobs, max_src, s); break;
        case 16: launch_modup<16>(c, d_jobs, njobs, max_src, s); break;
        default: fail(kInvalid, "fused modup: ring degree must be 2^10 .. 2^16");
    }
    check_cuda(cudaGetLastError(), "fused modup launch");
}

void rescale_ntt_jobs(const Context& c, const RescaleNttJob* d_jobs, int njobs, double bytes, cudaStream_t s) {
    if (njobs <= 0) return;
    Probe probe(kClsElementwise, bytes, s);
    switch (c.logN) {
        case 10: launch_rescale<10>(c, d_jobs, njobs, s); break;
        case 11: launch_rescale<11>(c, d_jobs, njobs, s); break;
        case 12: launch_rescale<12>(c, d_jobs, njobs, s); break;
        case 13: launch_rescale<13>(c, d_jobs, njobs, s); break;
        case 14: launch_rescale<14>(c, d_jobs, njobs, s); break;
        case 15: launch_rescale<15>(c, d_jobs, njobs, s); break;
        case 16: launch_rescale<16>(c, d_jobs, njobs, s); break;
        default: fail(kInvalid, "fused rescale: ring degree must be 2^10 .. 2^16");
    }
    check_cuda(cudaGetLastError(), "fused rescale launch");
}

void moddown_ntt_jobs(const Context& c, const ModDownNttJob* d_jobs, int njobs, double bytes, cudaStream_t s,
                      bool fma_alpha) {
    if (njobs <= 0) return;
    if (c.np < 1 || c.np > (size_t)kMaxPLimbs) fail(kInvalid, "fused moddown: P limb count out of range");
    Probe probe(kClsModDown, bytes, s);
    switch (c.logN) {
        case 10: launch_moddown<10>(c, d_jobs, njobs, fma_alpha, s); break;
        case 11: launch_moddown<11>(c, d_jobs, njobs, fma_alpha, s); break;
        case 12: launch_moddown<12>(c, d_jobs, njobs, fma_alpha, s); break;
        case 13: launch_moddown<13>(c, d_jobs, njobs, fma_alpha, s); break;
        case 14: launch_moddown<14>(c, d_jobs, njobs, fma_alpha, s); break;
        case 15: launch_moddown<15>(c, d_jobs, njobs, fma_alpha, s); break;
        case 16: launch_moddown<16>(c, d_jobs, njobs, fma_alpha, s); break;
        default: fail(kInvalid, "fused moddown: ring degree must be 2^10 .. 2^16");
    }
    check_cuda(cudaGetLastError(), "fused moddown launch");
}

}  // namespace wg
