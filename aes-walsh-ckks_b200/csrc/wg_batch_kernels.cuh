// Job structures and kernels of the batched path, shared by wg_batch.cu and wg_bsgs.cu.
//
// Block (x, y + 65535 z) runs tile x (256 coefficients) of job y of a device job table.
#pragma once
#include <algorithm>

#include "wg_batch.hpp"
#include "wg_internal.hpp"
#include "wg_keyswitch.cuh"

namespace wg {
namespace bk {
namespace {  // each translation unit gets its own copy of the kernels

constexpr int kT = 256;

// One digit (ModUp) or one accumulator polynomial (ModDown): the same jobs feed the fused
// kernels of wg_ksfuse.cu.
using ModUpJob = ModUpNttJob;
using ModDownJob = ModDownNttJob;
struct MacJob {
    const uint64_t* key;
    const uint64_t* key_term;
    const uint64_t* digits;
    uint64_t* acc;
    size_t part_stride;
    int L, K, parts, alpha, key_level, i;
};
// Key inner product of up to kMacGroup switches that share the key, the level and the digit
// layout, for one QP limb: the key words of a coefficient are loaded once for all of them.
constexpr int kMacGroup = 8;
struct MacGroupJob {
    const uint64_t* key;
    const uint64_t* key_term[kMacGroup];
    const uint64_t* digits[kMacGroup];
    uint64_t* acc[kMacGroup];
    size_t part_stride;
    int L, K, parts, alpha, key_level, i, n, pad;
};
struct CombineJob {
    const uint64_t* acc;
    const uint64_t* contrib;
    const uint64_t* b_in;
    const uint64_t* a_in;
    uint64_t* b_out;
    uint64_t* a_out;
    int L, K, qi, b_add, a_add, pad;
};
struct GatherJob {
    const uint64_t* src_b;
    const uint64_t* src_a;
    uint64_t* b;
    uint64_t* a;
    uint64_t galois;
};
struct TensorJob {
    uint64_t* b1;
    uint64_t* a1;
    const uint64_t* b2;
    const uint64_t* a2;
    uint64_t* c2;
    int mod;
    int pad;
};
struct RescalePrepJob {
    const uint64_t* drop;
    uint64_t* rem;
    uint64_t one_s, half;
    int pmod, qmod;
};
struct RescaleFinishJob {
    uint64_t* x;
    const uint64_t* rem;
    uint64_t inv_p, inv_p_s;
    int mod, pad;
};

// The elementwise kernels take kWide words per thread, kT x kWide coefficients per block (N is at
// least 1024): a thread's loads all go out before its arithmetic, and a block outlives its read of
// the job table by more than one word.  Word r of a thread is wide_index(r), so each of the kWide
// loads of a warp is coalesced.  These kernels (kb_tensor here; kb_scalar, kb_lincomb, kb_pmul,
// kb_copy and kb_add in wg_ctops.cuh) are launched with grid_wide only.
constexpr int kWide = 4;
__device__ __forceinline__ size_t wide_index(int r) {
    return ((size_t)blockIdx.x * kWide + r) * kT + threadIdx.x;
}

template <class J>
__device__ __forceinline__ const J* job_of(const J* jobs, int n) {
    const int j = blockIdx.y + 65535 * blockIdx.z;
    return j < n ? jobs + j : nullptr;
}

__global__ void __launch_bounds__(kT) kb_modup(const ModUpJob* jobs, int n, const Modulus* mods, size_t N) {
    const ModUpJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t coeff = (size_t)blockIdx.x * kT + threadIdx.x;
    modup_coeff(*j->desc, mods, j->src, j->digit, N, coeff);
}

__global__ void __launch_bounds__(kT) kb_mac(const MacJob* jobs, int n, const Modulus* mods, int nq, size_t N) {
    const MacJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t coeff = (size_t)blockIdx.x * kT + threadIdx.x;
    mac_coeff(mods, nq, j->L, j->K, j->parts, j->alpha, j->key, j->key_level, j->key_term, j->digits, j->part_stride,
              j->acc, N, j->i, coeff);
}

// acc_{a,b}[i] = sum_parts REDC(digit_part[i] * key_part_{a,b}[i]) for the NC switches of a group,
// parts accumulated in order as in mac_accumulate (wg_keyswitch.cuh).  NC is a compile-time
// count so that every digit load of a part is unconditional and all of them are in flight at once.
template <int NC>
__device__ __forceinline__ void mac_group(const MacGroupJob* j, const Modulus* mods, int nq, size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kT + threadIdx.x;
    const int i = j->i, L = j->L, K = j->K, T = L + K;
    const bool is_p = i >= L;
    const Modulus& m = mods[is_p ? nq + (i - L) : i];
    const uint64_t q = m.q, qninv = m.qninv;
    const size_t key_limbs = (size_t)j->key_level + 1 + K;
    const size_t klimb = is_p ? (size_t)j->key_level + 1 + (i - L) : (size_t)i;
    const size_t at = (size_t)i * N + coeff;
    uint64_t acc_a[NC], acc_b[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc_a[c] = acc_b[c] = 0;
    for (int p = 0; p < j->parts; ++p) {
        const int s0 = p * j->alpha, s1 = s0 + j->alpha < L ? s0 + j->alpha : L;
        const bool own = !is_p && i >= s0 && i < s1;
        const uint64_t ka = j->key[(((size_t)p * 2 + 0) * key_limbs + klimb) * N + coeff];
        const uint64_t kb = j->key[(((size_t)p * 2 + 1) * key_limbs + klimb) * N + coeff];
        uint64_t d[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) d[c] = own ? j->key_term[c][at] : j->digits[c][p * j->part_stride + at];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            acc_a[c] = add_mod(acc_a[c], mont_mul(d[c], ka, q, qninv), q);
            acc_b[c] = add_mod(acc_b[c], mont_mul(d[c], kb, q, qninv), q);
        }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        j->acc[c][at] = acc_a[c];
        j->acc[c][(size_t)T * N + at] = acc_b[c];
    }
}

__global__ void __launch_bounds__(kT, 3) kb_mac_group(const MacGroupJob* jobs, int n, const Modulus* mods, int nq,
                                                      size_t N) {
    const MacGroupJob* j = job_of(jobs, n);
    if (!j) return;
    static_assert(kMacGroup == 8, "one case per group size");
    switch (j->n) {  // the same for every thread of the block
        case 1: mac_group<1>(j, mods, nq, N); break;
        case 2: mac_group<2>(j, mods, nq, N); break;
        case 3: mac_group<3>(j, mods, nq, N); break;
        case 4: mac_group<4>(j, mods, nq, N); break;
        case 5: mac_group<5>(j, mods, nq, N); break;
        case 6: mac_group<6>(j, mods, nq, N); break;
        case 7: mac_group<7>(j, mods, nq, N); break;
        default: mac_group<8>(j, mods, nq, N); break;
    }
}

__global__ void __launch_bounds__(kT) kb_moddown(const ModDownJob* jobs, int n, const Modulus* mods, int nq, int K,
                                                 size_t N) {
    const ModDownJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t coeff = (size_t)blockIdx.x * kT + threadIdx.x;
    moddown_all_limbs(mods, nq, j->L, K, j->src_p, N, coeff, j->inv, j->inv_s, j->out);
}

__global__ void __launch_bounds__(kT) kb_combine(const CombineJob* jobs, int n, const Modulus* mods, size_t N) {
    const CombineJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t coeff = (size_t)blockIdx.x * kT + threadIdx.x;
    combine_coeff(mods[j->qi].q, j->L, j->K, j->acc, j->contrib, j->b_in, j->a_in, j->b_out, j->a_out, j->b_add,
                  j->a_add, N, j->qi, coeff);
}

__global__ void __launch_bounds__(kT) kb_gather(const GatherJob* jobs, int n, int logN) {
    const GatherJob* j = job_of(jobs, n);
    if (!j) return;
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    const uint32_t s = automorphism_src(i, j->galois, logN);
    j->b[i] = j->src_b[s];
    j->a[i] = j->src_a[s];
}

__global__ void __launch_bounds__(kT) kb_tensor(const TensorJob* jobs, int n, const Modulus* mods) {
    const TensorJob* j = job_of(jobs, n);
    if (!j) return;
    const Modulus m = mods[j->mod];
    uint64_t xa[kWide], xb[kWide], ya[kWide], yb[kWide];
#pragma unroll
    for (int r = 0; r < kWide; ++r) {
        const size_t k = wide_index(r);
        xa[r] = j->a1[k], xb[r] = j->b1[k], ya[r] = j->a2[k], yb[r] = j->b2[k];
    }
#pragma unroll
    for (int r = 0; r < kWide; ++r) {
        const size_t k = wide_index(r);
        j->c2[k] = barrett_mul(xa[r], ya[r], m);
        const uint64_t tmp = barrett_mul(xb[r], ya[r], m);
        j->b1[k] = barrett_mul(xb[r], yb[r], m);
        j->a1[k] = add_mod(barrett_mul(xa[r], yb[r], m), tmp, m.q);
    }
}

// Same two steps as k_rescale_prep / k_rescale_finish in wg_ops.cu.
__global__ void __launch_bounds__(kT) kb_rescale_prep(const RescalePrepJob* jobs, int n, const Modulus* mods) {
    const RescalePrepJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t p = mods[j->pmod].q, q = mods[j->qmod].q;
    uint64_t shift = j->drop[k] + (p >> 1);
    if (shift >= p) shift -= p;
    j->rem[k] = sub_mod(reduce_shoup(shift, q, j->one_s), j->half, q);
}

__global__ void __launch_bounds__(kT) kb_rescale_finish(const RescaleFinishJob* jobs, int n, const Modulus* mods) {
    const RescaleFinishJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q = mods[j->mod].q;
    uint64_t x = j->x[k];
    if (x >= q) x -= q;
    j->x[k] = mul_shoup(sub_mod(x, j->rem[k], q), j->inv_p, j->inv_p_s, q);
}

dim3 grid_for(const Context& c, size_t njobs) {
    return dim3((unsigned)(c.N / kT), (unsigned)std::min<size_t>(njobs, 65535), (unsigned)((njobs + 65534) / 65535));
}
// The grid of the kWide-words-per-thread kernels.
dim3 grid_wide(const Context& c, size_t njobs) {
    return dim3((unsigned)(c.N / (kT * kWide)), (unsigned)std::min<size_t>(njobs, 65535),
                (unsigned)((njobs + 65534) / 65535));
}

// The launches of one batched rescale (ckks_rescale, src/ckks/operations/arith/ckks_rescale.cpp:
// 68-148) over polynomials of any levels: add() records a polynomial x at level lv with lv
// remainder limbs of scratch, plan() puts the job tables into a JobTable, run() launches.
// Fused (Context::fuse over the polynomials): the inverse row phase of the dropped limbs, one
// fused launch (inverse column phase, rounded remainders, forward column phase; k_rescale_ntt)
// and the forward row phase with the finish step as its epilogue (k_ntt_rows_epi): 3 launches.
// Without: inverse NTT, kb_rescale_prep, forward NTT, kb_rescale_finish: 6 launches.  Same words.
struct RescaleJobs {
    struct Poly {
        uint64_t* x;
        size_t lv;
        uint64_t* rem;
    };
    std::vector<Poly> polys;
    bool fused = false;
    std::vector<NttJob> drop, rem_ntt;
    std::vector<RescalePrepJob> prep;
    std::vector<RescaleFinishJob> fin;
    std::vector<RescaleNttJob> cols;
    std::vector<NttEpiJob> rows;
    double prep_bytes = 0.0, fin_bytes = 0.0;
    const NttJob *jd = nullptr, *jr = nullptr;
    const RescalePrepJob* jp = nullptr;
    const RescaleFinishJob* jf = nullptr;
    const RescaleNttJob* jc = nullptr;
    const NttEpiJob* je = nullptr;

    bool empty() const { return polys.empty(); }
    void add(uint64_t* x, size_t lv, uint64_t* rem) { polys.push_back({x, lv, rem}); }
    // builds the jobs (fused when the batch fills the device: Context::fuse) into t
    void plan(const Context& c, JobTable& t) {
        const size_t N = c.N;
        fused = c.fuse(polys.size());
        for (const Poly& pl : polys) {
            const size_t lv = pl.lv;
            uint64_t* x = pl.x;
            uint64_t* rem = pl.rem;
            const uint64_t* rc = c.rs_host.data() + c.rs_host_off[lv];
            uint64_t* dl = x + lv * N;
            drop.push_back({dl, dl, (int)lv, 0});
            if (fused) {
                cols.push_back({dl, rem, c.rs_one_s[lv], (int)lv, 0});
                for (size_t q = 0; q < lv; ++q)
                    rows.push_back({rem + q * N, nullptr, x + q * N, x + q * N, rc[lv + q], rc[2 * lv + q], (int)q,
                                    kEpiRescale});
            } else {
                for (size_t q = 0; q < lv; ++q) {
                    prep.push_back({dl, rem + q * N, rc[q], rc[3 * lv + q], (int)lv, (int)q});
                    rem_ntt.push_back({rem + q * N, rem + q * N, (int)q, 0});
                    fin.push_back({x + q * N, rem + q * N, rc[lv + q], rc[2 * lv + q], (int)q, 0});
                }
            }
            prep_bytes += 8.0 * N * (1.0 + lv);
            fin_bytes += 8.0 * N * 3.0 * lv;
        }
        jd = t.add(drop);
        if (fused) {
            jc = t.add(cols);
            je = t.add(rows);
        } else {
            jp = t.add(prep);
            jr = t.add(rem_ntt);
            jf = t.add(fin);
        }
    }
    void run(const Context& c, const JobTable& t, cudaStream_t s) const {
        if (drop.empty()) return;
        const size_t N = c.N;
        if (fused) {
            ntt_jobs_phase(c, t.at(jd), (int)drop.size(), false, false, s);
            rescale_ntt_jobs(c, t.at(jc), (int)cols.size(), prep_bytes, s);
            ntt_rows_epilogue_jobs(c, t.at(je), (int)rows.size(), ntt_epilogue_bytes(rows, N), s);
        } else {
            ntt_jobs(c, t.at(jd), (int)drop.size(), false, s);
            {
                Probe probe(kClsElementwise, prep_bytes, s);
                kb_rescale_prep<<<grid_for(c, prep.size()), kT, 0, s>>>(t.at(jp), (int)prep.size(), c.d_mod);
            }
            ntt_jobs(c, t.at(jr), (int)rem_ntt.size(), true, s);
            Probe probe(kClsElementwise, fin_bytes, s);
            kb_rescale_finish<<<grid_for(c, fin.size()), kT, 0, s>>>(t.at(jf), (int)fin.size(), c.d_mod);
        }
        check_cuda(cudaGetLastError(), "batched rescale launch");
    }
};

}  // namespace
}  // namespace bk
}  // namespace wg
