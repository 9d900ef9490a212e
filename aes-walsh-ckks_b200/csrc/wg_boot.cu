// Bootstrapping boundary steps, batched over ciphertexts: ModRaise from q0 to a target level and
// the level-0 dense-to-sparse key switch through q0 and p0.
//
// Reference:
//   ModRaise                ckks_modraise_inplace, modraise_eval_poly_from_q0,
//                           src/ckks/operations/bootstrap/ckks_modraise.cpp:12-110
//   dense-to-sparse switch  ckks_q0p0_key_switch_level0_inplace (folded Montgomery key),
//                           hps_base_change_single_limb,
//                           src/ckks/operations/keyswitch/ckks_keyswitch.cpp:1645-1856
// The q0p0 switch reuses the batched key-switch kernels with a two-limb QP basis (q0, p0): the
// compact key [a: q0, p0][b: q0, p0] is a one-part key of level 0 with one P limb, and the
// level-0 folded ModDown inverse row starts with p0^-1 mod q0.
#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_internal.hpp"

namespace wg {
using namespace bk;

namespace {

struct LiftJob {
    const uint64_t* src;  // q0 limb, coefficient form
    uint64_t* dst;        // target limb
    int mod;              // target modulus index
    int pad;
};

struct BaseChangeJob {
    const uint64_t* src;  // q0 limb, coefficient form
    uint64_t* dst;        // p0 limb
};

// out = (centered lift of x mod q0) mod q_l  (center_lift_mod_q / signed_to_mod_q)
__global__ void __launch_bounds__(kT) kb_modraise_lift(const LiftJob* jobs, int n, const Modulus* mods) {
    const LiftJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t x = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q0 = mods[0].q, q = mods[j->mod].q;
    const uint64_t v = j->src[x];
    uint64_t r;
    if (v > (q0 >> 1)) {
        const uint64_t m = (q0 - v) % q;
        r = m == 0 ? 0 : q - m;
    } else {
        r = v % q;
    }
    j->dst[x] = r;
}

// hps_base_change_single_limb from q0 to p0
__global__ void __launch_bounds__(kT) kb_q0_to_p0(const BaseChangeJob* jobs, int n, const Modulus* mods, int nq) {
    const BaseChangeJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t x = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q0 = mods[0].q;
    const Modulus& mp = mods[nq];
    const uint64_t reduced = red4q(j->src[x], q0);
    const uint64_t r = barrett_u64(reduced, mp.q, mp.mu_hi);
    const uint64_t s = barrett_u64(q0, mp.q, mp.mu_hi);
    j->dst[x] = reduced >= (q0 >> 1) + 1 ? sub_mod(r, s, mp.q) : r;
}

}  // namespace

void modraise(Context& c, size_t count, size_t target_level, uint64_t* const* b, uint64_t* const* a,
              cudaStream_t s) {
    if (count == 0) return;
    const size_t N = c.N, L = target_level + 1;
    uint64_t* coeff = c.batch_buffers(s).arena(c, 2 * count * N, s);
    std::vector<NttJob> intt, ntt;
    std::vector<LiftJob> lift;
    for (size_t ci = 0; ci < count; ++ci)
        for (int poly = 0; poly < 2; ++poly) {
            uint64_t* x = poly ? a[ci] : b[ci];
            uint64_t* cf = coeff + (2 * ci + poly) * N;
            intt.push_back({x, cf, 0, 0});
            for (size_t l = 0; l < L; ++l) {
                lift.push_back({cf, x + l * N, (int)l, 0});
                ntt.push_back({x + l * N, x + l * N, (int)l, 0});
            }
        }
    JobTable t;
    const NttJob* j1 = t.add(intt);
    const LiftJob* j2 = t.add(lift);
    const NttJob* j3 = t.add(ntt);
    t.upload(c, s);
    ntt_jobs(c, t.at(j1), (int)intt.size(), false, s);
    {
        Probe probe(kClsElementwise, 8.0 * N * (double)(lift.size() + 2 * count), s);
        kb_modraise_lift<<<grid_for(c, lift.size()), kT, 0, s>>>(t.at(j2), (int)lift.size(), c.d_mod);
    }
    ntt_jobs(c, t.at(j3), (int)ntt.size(), true, s);
    check_cuda(cudaGetLastError(), "modraise launch");
}

void q0p0_switch(Context& c, size_t count, uint64_t* const* b, uint64_t* const* a, const KeyEntry& key,
                 cudaStream_t s) {
    if (count == 0) return;
    const size_t N = c.N, nq = c.nq;
    // per ciphertext: coefficient copy of a (N), digit [q0 unused, p0] (2N),
    // accumulators [a: q0, p0][b: q0, p0] (4N), contributions [a, b] (2N)
    const size_t per = 9 * N;
    uint64_t* ws = c.batch_buffers(s).arena(c, count * per, s);
    std::vector<NttJob> intt_a, ntt_dp, intt_p, ntt_c;
    std::vector<BaseChangeJob> bc;
    std::vector<MacJob> mac;
    std::vector<ModDownJob> md;
    std::vector<CombineJob> comb;
    for (size_t ci = 0; ci < count; ++ci) {
        uint64_t* cf = ws + ci * per;
        uint64_t* dg = cf + N;
        uint64_t* acc = dg + 2 * N;
        uint64_t* ct = acc + 4 * N;
        intt_a.push_back({a[ci], cf, 0, 0});
        bc.push_back({cf, dg + N});
        ntt_dp.push_back({dg + N, dg + N, (int)nq, 0});
        for (int i = 0; i < 2; ++i)
            mac.push_back({key.d_data, a[ci], dg, acc, 2 * N, 1, 1, 1, (int)c.alpha, 0, i});
        intt_p.push_back({acc + N, acc + N, (int)nq, 0});
        intt_p.push_back({acc + 3 * N, acc + 3 * N, (int)nq, 0});
        md.push_back({acc + N, ct, c.fold_inv[0], c.fold_inv_s[0], 1, 0});
        md.push_back({acc + 3 * N, ct + N, c.fold_inv[0], c.fold_inv_s[0], 1, 0});
        ntt_c.push_back({ct, ct, 0, 0});
        ntt_c.push_back({ct + N, ct + N, 0, 0});
        comb.push_back({acc, ct, b[ci], a[ci], b[ci], a[ci], 1, 1, 0, 1, 0, 0});
    }
    JobTable t;
    const NttJob* j1 = t.add(intt_a);
    const BaseChangeJob* j2 = t.add(bc);
    const NttJob* j3 = t.add(ntt_dp);
    const MacJob* j4 = t.add(mac);
    const NttJob* j5 = t.add(intt_p);
    const ModDownJob* j6 = t.add(md);
    const NttJob* j7 = t.add(ntt_c);
    const CombineJob* j8 = t.add(comb);
    t.upload(c, s);
    ntt_jobs(c, t.at(j1), (int)intt_a.size(), false, s);
    {
        Probe probe(kClsModUp, 16.0 * N * bc.size(), s);
        kb_q0_to_p0<<<grid_for(c, bc.size()), kT, 0, s>>>(t.at(j2), (int)bc.size(), c.d_mod, (int)nq);
    }
    ntt_jobs(c, t.at(j3), (int)ntt_dp.size(), true, s);
    {
        Probe probe(kClsKeyMac, 8.0 * N * mac.size() * 5.0, s);
        kb_mac<<<grid_for(c, mac.size()), kT, 0, s>>>(t.at(j4), (int)mac.size(), c.d_mod, (int)nq, N);
    }
    ntt_jobs(c, t.at(j5), (int)intt_p.size(), false, s);
    {
        Probe probe(kClsModDown, 16.0 * N * md.size(), s);
        kb_moddown<<<grid_for(c, md.size()), kT, 0, s>>>(t.at(j6), (int)md.size(), c.d_mod, (int)nq, 1, N);
    }
    ntt_jobs(c, t.at(j7), (int)ntt_c.size(), true, s);
    {
        Probe probe(kClsCombine, 8.0 * N * 7.0 * comb.size(), s);
        kb_combine<<<grid_for(c, comb.size()), kT, 0, s>>>(t.at(j8), (int)comb.size(), c.d_mod, N);
    }
    check_cuda(cudaGetLastError(), "dense-to-sparse launch");
}

}  // namespace wg
