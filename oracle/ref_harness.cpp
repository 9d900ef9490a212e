// Test-infrastructure harness around the reference library compiled from its own sources.
//
// It exposes the reference's own functions through plain C entry points so the Python tests
// can (1) pin the C restatement in ckks_oracle.c against the real thing and (2) write golden
// fixtures.  Nothing in the product links this file.  Every entry point returns 0 on success
// and a negative value when the reference threw (the message is kept for ref_last_error()).
//
// Reference entry points wrapped here:
//   find_p_and_q_primes                src/util/random.cpp:115
//   generate_negacyclic_ntt_twiddles   src/math/ntt/ntt.cpp:54
//   ntt_{forward,inverse}_rns_flat_inplace  src/math/ntt/ntt.cpp:416,433
//   CKKSContext::CKKSContext           src/ckks/context/ckks_context.cpp:603
//   ckks_hybrid_key_switch_inplace     src/ckks/operations/keyswitch/ckks_keyswitch.cpp:1330
//   ckks_rotate_inplace                src/ckks/operations/keyswitch/ckks_rotation.cpp:41
//   ckks_conjugate_inplace             src/ckks/operations/keyswitch/ckks_conjugate.cpp:112
//   ckks_relin_hybrid_inplace          src/ckks/operations/keyswitch/ckks_relin.cpp:8
//   ckks_mul_inplace (ct x ct)         src/ckks/operations/arith/ckks_mul.cpp:90
//   ckks_rescale                       src/ckks/operations/arith/ckks_rescale.cpp:68
//   ckks_hoist_ciphertext_a_qp_eval / ckks_hybrid_key_switch_hoisted_inplace
//                                      src/ckks/operations/keyswitch/ckks_keyswitch.cpp:344,1072

#include <algorithm>
#include <map>
#include <array>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include <omp.h>

#include "ckks_aes_params.hpp"
#include "ckks_ciphertext.hpp"
#include "ckks_linear_transform.hpp"
#include "ckks_modraise.hpp"
#include "ckks_evalpoly.hpp"
#include "ckks_bootstrap_dft.hpp"
#include "ckks_aes_ctr_walsh_sbox.hpp"
#include "ckks_aes_ctr.hpp"
#include "hybrid_key_folding.hpp"
#include "polynomial.hpp"
#include "hybrid_key_montgomery.hpp"
#include "secret_key_generation.hpp"
#include "rotation_key_generation.hpp"
#include "conjugation_key_generation.hpp"
#include "ckks_walsh_sbox.hpp"
#include "ckks_encoding.hpp"
#include "ckks_bootstrap_evalmod_inplace.hpp"
#include "ckks_evalmod_scale_plan.hpp"
#include "binboot_k_bound.hpp"
#include "poly_approx.hpp"
#include "ckks_context.hpp"
#include "ckks_conjugate.hpp"
#include "ckks_keyswitch.hpp"
#include "ckks_mul.hpp"
#include "ckks_addition.hpp"
#include "aes/aes_tables.hpp"
#include "ckks_params.hpp"
#include "ckks_relin.hpp"
#include "ckks_rescale.hpp"
#include "ckks_rotation.hpp"
#include "ntt.hpp"
#include "fft.hpp"
#include "random.hpp"

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    } catch (...) {
        g_last_error = "unknown exception";
        return -2;
    }
}

MyVector<uint64_t> copy_in(const uint64_t* src, size_t n) {
    return MyVector<uint64_t>(src, src + n);
}

void copy_out(const MyVector<uint64_t>& src, uint64_t* dst) {
    std::memcpy(dst, src.data(), src.size() * sizeof(uint64_t));
}

// Key layout shared with the oracle and the device library:
// [part][poly: 0 = a, 1 = b][limb: key_level+1 Q limbs then K P limbs][N]
std::vector<CKKSCiphertext> keys_from_flat(const uint64_t* flat, size_t parts, size_t key_level,
                                           size_t p_count, size_t N) {
    const size_t limbs = key_level + 1 + p_count;
    std::vector<CKKSCiphertext> out;
    out.reserve(parts);
    for (size_t part = 0; part < parts; ++part) {
        const uint64_t* a = flat + (part * 2 + 0) * limbs * N;
        const uint64_t* b = flat + (part * 2 + 1) * limbs * N;
        out.emplace_back(N, copy_in(a, limbs * N), copy_in(b, limbs * N), 1.0L, key_level);
    }
    return out;
}

void keys_to_flat(std::span<const CKKSCiphertext> keys, uint64_t* flat) {
    size_t off = 0;
    for (const auto& k : keys) {
        std::memcpy(flat + off, k.getA().data(), k.getA().size() * sizeof(uint64_t));
        off += k.getA().size();
        std::memcpy(flat + off, k.getB().data(), k.getB().size() * sizeof(uint64_t));
        off += k.getB().size();
    }
}

}  // namespace

// Defined with external linkage in src/ckks/operations/bootstrap/ckks_linear_transform.cpp:1174
// but not declared in its header.
CKKSCiphertext ckks_apply_linear_transform_owned_stage_qp(const CKKSContext& context, const CKKSCiphertext& ct,
                                                          const CKKSLinearTransformOwnedStage& owned_stage);

namespace {

struct RefCtx {
    CKKSContext ctx;
    std::map<uint64_t, CKKSLinearTransformPlan> scaled_s2c;  // SlotToCoeff plans by input scale ratio
    explicit RefCtx(CKKSParams p) : ctx(std::move(p)) {}
};

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_last_error.c_str(); }

int ref_find_primes(const uint64_t* p_bits, size_t np, const uint64_t* q_bits, size_t nq,
                    uint64_t N, uint64_t* p_out, uint64_t* q_out) {
    return guarded([&] {
        std::vector<uint64_t> pb(p_bits, p_bits + np), qb(q_bits, q_bits + nq);
        auto [p, q] = find_p_and_q_primes(pb, qb, N);
        std::copy(p.begin(), p.end(), p_out);
        std::copy(q.begin(), q.end(), q_out);
    });
}

int ref_ntt_tables(uint64_t N, uint64_t q, uint64_t* fwd, uint64_t* fwd_shoup, uint64_t* inv,
                   uint64_t* inv_shoup_np1, uint64_t* n_inv, uint64_t* barrett_lo_hi) {
    return guarded([&] {
        auto t = generate_negacyclic_ntt_twiddles(N, q);
        copy_out(t.forward_ntt, fwd);
        copy_out(t.forward_shoup, fwd_shoup);
        copy_out(t.inverse_ntt, inv);
        copy_out(t.inverse_shoup, inv_shoup_np1);
        *n_inv = t.N_inv;
        barrett_lo_hi[0] = t.barrett_const.low;
        barrett_lo_hi[1] = t.barrett_const.high;
    });
}

// Context with custom moduli schedule and no bootstrapping keys.
void* ref_ctx_create(uint64_t N, const uint64_t* q_bits, size_t nq, const uint64_t* p_bits,
                     size_t np, size_t dnum, size_t hamming_weight, double sigma, double scale,
                     const int64_t* rotations, size_t nrot) {
    RefCtx* out = nullptr;
    const int rc = guarded([&] {
        CKKSParamsConfig cfg;
        cfg.secure = false;
        cfg.bts_keys = false;
        cfg.N = N;
        cfg.q_bits.assign(q_bits, q_bits + nq);
        cfg.mult_depth = nq - 1;
        cfg.q0_bit = q_bits[0];
        cfg.q_bit = nq > 1 ? q_bits[1] : q_bits[0];
        cfg.p_bits.assign(p_bits, p_bits + np);
        cfg.pmoduli_count = np;
        cfg.dnum = dnum;
        cfg.secret_key_hamming_weight = hamming_weight;
        cfg.sigma = sigma;
        cfg.scale = scale;
        cfg.rotate_values.assign(rotations, rotations + nrot);
        out = new RefCtx(CKKSParams(std::move(cfg)));
    });
    return rc == 0 ? out : nullptr;
}

void ref_ctx_destroy(void* h) { delete static_cast<RefCtx*>(h); }

int ref_ctx_moduli(void* h, uint64_t* q_out, size_t* nq, uint64_t* p_out, size_t* np) {
    return guarded([&] {
        const auto& p = static_cast<RefCtx*>(h)->ctx.getParams();
        *nq = p.getModuli().size();
        *np = p.getPModuli().size();
        if (q_out) std::copy(p.getModuli().begin(), p.getModuli().end(), q_out);
        if (p_out) std::copy(p.getPModuli().begin(), p.getPModuli().end(), p_out);
    });
}

// Forward/inverse NTT of `limbs` consecutive Q limbs (limb-major, N each).
int ref_ctx_ntt(void* h, uint64_t* poly, size_t limbs, int inverse, int lazy) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const auto& p = c.getParams();
        if (inverse)
            ntt_inverse_rns_flat_inplace(poly, p.getN(), limbs, p.getModuli(), c.getTwiddleNtt(), lazy != 0);
        else
            ntt_forward_rns_flat_inplace(poly, p.getN(), limbs, p.getModuli(), c.getTwiddleNtt(), lazy != 0);
    });
}

// kind: 0 = rotation (by `rot`), 1 = conjugation, 2 = relinearization.
// Switching keys by kind: 0 rotation, 1 conjugation, 2 relinearization, 3 dense-to-sparse
// (compact q0/p0 key: one level-0 part whose a and b hold the q0 limb then the p0 limb),
// 4 sparse-to-dense (hybrid key at the top level).  Kinds 3 and 4 exist in bootstrapping
// contexts only.
static std::span<const CKKSCiphertext> key_span(const CKKSContext& c, int kind, int64_t rot) {
    switch (kind) {
        case 0: return c.getRotationKey(rot);
        case 1: return c.getConjugationKey();
        case 2: return c.getRelinHybrid(c.getParams().getMaxLevel());
        case 3: return c.getDenseToSparseSwitchKey();
        case 4: return c.getSparseToDenseSwitchKey();
        default: throw std::invalid_argument("ref_ctx_key: unknown key kind");
    }
}

int ref_ctx_key_shape(void* h, int kind, int64_t rot, size_t* parts, size_t* key_level) {
    return guarded([&] {
        std::span<const CKKSCiphertext> k = key_span(static_cast<RefCtx*>(h)->ctx, kind, rot);
        *parts = k.size();
        *key_level = k.empty() ? 0 : k.front().getLevel();
    });
}

// Words of one part's a (or b) polynomial of a key (kind 3 keys are compact).
int ref_ctx_key_words(void* h, int kind, int64_t rot, size_t* words) {
    return guarded([&] {
        std::span<const CKKSCiphertext> k = key_span(static_cast<RefCtx*>(h)->ctx, kind, rot);
        *words = k.empty() ? 0 : k.front().getA().size();
    });
}

int ref_ctx_key(void* h, int kind, int64_t rot, uint64_t* flat) {
    return guarded([&] { keys_to_flat(key_span(static_cast<RefCtx*>(h)->ctx, kind, rot), flat); });
}

// NTT-domain automorphism map (dst -> src) used by rotation (kind 0) or conjugation (kind 1).
int ref_ctx_map(void* h, int kind, int64_t rot, uint64_t* map_out) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const auto& m = kind == 0 ? c.getRotationNttMap(rot) : c.getConjugationNttMap();
        for (size_t i = 0; i < m.size(); ++i) map_out[i] = m[i];
    });
}

// The rotation (kind 0), conjugation (kind 1), relinearisation (kind 2), dense-to-sparse (kind 3)
// or sparse-to-dense (kind 4) switching key that generate_rotation_key_hybrid
// (src/ckks/context/rotation_key_generation.cpp:92-199) / generate_conjugation_key_hybrid
// (conjugation_key_generation.cpp) / encrypt_rlk_hybrid (relinearization_key_generation.cpp:
// 131-199, through ckks_encrypt_custom_eval) / generate_secret_key_switch_key_q0p0_hybrid and
// generate_secret_key_switch_key_hybrid (secret_key_generation.cpp:227-364; source `secret`,
// target `target`) build from `secret` (N ternary coefficients), with the mask
// `a` ([part][limbs][N], canonical, evaluation form) and the noise `e` ([part][N] integers)
// given instead of drawn: the same steps on the reference's own NTT, pointwise, folding and
// Montgomery helpers.  out: [part][a|b][limbs][N] as the context stores keys.
int ref_switch_key_from_parts(void* h, int kind, int64_t rotation, const int8_t* secret, const int8_t* target,
                              const uint64_t* a, const int64_t* e, uint64_t* out) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const auto& params = c.getParams();
        const size_t N = params.getN(), L = params.getMaxLevel() + 1, dnum = params.getDnum();
        const auto& qm = params.getModuli();
        const auto& pm = params.getPModuli();
        MyVector<uint64_t> qup(qm.begin(), qm.begin() + L);
        qup.insert(qup.end(), pm.begin(), pm.end());
        MyVector<Negacyclic_NTT_Twiddles> tw;
        for (size_t i = 0; i < L; ++i) tw.emplace_back(c.getTwiddleNtt()[i]);
        for (size_t i = 0; i < pm.size(); ++i) tw.emplace_back(c.getPTwiddleNtt()[i]);
        // apply_automorphism_to_secret with build_automorphism_map: coefficient i goes to
        // i * index mod 2N, negated past N
        auto automorph = [&](const MyVector<int8_t>& x, uint64_t index) {
            MyVector<int8_t> y(N, int8_t{0});
            for (size_t i = 0; i < N; ++i) {
                const size_t m = (size_t)(((unsigned __int128)i * index) % (2 * N));
                y[m >= N ? m - N : m] = m >= N ? (int8_t)-x[i] : x[i];
            }
            return y;
        };
        const MyVector<int8_t> s(secret, secret + N);
        MyVector<int8_t> x, y;  // b = P x (own limbs) + e - a y; kind 2: P s^2 + e - a s
        if (kind == 0) {
            x = s;
            y = automorph(s, rotation_automorphism_index(N, -rotation));
        } else if (kind == 1) {
            x = automorph(s, conjugation_automorphism_index(N));
            y = s;
        } else if (kind == 2) {
            x = s;
            y = s;
        } else {
            x = s;  // secret switch from `secret` to `target`
            y = MyVector<int8_t>(target, target + N);
        }
        if (kind == 3) {
            // generate_secret_key_switch_key_q0p0_hybrid (secret_key_generation.cpp:302-364): the
            // compact key over (q0, p0), plaintext source * p0 on q0, folded over {q0} and {p0}
            const MyVector<uint64_t> b01{qm[0], pm[0]}, q0v{qm[0]}, p0v{pm[0]};
            MyVector<Negacyclic_NTT_Twiddles> t01{c.getTwiddleNtt()[0], c.getPTwiddleNtt()[0]};
            const auto xs = ntt_secret_key(x, t01, N, b01);
            const auto ys = ntt_secret_key(y, t01, N, b01);
            MyVector<uint64_t> ptxt(2 * N, 0);
            std::copy(xs[0].begin(), xs[0].end(), ptxt.begin());
            pointwise_multiply_scalar_inplace_dispatch(ptxt.data(), pm[0] % qm[0], N, qm[0], t01[0]);
            MyVector<uint64_t> a_poly(a, a + 2 * N), e_poly(2 * N);
            for (size_t i = 0; i < 2; ++i)
                for (size_t j = 0; j < N; ++j) e_poly[i * N + j] = reduce_i64_mod_q(e[j], b01[i]);
            ntt_forward_rns_flat_inplace(e_poly.data(), N, 2, b01, t01, false);
            MyVector<uint64_t> as(N);
            for (size_t i = 0; i < 2; ++i) {
                pointwise_multiply_dispatch(a_poly.data() + i * N, ys[i].data(), as.data(), N, b01[i], t01[i]);
                poly_add_modq_inplace(ptxt.data() + i * N, e_poly.data() + i * N, N, b01[i]);
                poly_sub_modq_inplace(ptxt.data() + i * N, as.data(), N, b01[i]);
            }
            CKKSCiphertext key(N, std::move(a_poly), std::move(ptxt), 1.0, 0);
            if (params.fold_hybrid_keyswitch) ckks_fold_hybrid_switch_key_constants(key, q0v, p0v, t01);
            if (params.montgomery) ckks_convert_switch_key_to_montgomery_inplace(key, b01, t01);
            copy_out(key.getA(), out);
            copy_out(key.getB(), out + 2 * N);
            return;
        }
        const auto x_qup = ntt_secret_key(x, tw, N, qup);
        const auto y_qup = ntt_secret_key(y, tw, N, qup);
        MyVector<uint64_t> p_mod_m(qup.size(), 1);
        for (size_t i = 0; i < qup.size(); ++i)
            for (uint64_t p : pm) p_mod_m[i] = mul_mod_u64(p_mod_m[i], p % qup[i], qup[i], &tw[i].barrett_const);
        const size_t alpha = (L + dnum - 1) / dnum;
        const size_t T = qup.size();
        size_t off = 0, part_index = 0;
        for (size_t part = 0; part < dnum; ++part) {
            const size_t s0 = part * alpha, s1 = std::min(s0 + alpha, L);
            if (s0 >= s1) continue;
            MyVector<uint64_t> b_poly(N * T, 0);
            for (size_t i = s0; i < s1; ++i) {
                std::copy(x_qup[i].begin(), x_qup[i].end(), b_poly.data() + i * N);
                // encrypt_rlk_hybrid (relinearization_key_generation.cpp:131-199): s times s first
                if (kind == 2) pointwise_multiply_inplace_dispatch(b_poly.data() + i * N, x_qup[i].data(), N, qup[i], tw[i]);
                pointwise_multiply_scalar_inplace_dispatch(b_poly.data() + i * N, p_mod_m[i], N, qup[i], tw[i]);
            }
            MyVector<uint64_t> a_poly(a + part_index * T * N, a + (part_index + 1) * T * N);
            MyVector<uint64_t> e_poly(N * T);
            for (size_t i = 0; i < T; ++i)
                for (size_t j = 0; j < N; ++j) e_poly[i * N + j] = reduce_i64_mod_q(e[part_index * N + j], qup[i]);
            ntt_forward_rns_flat_inplace(e_poly.data(), N, T, qup, tw, false);
            MyVector<uint64_t> as(N);
            for (size_t i = 0; i < T; ++i) {
                pointwise_multiply_dispatch(a_poly.data() + i * N, y_qup[i].data(), as.data(), N, qup[i], tw[i]);
                poly_add_modq_inplace(b_poly.data() + i * N, e_poly.data() + i * N, N, qup[i]);
                poly_sub_modq_inplace(b_poly.data() + i * N, as.data(), N, qup[i]);
            }
            CKKSCiphertext key(N, std::move(a_poly), std::move(b_poly), 1.0, L - 1);
            if (params.fold_hybrid_keyswitch) ckks_fold_hybrid_switch_key_constants(key, qm, pm, tw);
            if (params.montgomery) ckks_convert_switch_key_to_montgomery_inplace(key, qup, tw);
            copy_out(key.getA(), out + off);
            off += key.getA().size();
            copy_out(key.getB(), out + off);
            off += key.getB().size();
            ++part_index;
        }
    });
}

// Secret key in NTT form for every Q limb: [limb][N].
int ref_ctx_secret(void* h, uint64_t* out) {
    return guarded([&] {
        const auto& sk = static_cast<RefCtx*>(h)->ctx.getSecretKey();
        size_t off = 0;
        for (const auto& limb : sk) {
            std::memcpy(out + off, limb.data(), limb.size() * sizeof(uint64_t));
            off += limb.size();
        }
    });
}

// The bootstrapping sparse secret in NTT form for every Q limb: [limb][N].
int ref_ctx_low_secret(void* h, uint64_t* out) {
    return guarded([&] {
        const auto& sk = static_cast<RefCtx*>(h)->ctx.getLowSecretKey();
        size_t off = 0;
        for (const auto& limb : sk) {
            std::memcpy(out + off, limb.data(), limb.size() * sizeof(uint64_t));
            off += limb.size();
        }
    });
}

// ckks_encrypt_custom_eval (src/ckks/encoding/ckks_encoding.cpp:478-520) of the evaluation-form
// plaintext `pt` at `level` under `secret` (N ternary coefficients), with the mask `a`
// ([level + 1][N]) and the noise `e` ([N] integers) given instead of drawn.
int ref_encrypt_from_parts(void* h, size_t level, const uint64_t* pt, const int8_t* secret, const uint64_t* a,
                           const int64_t* e, uint64_t* out_b, uint64_t* out_a) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN(), L = level + 1;
        const auto& qm = c.getParams().getModuli();
        MyVector<uint64_t> mods(qm.begin(), qm.begin() + L);
        MyVector<Negacyclic_NTT_Twiddles> tw(c.getTwiddleNtt().begin(), c.getTwiddleNtt().begin() + L);
        const auto sk = ntt_secret_key(MyVector<int8_t>(secret, secret + N), tw, N, mods);
        MyVector<uint64_t> e_poly(L * N), m(pt, pt + L * N), as(N);
        for (size_t i = 0; i < L; ++i)
            for (size_t j = 0; j < N; ++j) e_poly[i * N + j] = reduce_i64_mod_q(e[j], mods[i]);
        ntt_forward_rns_flat_inplace(e_poly.data(), N, L, mods, tw, false);
        for (size_t i = 0; i < L; ++i) {
            pointwise_multiply_dispatch(a + i * N, sk[i].data(), as.data(), N, mods[i], tw[i]);
            poly_add_modq_inplace(m.data() + i * N, e_poly.data() + i * N, N, mods[i]);
            poly_sub_modq_inplace(m.data() + i * N, as.data(), N, mods[i]);
        }
        copy_out(m, out_b);
        std::memcpy(out_a, a, L * N * sizeof(uint64_t));
    });
}

// Hybrid key switch with caller-supplied key material (flat layout as above).
int ref_keyswitch(void* h, size_t level, uint64_t* key_term, const uint64_t* key_flat, size_t parts,
                  size_t key_level, uint64_t* b, uint64_t* a, int b_add, int a_add, int montgomery) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t L = level + 1;
        auto keys = keys_from_flat(key_flat, parts, key_level, c.getParams().getPModuli().size(), N);
        auto kt = copy_in(key_term, L * N);
        auto bv = copy_in(b, L * N);
        auto av = copy_in(a, L * N);
        ckks_hybrid_key_switch_inplace(
            c, level, kt, std::span<const CKKSCiphertext>(keys.data(), keys.size()), bv, av,
            b_add ? CKKSHybridKeySwitchCombine::Add : CKKSHybridKeySwitchCombine::Assign,
            a_add ? CKKSHybridKeySwitchCombine::Add : CKKSHybridKeySwitchCombine::Assign,
            montgomery != 0);
        copy_out(bv, b);
        copy_out(av, a);
    });
}

// In-place ciphertext ops on (b, a) buffers of (level+1)*N residues each.
int ref_rotate(void* h, size_t level, uint64_t* b, uint64_t* a, int64_t rot) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t n = (level + 1) * c.getParams().getN();
        CKKSCiphertext ct(c.getParams().getN(), copy_in(a, n), copy_in(b, n), 1.0L, level);
        ckks_rotate_inplace(c, ct, rot);
        copy_out(ct.getB(), b);
        copy_out(ct.getA(), a);
    });
}

int ref_conjugate(void* h, size_t level, uint64_t* b, uint64_t* a) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t n = (level + 1) * c.getParams().getN();
        CKKSCiphertext ct(c.getParams().getN(), copy_in(a, n), copy_in(b, n), 1.0L, level);
        ckks_conjugate_inplace(c, ct);
        copy_out(ct.getB(), b);
        copy_out(ct.getA(), a);
    });
}

// (b1,a1) <- tensor with (b2,a2); writes c0 -> b1, c1 -> a1, c2 -> c2_out.
int ref_mul(void* h, size_t level, uint64_t* b1, uint64_t* a1, const uint64_t* b2, const uint64_t* a2,
            uint64_t* c2_out) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        CKKSCiphertext x(N, copy_in(a1, n), copy_in(b1, n), 1.0L, level);
        CKKSCiphertext y(N, copy_in(a2, n), copy_in(b2, n), 1.0L, level);
        ckks_mul_inplace(c, x, y);
        copy_out(x.getB(), b1);
        copy_out(x.getA(), a1);
        copy_out(x.getPoly(2), c2_out);
    });
}

int ref_relin(void* h, size_t level, uint64_t* c0, uint64_t* c1, const uint64_t* c2) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        MyVector<MyVector<uint64_t>> polys;
        polys.emplace_back(copy_in(c0, n));
        polys.emplace_back(copy_in(c1, n));
        polys.emplace_back(copy_in(c2, n));
        CKKSCiphertext ct(N, std::move(polys), 1.0L, level);
        ckks_relin_hybrid_inplace(c, ct);
        copy_out(ct.getB(), c0);
        copy_out(ct.getA(), c1);
    });
}

// Rescale `npolys` polynomials stored back to back ((level+1)*N each); the output keeps the
// same stride but only the first level*N residues of each polynomial are meaningful.
int ref_rescale(void* h, size_t level, size_t npolys, uint64_t* polys_flat) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        MyVector<MyVector<uint64_t>> polys;
        for (size_t i = 0; i < npolys; ++i) polys.emplace_back(copy_in(polys_flat + i * n, n));
        CKKSCiphertext ct(N, std::move(polys), 1.0L, level);
        ckks_rescale(c, ct);
        for (size_t i = 0; i < npolys; ++i)
            std::memcpy(polys_flat + i * n, ct.getPoly(i).data(), level * N * sizeof(uint64_t));
    });
}

// Hoisted rotations: one hoist of `a`, then one switch per rotation (rotation-key maps applied).
// out layout: [rot][poly: b then a][limb][N].
int ref_hoisted_rotations(void* h, size_t level, const uint64_t* b, const uint64_t* a,
                          const int64_t* rots, size_t nrot, uint64_t* out) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        CKKSCiphertext ct(N, copy_in(a, n), copy_in(b, n), 1.0L, level);
        CKKSHoistWorkspace ws;
        CKKSEvalHoistedCiphertextQP hoisted;
        ckks_hoist_ciphertext_a_qp_eval(c, ct, ws, hoisted);
        for (size_t r = 0; r < nrot; ++r) {
            MyVector<uint64_t> bo = copy_in(b, n);
            MyVector<uint64_t> ao(n, 0);
            const auto& map = c.getRotationNttMap(rots[r]);
            ckks_hybrid_key_switch_hoisted_inplace(
                c, hoisted, c.getRotationKey(rots[r]), bo, ao, CKKSHybridKeySwitchCombine::Add,
                CKKSHybridKeySwitchCombine::Assign, c.getParams().montgomery,
                std::span<const size_t>(map.data(), map.size()));
            copy_out(bo, out + (r * 2 + 0) * n);
            copy_out(ao, out + (r * 2 + 1) * n);
        }
    });
}

// The batched-ops workload on the reference CPU path: for each ciphertext i at level[i],
// multiply by its partner, relinearize, rescale and rotate by rots[i], with OpenMP over
// ciphertexts (the way the reference parallelizes independent ciphertexts).  Buffers hold
// (level_max+1)*N residues per polynomial; x_b/x_a are updated in place (rescaled level).
// Returns the wall time in seconds through *seconds.
int ref_batched_ops(void* h, size_t count, const size_t* levels, uint64_t* x_b, uint64_t* x_a,
                    const uint64_t* y_b, const uint64_t* y_a, const int64_t* rots, size_t stride,
                    int threads, double* seconds) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        std::string err;
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic) num_threads(threads)
        for (std::ptrdiff_t i = 0; i < static_cast<std::ptrdiff_t>(count); ++i) {
            try {
                const size_t level = levels[i];
                const size_t n = (level + 1) * N;
                const size_t off = static_cast<size_t>(i) * stride;
                CKKSCiphertext x(N, copy_in(x_a + off, n), copy_in(x_b + off, n), 1.0L, level);
                CKKSCiphertext y(N, copy_in(y_a + off, n), copy_in(y_b + off, n), 1.0L, level);
                ckks_mul_inplace(c, x, y);
                ckks_relin_hybrid_inplace(c, x);
                ckks_rescale(c, x);
                ckks_rotate_inplace(c, x, rots[i]);
                std::memcpy(x_b + off, x.getB().data(), x.getB().size() * sizeof(uint64_t));
                std::memcpy(x_a + off, x.getA().data(), x.getA().size() * sizeof(uint64_t));
            } catch (const std::exception& e) {
#pragma omp critical
                err = e.what();
            }
        }
        const auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
        if (!err.empty()) throw std::runtime_error(err);
    });
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// The reference's own CKKSParams presets (src/ckks/parameters/ckks_aes_params.hpp:211-235):
// 0 AESWalsh15, 1 XBootParamAes13Reference, 2 AESXBoot14Secure, 3 AESXBoot14SecureSparse1024,
// 4 AESXBoot15, 5 AESXBoot15Sparse1024.  Moduli (q: room for 64, p: room for 16), scale,
// depth, active slots, EvalMod K, S2C and C2S depths.
int ref_preset(int which, uint64_t* q, size_t* nq, uint64_t* p, size_t* np, double* scale, size_t* info) {
    return guarded([&] {
        const CKKSParams prm = which == 0   ? CKKSParams::AESWalsh15()
                               : which == 1 ? CKKSParams::XBootParamAes13Reference()
                               : which == 2 ? CKKSParams::AESXBoot14Secure()
                               : which == 3 ? CKKSParams::AESXBoot14SecureSparse1024()
                               : which == 4 ? CKKSParams::AESXBoot15()
                                            : CKKSParams::AESXBoot15Sparse1024();
        *nq = prm.getModuli().size();
        *np = prm.getPModuli().size();
        std::copy(prm.getModuli().begin(), prm.getModuli().end(), q);
        std::copy(prm.getPModuli().begin(), prm.getPModuli().end(), p);
        *scale = prm.getScale();
        info[0] = prm.getDepth();
        info[1] = prm.getBootstrapActiveSlotCount();
        info[2] = prm.getBootstrapEvalModK();
        info[3] = prm.getBootstrapS2CDepth();
        info[4] = prm.getBootstrapC2SDepth();
    });
}

// binboot_han_ki_discrete_multi_interval_approximate (src/math/poly_approx.cpp:565) called
// directly: coefficients, their count, max_error and the interval it reports.
int ref_evalmod_fit(double K, size_t degree, size_t double_angle, double radius, size_t points, double prune,
                    double* coeffs, size_t* n, double* max_error, double* interval) {
    return guarded([&] {
        const PolynomialApproximation a =
            binboot_han_ki_discrete_multi_interval_approximate(K, degree, double_angle, radius, points, prune);
        std::copy(a.chebyshev_coeffs.begin(), a.chebyshev_coeffs.end(), coeffs);
        *n = a.chebyshev_coeffs.size();
        *max_error = a.max_error;
        interval[0] = a.interval_min;
        interval[1] = a.interval_max;
    });
}

// required_binboot_k_bound (src/math/binboot_k_bound.cpp:53) at failure probability
// 2^log2_failure: its evalmod_k.
int ref_evalmod_k_bound(size_t coefficients, size_t h, double log2_failure, size_t* k) {
    return guarded([&] { *k = required_binboot_k_bound(coefficients, h, std::exp2((long double)log2_failure)).evalmod_k; });
}

// The AESWalsh15 modulus chain and bootstrapping DFT parameters with CoeffToSlot / SlotToCoeff
// plaintext plans but no bootstrapping keys (the EvalMod fit needs MPFR): the context builds
// the reference's own S2C and C2S plans and the rotation keys they need.  The chain is the
// preset's (36 | 61 | 42 42 | 38 x7 | 50 50); mult_depth absorbs the EvalMod levels so the
// depth check holds with the explicit chain.
void* ref_walsh15_plans_create(void) {
    RefCtx* out = nullptr;
    const int rc = guarded([&] {
        CKKSParamsConfig cfg = ckks_aes_params_detail::AESWalsh15Config();
        cfg.secure = false;
        cfg.bts_keys = false;
        cfg.s2c_ptxt = true;
        cfg.c2s_ptxt = true;
        cfg.aes_walsh_params.enabled = false;
        cfg.q_mult_bits.clear();
        cfg.q_bits = {36, 61, 42, 42, 38, 38, 38, 38, 38, 38, 38, 50, 50};
        cfg.mult_depth = 9;
        out = new RefCtx(CKKSParams(std::move(cfg)));
    });
    return rc == 0 ? out : nullptr;
}

// The same chain with bootstrapping keys (dense-to-sparse, sparse-to-dense) and the EvalMod
// polynomial of the reference's own MPFR fit (src/math/poly_approx.cpp:565).
void* ref_walsh15_bts_create(void) {
    RefCtx* out = nullptr;
    const int rc = guarded([&] {
        CKKSParamsConfig cfg = ckks_aes_params_detail::AESWalsh15Config();
        cfg.secure = false;
        cfg.bts_keys = true;
        cfg.s2c_ptxt = true;
        cfg.c2s_ptxt = true;
        cfg.aes_walsh_params.enabled = true;
        cfg.q_mult_bits.clear();
        cfg.q_bits = {36, 61, 42, 42, 38, 38, 38, 38, 38, 38, 38, 50, 50};
        // the mask-packed S-box's segment rotations (+-512 k) as the AES parameter set adds them
        for (int64_t k = 1; k <= 31; ++k) {
            cfg.rotate_values.push_back(512 * k);
            cfg.rotate_values.push_back(-512 * k);
        }
        cfg.mult_depth = 2;  // the EvalMod, S2C and C2S levels are the bootstrap depths here
        out = new RefCtx(CKKSParams(std::move(cfg)));
    });
    return rc == 0 ? out : nullptr;
}

// ckks_modraise_inplace (src/ckks/operations/bootstrap/ckks_modraise.cpp:103) on a level-0
// sparse-secret ciphertext: limb 0 of b and a in, target_level+1 limbs out (in place).
int ref_modraise(void* h, size_t target_level, uint64_t* b, uint64_t* a) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        CKKSCiphertext ct(N, copy_in(a, N), copy_in(b, N), 1.0L, 0, CKKSSecretOwner::BootstrapSparse);
        ckks_modraise_inplace(c, ct, target_level);
        copy_out(ct.getB(), b);
        copy_out(ct.getA(), a);
    });
}

// ckks_key_switch_dense_to_sparse_inplace (ckks_keyswitch.cpp:1844) on a level-0 ciphertext.
int ref_dense_to_sparse(void* h, uint64_t* b, uint64_t* a) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        CKKSCiphertext ct(N, copy_in(a, N), copy_in(b, N), 1.0L, 0, CKKSSecretOwner::Dense);
        ckks_key_switch_dense_to_sparse_inplace(c, ct);
        copy_out(ct.getB(), b);
        copy_out(ct.getA(), a);
    });
}

// ckks_key_switch_sparse_to_dense_inplace (ckks_keyswitch.cpp:1858) at `level`.
int ref_sparse_to_dense(void* h, size_t level, uint64_t* b, uint64_t* a) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t n = (level + 1) * c.getParams().getN();
        CKKSCiphertext ct(c.getParams().getN(), copy_in(a, n), copy_in(b, n), 1.0L, level,
                          CKKSSecretOwner::BootstrapSparse);
        ckks_key_switch_sparse_to_dense_inplace(c, ct);
        copy_out(ct.getB(), b);
        copy_out(ct.getA(), a);
    });
}

// ckks_evalchebyshev_preconditioned (src/ckks/operations/evalpoly/ckks_evalpoly.cpp:1221-1256)
// on a ciphertext at `level` with scale `scale`; target_scale 0 keeps the input scale.  The
// output (b, a) has (*out_level + 1) * N residues; *out_scale is its scale.
int ref_evalchebyshev(void* h, size_t level, double scale, const double* coeffs, size_t ncoeffs,
                      double target_scale, const uint64_t* b, const uint64_t* a, size_t* out_level,
                      double* out_scale, uint64_t* out_b, uint64_t* out_a) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        CKKSCiphertext ct(N, copy_in(a, n), copy_in(b, n), (long double)scale, level);
        CKKSEvalPolyOptions opt;
        opt.target_scale = target_scale;
        CKKSCiphertext out = ckks_evalchebyshev_preconditioned(c, ct, std::span<const double>(coeffs, ncoeffs), opt);
        if (out.getNumPolys() != 2) throw std::runtime_error("ref_evalchebyshev: unexpected polynomial count");
        *out_level = out.getLevel();
        *out_scale = (double)out.getScale();
        copy_out(out.getB(), out_b);
        copy_out(out.getA(), out_a);
    });
}

// The context's default scale and the EvalMod polynomial it built (Chebyshev coefficients on
// [interval_min, interval_max]).
int ref_ctx_scale(void* h, double* scale) {
    return guarded([&] { *scale = (double)static_cast<RefCtx*>(h)->ctx.getParams().getScale(); });
}

// Parameters the EvalMod bootstrap reads (ckks_bootstrap_evalmod_inplace.cpp:246-416) and the
// size of the EvalMod polynomial the context built.
int ref_bts_info(void* h, size_t* s2c_depth, size_t* depth, size_t* evalmod_log_scale, size_t* double_angle,
                 size_t* active_slots, size_t* slots, double* scale, size_t* ncoeffs) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const auto& p = c.getParams();
        *s2c_depth = p.getBootstrapS2CDepth();
        *depth = p.getDepth();
        *evalmod_log_scale = ckks_evalmod_log_scale_bits(p);
        *double_angle = p.getBootstrapEvalModDoubleAngle();
        *active_slots = p.getBootstrapActiveSlotCount();
        *slots = p.getSlots();
        *scale = (double)p.getScale();
        *ncoeffs = c.getEvalModPolynomial().chebyshev_coeffs.size();
    });
}

int ref_bts_evalmod_coeffs(void* h, double* out) {
    return guarded([&] {
        const auto& v = static_cast<RefCtx*>(h)->ctx.getEvalModPolynomial().chebyshev_coeffs;
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    });
}

// ckks_batch_bootstrap_evalmod_from_complex_packed (ckks_bootstrap_evalmod_inplace.cpp:416-434)
// on a packed ciphertext at level `level` with scale `scale`: both outputs (b, a) with
// (*out_level + 1) * N residues each.
int ref_bootstrap_evalmod(void* h, size_t level, double scale, const uint64_t* b, const uint64_t* a,
                          uint64_t* out0_b, uint64_t* out0_a, uint64_t* out1_b, uint64_t* out1_a, size_t* out_level,
                          double* out_scale) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        CKKSCiphertext ct(N, copy_in(a, n), copy_in(b, n), (long double)scale, level);
        auto outs = ckks_batch_bootstrap_evalmod_from_complex_packed(c, std::move(ct));
        if (outs.first.getLevel() != outs.second.getLevel()) throw std::runtime_error("ref_bootstrap_evalmod: level mismatch");
        *out_level = outs.first.getLevel();
        *out_scale = (double)outs.first.getScale();
        copy_out(outs.first.getB(), out0_b);
        copy_out(outs.first.getA(), out0_a);
        copy_out(outs.second.getB(), out1_b);
        copy_out(outs.second.getA(), out1_a);
    });
}

// ckks_encode of a constant slot vector (coefficient form, eval = false): the plaintext's
// (level+1)*N residues and its Montgomery flag.
int ref_encode_constant(void* h, double re, double im, double scale, size_t level, uint64_t* out, int* montgomery) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        MyVector<Complex> slots(c.getParams().getSlots(), Complex(re, im));
        CKKSEncoding pt = ckks_encode(c, slots, scale, level, /*eval=*/false);
        copy_out(pt.getPlaintext(), out);
        *montgomery = pt.isMontgomeryForm() ? 1 : 0;
    });
}

// ckks_walsh_sbox_complex_blocks_mask_packed (src/ckks/operations/circuits/ckks_walsh_sbox.cpp:
// 1286-1323) on 8 bit ciphertexts at `level` with scale `scale`: in holds, per bit, b then a
// ((level+1)*N words each); out receives, per output bit, b then a with
// (out_levels[bit]+1)*N words each, packed back to back.
int ref_walsh_sbox(void* h, size_t block_count, size_t level, double scale, const uint64_t* in, uint64_t* out,
                   size_t* out_levels, double* out_scales) {
    return guarded([&] {
        auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        MyVector<CKKSCiphertext> bits;
        for (size_t k = 0; k < 8; ++k)
            bits.emplace_back(N, copy_in(in + (2 * k + 1) * n, n), copy_in(in + 2 * k * n, n), (long double)scale,
                              level);
        CKKSWalshSboxScratch scratch;
        auto res = ckks_walsh_sbox_complex_blocks_mask_packed(c, std::move(bits), block_count, scratch);
        if (res.size() != 8) throw std::runtime_error("ref_walsh_sbox: expected 8 output bits");
        size_t off = 0;
        for (size_t k = 0; k < 8; ++k) {
            if (res[k].getNumPolys() != 2) throw std::runtime_error("ref_walsh_sbox: unexpected polynomial count");
            out_levels[k] = res[k].getLevel();
            out_scales[k] = (double)res[k].getScale();
            copy_out(res[k].getB(), out + off);
            off += res[k].getB().size();
            copy_out(res[k].getA(), out + off);
            off += res[k].getA().size();
        }
    });
}

// ---- XBOOT S-box (src/ckks/operations/circuits/aes/ckks_aes_ctr.cpp:48-336).  The reference
// keeps it in an anonymous namespace of that file, so the harness restates its steps on the
// reference's public operations: exact-add alignment (:48-158), multiply + relinearize + rescale
// at a fixed scale (:160-183), the layered monomial tree (:185-256), the Moebius coefficients of
// the S-box bits (:258-278) and the per-bit integer combination (:280-336).
namespace xboot_ref {

using Byte = MyVector<CKKSCiphertext>;

bool close(long double l, long double r) {
    if (!std::isfinite(l) || !std::isfinite(r)) return false;
    return std::abs(l - r) <= 0x1p-45L * std::max<long double>({1.0L, std::abs(l), std::abs(r)});
}

bool is_zero(const CKKSCiphertext& ct) {
    for (size_t k = 0; k < ct.getNumPolys(); ++k)
        for (uint64_t v : ct.getPoly(k))
            if (v) return false;
    return true;
}

CKKSCiphertext align(const CKKSContext& c, CKKSCiphertext ct, size_t level, long double scale, size_t polys) {
    ckks_drop_to_level_inplace(ct, level);
    while (ct.getNumPolys() < polys) ct.addPoly(MyVector<uint64_t>(ct.getN() * (ct.getLevel() + 1), 0));
    if (close(ct.getScale(), scale) || is_zero(ct)) {
        ct.setScale(scale);
        return ct;
    }
    if (ct.getScale() > scale) throw std::invalid_argument("xboot: cannot scale down");
    const long double k = std::round(scale / ct.getScale());
    if (k != 1.0L) ckks_mul_inplace(c, ct, (int64_t)k);
    ct.setScale(scale);
    return ct;
}

void add_term(const CKKSContext& c, CKKSCiphertext& acc, CKKSCiphertext term) {
    const size_t level = std::min(acc.getLevel(), term.getLevel());
    const long double scale = std::max(acc.getScale(), term.getScale());
    const size_t polys = std::max(acc.getNumPolys(), term.getNumPolys());
    acc = align(c, std::move(acc), level, scale, polys);
    term = align(c, std::move(term), level, scale, polys);
    ckks_add_inplace(c, acc, term);
}

CKKSCiphertext mul_relin_rescale(const CKKSContext& c, const CKKSCiphertext& l, const CKKSCiphertext& r,
                                 long double scale) {
    const size_t level = std::min(l.getLevel(), r.getLevel());
    auto out = l.clone();
    ckks_drop_to_level_inplace(out, level);
    out.setScale(scale);
    auto rr = r.clone();
    ckks_drop_to_level_inplace(rr, level);
    rr.setScale(scale);
    ckks_mul_inplace(c, out, rr);
    ckks_relin_hybrid_inplace(c, out);
    ckks_rescale(c, out);
    out.setScale(scale);
    return out;
}

struct Mono {
    size_t mask;
    CKKSCiphertext value;
};

std::vector<Mono> layered(const CKKSContext& c, const Byte& in, size_t begin, size_t end, long double scale) {
    const size_t n = end - begin;
    std::vector<Mono> out;
    if (n == 1) {
        auto v = in[begin].clone();
        v.setScale(scale);
        out.push_back({size_t{1} << begin, std::move(v)});
        return out;
    }
    if (n == 2) {
        auto l = in[begin].clone();
        l.setScale(scale);
        auto r = in[begin + 1].clone();
        r.setScale(scale);
        auto p = mul_relin_rescale(c, l, r, scale);
        out.push_back({size_t{1} << begin, std::move(l)});
        out.push_back({size_t{1} << (begin + 1), std::move(r)});
        out.push_back({(size_t{1} << begin) | (size_t{1} << (begin + 1)), std::move(p)});
        return out;
    }
    const size_t mid = begin + n / 2;
    auto left = layered(c, in, begin, mid, scale);
    auto right = layered(c, in, mid, end, scale);
    for (const auto& a : left)
        for (const auto& b : right) out.push_back({a.mask | b.mask, mul_relin_rescale(c, a.value, b.value, scale)});
    for (auto& a : left) out.push_back(std::move(a));
    for (auto& b : right) out.push_back(std::move(b));
    return out;
}

std::array<std::array<int64_t, 256>, 8> coefficients() {
    std::array<std::array<int64_t, 256>, 8> out{};
    for (size_t bit = 0; bit < 8; ++bit) {
        for (size_t x = 0; x < 256; ++x) out[bit][x] = (int64_t)((kAesSboxTable[x] >> bit) & 1U);
        for (size_t v = 0; v < 8; ++v)
            for (size_t m = 0; m < 256; ++m)
                if (m & (size_t{1} << v)) out[bit][m] -= out[bit][m ^ (size_t{1} << v)];
    }
    return out;
}

Byte sbox(const CKKSContext& c, const Byte& in) {
    const long double scale = in.front().getScale();
    std::vector<std::optional<CKKSCiphertext>> mono(256);
    for (auto& m : layered(c, in, 0, 8, scale)) mono[m.mask] = std::move(m.value);
    const auto cf = coefficients();
    Byte out;
    for (size_t bit = 0; bit < 8; ++bit) {
        std::optional<CKKSCiphertext> acc;
        if (cf[bit][0] != 0) {
            acc = in.front().clone();
            ckks_mul_inplace(c, *acc, int64_t{0});
            ckks_add_integer_constant_inplace(c, *acc, cf[bit][0]);
        }
        for (size_t m = 1; m < 256; ++m) {
            if (cf[bit][m] == 0) continue;
            auto t = mono[m]->clone();
            ckks_mul_inplace(c, t, cf[bit][m]);
            if (acc)
                add_term(c, *acc, std::move(t));
            else
                acc = std::move(t);
        }
        out.emplace_back(std::move(*acc));
    }
    return out;
}

// make_batched_initial_counter_state (ckks_aes_ctr.cpp:576-683), restated on the reference's
// public operations (the original is file-internal): the round-0 key bits XOR the counter bit
// planes, one level down.
MyVector<CKKSCiphertext> initial_state(const CKKSContext& c, const MyVector<CKKSCiphertext>& keys,
                                       const std::vector<std::array<uint8_t, 16>>& blocks) {
    const auto& params = c.getParams();
    const size_t logical = params.hasBootstrapParams() ? params.getBootstrapActiveSlotCount() : params.getSlots();
    if (blocks.empty() || blocks.size() > logical) throw std::invalid_argument("xboot: invalid counter count");
    MyVector<CKKSCiphertext> state;
    for (size_t bit = 0; bit < 128; ++bit) {
        bool saw_zero = blocks.size() < logical, saw_one = false;
        for (const auto& b : blocks) {
            const bool v = ((b[bit / 8] >> (bit % 8)) & 1u) != 0;
            saw_zero = saw_zero || !v;
            saw_one = saw_one || v;
        }
        auto out = keys[bit].clone();
        if (out.getLevel() == 0) throw std::invalid_argument("xboot: exact public XOR requires one level");
        const size_t in_level = out.getLevel();
        if (!saw_one || !saw_zero) {
            ckks_drop_to_level_inplace(out, in_level - 1);
            if (saw_one) {
                ckks_mul_inplace(c, out, int64_t{-1});
                ckks_add_integer_constant_inplace(c, out, int64_t{1});
            }
            state.emplace_back(std::move(out));
            continue;
        }
        MyVector<Complex> signs(params.getSlots()), bits(params.getSlots());
        for (size_t s = 0; s < params.getSlots(); ++s) {
            const size_t ls = s % logical;
            const uint8_t v = ls < blocks.size() ? (uint8_t)((blocks[ls][bit / 8] >> (bit % 8)) & 1u) : 0;
            bits[s] = Complex((double)v, 0.0);
            signs[s] = Complex(v == 0 ? 1.0 : -1.0, 0.0);
        }
        auto sel = ckks_encode(c, signs, (double)params.getModuli()[in_level], in_level, true);
        ckks_mul_inplace(c, out, sel);
        ckks_rescale(c, out);
        auto pt = ckks_encode(c, bits, out.getLevel(), true);
        ckks_add_inplace(c, out, pt);
        state.emplace_back(std::move(out));
    }
    return state;
}

// shift_rows_inplace, fmix_columns_inplace (when `mix`) and add_round_key_lazy_inplace
// (ckks_aes_ctr.cpp:365-472, 511-554), restated with the same clones and in-place additions.
MyVector<CKKSCiphertext> linear_layer(const CKKSContext& c, MyVector<CKKSCiphertext> state,
                                      const MyVector<CKKSCiphertext>& round_keys, bool mix) {
    MyVector<CKKSCiphertext> sh;
    for (size_t col = 0; col < 4; ++col)
        for (size_t row = 0; row < 4; ++row) {
            const size_t src = 4 * ((col + row) % 4) + row;
            for (size_t bit = 0; bit < 8; ++bit) sh.emplace_back(std::move(state[src * 8 + bit]));
        }
    auto add = [&](const CKKSCiphertext& l, const CKKSCiphertext& r) {
        auto o = l.clone();
        ckks_add_inplace(c, o, r);
        return o;
    };
    MyVector<CKKSCiphertext> out;
    if (!mix) {
        out = std::move(sh);
    } else {
        std::array<Byte, 16> bytes;
        auto byte = [&](size_t b) {
            Byte o;
            for (size_t k = 0; k < 8; ++k) o.emplace_back(sh[b * 8 + k].clone());
            return o;
        };
        auto mixb = [&](const Byte& b0, const Byte& b1, const Byte& b2, const Byte& b3) {
            Byte s01;
            for (size_t k = 0; k < 8; ++k) s01.emplace_back(add(b0[k], b1[k]));
            Byte d;
            d.emplace_back(s01[7].clone());
            d.emplace_back(add(s01[0], s01[7]));
            d.emplace_back(s01[1].clone());
            d.emplace_back(add(s01[2], s01[7]));
            d.emplace_back(add(s01[3], s01[7]));
            d.emplace_back(s01[4].clone());
            d.emplace_back(s01[5].clone());
            d.emplace_back(s01[6].clone());
            for (const Byte* t : {&b1, &b2, &b3})
                for (size_t k = 0; k < 8; ++k) ckks_add_inplace(c, d[k], (*t)[k]);
            return d;
        };
        for (size_t col = 0; col < 4; ++col) {
            const Byte b0 = byte(4 * col), b1 = byte(4 * col + 1), b2 = byte(4 * col + 2), b3 = byte(4 * col + 3);
            bytes[4 * col] = mixb(b0, b1, b2, b3);
            bytes[4 * col + 1] = mixb(b1, b2, b3, b0);
            bytes[4 * col + 2] = mixb(b2, b3, b0, b1);
            bytes[4 * col + 3] = mixb(b3, b0, b1, b2);
        }
        for (auto& b : bytes)
            for (auto& x : b) out.emplace_back(std::move(x));
    }
    for (size_t bit = 0; bit < 128; ++bit) ckks_add_inplace(c, out[bit], round_keys[bit]);
    return out;
}

}  // namespace xboot_ref

// The XBOOT chain at N = 2^15 (AESXBoot15Config: 17 Q limbs of 36..38 bits, 5 P limbs, dnum 5,
// h 256) without bootstrapping, so only the relinearisation key is generated.
void* ref_xboot15_create(void) {
    RefCtx* out = nullptr;
    const int rc = guarded([&] {
        CKKSParamsConfig cfg = ckks_aes_params_detail::AESXBoot15Config();
        cfg.secure = false;
        cfg.bts_keys = false;
        cfg.bootstrap_params.reset();
        cfg.q_mult_bits.clear();
        cfg.mult_depth = cfg.q_bits.size() - 1;
        out = new RefCtx(CKKSParams(std::move(cfg)));
    });
    return rc == 0 ? out : nullptr;
}

// The XBOOT S-box on 8 bit ciphertexts at `level` and `scale` (in: [bit][b, a][level+1][N]);
// out: 8 x (b, a) at their levels, packed one after another.
int ref_xboot_sbox(void* h, size_t level, double scale, const uint64_t* in, uint64_t* out, size_t* out_levels,
                   double* out_scales) {
    return guarded([&] {
        auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        xboot_ref::Byte bits;
        for (size_t k = 0; k < 8; ++k)
            bits.emplace_back(N, copy_in(in + (2 * k + 1) * n, n), copy_in(in + 2 * k * n, n), (long double)scale,
                              level);
        auto res = xboot_ref::sbox(c, bits);
        size_t off = 0;
        for (size_t k = 0; k < 8; ++k) {
            out_levels[k] = res[k].getLevel();
            out_scales[k] = (double)res[k].getScale();
            copy_out(res[k].getB(), out + off);
            off += res[k].getB().size();
            copy_out(res[k].getA(), out + off);
            off += res[k].getA().size();
        }
    });
}

int ref_xboot_sbox_coefficients(int64_t* out) {
    return guarded([&] {
        const auto cf = xboot_ref::coefficients();
        for (size_t b = 0; b < 8; ++b)
            for (size_t m = 0; m < 256; ++m) out[b * 256 + m] = cf[b][m];
    });
}

// The XBOOT N = 2^15 parameter set as the reference defines it (AESXBoot15Config, or
// AESXBoot15Sparse1024Config when `sparse`, src/ckks/parameters/ckks_aes_params.hpp:179-209),
// bootstrapping keys and the reference's MPFR EvalMod fit included.
void* ref_xboot15_bts_create(int sparse) {
    RefCtx* out = nullptr;
    const int rc = guarded([&] {
        CKKSParamsConfig cfg = sparse ? ckks_aes_params_detail::AESXBoot15Sparse1024Config()
                                      : ckks_aes_params_detail::AESXBoot15Config();
        out = new RefCtx(CKKSParams(std::move(cfg)));
    });
    return rc == 0 ? out : nullptr;
}

// The secure XBOOT N = 2^14 parameter set (AESXBoot14SecureConfig, or
// AESXBoot14SecureSparse1024Config when `sparse`, ckks_aes_params.hpp:133-154) with its
// bootstrapping keys and the reference's MPFR EvalMod fit.
void* ref_xboot14_bts_create(int sparse) {
    RefCtx* out = nullptr;
    const int rc = guarded([&] {
        CKKSParamsConfig cfg = sparse ? ckks_aes_params_detail::AESXBoot14SecureSparse1024Config()
                                      : ckks_aes_params_detail::AESXBoot14SecureConfig();
        out = new RefCtx(CKKSParams(std::move(cfg)));
    });
    return rc == 0 ? out : nullptr;
}

// ckks_batch_bootstrap_evalmod_inplace (ckks_bootstrap_evalmod_inplace.cpp:393-414) on the
// pair (ct0, ct1) at `level` with scales scale0 / scale1: both results (b, a) with
// (*out_level + 1) * N residues each and their common scale.
int ref_bootstrap_pair(void* h, size_t level, double scale0, double scale1, const uint64_t* b0, const uint64_t* a0,
                       const uint64_t* b1, const uint64_t* a1, uint64_t* out0_b, uint64_t* out0_a, uint64_t* out1_b,
                       uint64_t* out1_a, size_t* out_level, double* out_scale) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        CKKSCiphertext ct0(N, copy_in(a0, n), copy_in(b0, n), (long double)scale0, level);
        CKKSCiphertext ct1(N, copy_in(a1, n), copy_in(b1, n), (long double)scale1, level);
        ckks_batch_bootstrap_evalmod_inplace(c, ct0, ct1);
        if (ct0.getLevel() != ct1.getLevel()) throw std::runtime_error("ref_bootstrap_pair: level mismatch");
        *out_level = ct0.getLevel();
        *out_scale = (double)ct0.getScale();
        copy_out(ct0.getB(), out0_b);
        copy_out(ct0.getA(), out0_a);
        copy_out(ct1.getB(), out1_b);
        copy_out(ct1.getA(), out1_a);
    });
}

// The XBOOT initial state (xboot_ref::initial_state) from 128 round-0 key bits at `key_level`
// (in: [bit][b, a][key_level + 1][N]) and `blocks` counter blocks: out [bit][b, a][level + 1][N]
// with the common output level and per-bit scales.
int ref_xboot_initial_state(void* h, const uint64_t* keys, const double* key_scales, size_t key_level,
                            const uint8_t* counters, size_t blocks, uint64_t* out, size_t* out_level,
                            double* out_scales) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (key_level + 1) * N;
        MyVector<CKKSCiphertext> kb;
        for (size_t k = 0; k < 128; ++k)
            kb.emplace_back(N, copy_in(keys + (2 * k + 1) * n, n), copy_in(keys + 2 * k * n, n),
                            (long double)key_scales[k], key_level);
        std::vector<std::array<uint8_t, 16>> bl(blocks);
        for (size_t b = 0; b < blocks; ++b) std::memcpy(bl[b].data(), counters + 16 * b, 16);
        auto st = xboot_ref::initial_state(c, kb, bl);
        *out_level = st[0].getLevel();
        const size_t m = (*out_level + 1) * N;
        for (size_t k = 0; k < 128; ++k) {
            if (st[k].getLevel() != *out_level) throw std::runtime_error("ref_xboot_initial_state: level mismatch");
            copy_out(st[k].getB(), out + 2 * k * m);
            copy_out(st[k].getA(), out + (2 * k + 1) * m);
            out_scales[k] = (double)st[k].getScale();
        }
    });
}

// The XBOOT round's linear layers (xboot_ref::linear_layer) on 128 state bits at `level` with
// scales in_scales (in: [bit][b, a][level + 1][N]) and 128 round-key bits at key_level (keys:
// [bit][b, a][key_level + 1][N]): out [bit][b, a][level + 1][N] and the output scales.
int ref_xboot_linear(void* h, const uint64_t* in, const double* in_scales, size_t level, const uint64_t* keys,
                     size_t key_level, int mix, uint64_t* out, double* out_scales) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N, kn = (key_level + 1) * N;
        MyVector<CKKSCiphertext> st, kb;
        for (size_t k = 0; k < 128; ++k) {
            st.emplace_back(N, copy_in(in + (2 * k + 1) * n, n), copy_in(in + 2 * k * n, n),
                            (long double)in_scales[k], level);
            // the reference adds a key bit above the state level limb by limb over the state's limbs
            CKKSCiphertext key(N, copy_in(keys + (2 * k + 1) * kn, kn), copy_in(keys + 2 * k * kn, kn), 1.0L,
                               key_level);
            ckks_drop_to_level_inplace(key, level);
            kb.emplace_back(std::move(key));
        }
        auto o = xboot_ref::linear_layer(c, std::move(st), kb, mix != 0);
        for (size_t k = 0; k < 128; ++k) {
            copy_out(o[k].getB(), out + 2 * k * n);
            copy_out(o[k].getA(), out + (2 * k + 1) * n);
            out_scales[k] = (double)o[k].getScale();
        }
    });
}

// ckks_aes128_encrypt_expanded_round_key_bits (ckks_aes_ctr.cpp:687-725): the 1408 key-bit
// ciphertexts, bit k as b then a with (levels[k] + 1) * N residues each, back to back.
int ref_xboot_key_bits(void* h, const uint8_t* expanded_key, size_t first_round_key_level, uint64_t* out,
                       double* scales, size_t* levels) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        std::array<uint8_t, 176> ek{};
        std::memcpy(ek.data(), expanded_key, 176);
        auto bits = ckks_aes128_encrypt_expanded_round_key_bits(c, ek, first_round_key_level);
        size_t off = 0;
        for (size_t k = 0; k < bits.size(); ++k) {
            copy_out(bits[k].getB(), out + off);
            off += bits[k].getB().size();
            copy_out(bits[k].getA(), out + off);
            off += bits[k].getA().size();
            scales[k] = (double)bits[k].getScale();
            levels[k] = bits[k].getLevel();
        }
    });
}

// Timing sample of the reference's SubBytes layer: `instances` independent mask-packed Walsh
// S-box calls on the same 8 input bits, run as sub_bytes_walsh_complex_blocks_mask_packed runs
// its 16 byte positions (src/ckks/operations/circuits/aes/ckks_aes_ctr_walsh_sbox.cpp:659-706:
// one OpenMP dynamic-schedule loop over bytes, one scratch per byte) on `threads` threads.
// Returns the wall time of the loop in *seconds; outputs are discarded.
int ref_walsh_sbox_layer(void* h, size_t block_count, size_t level, double scale, const uint64_t* in,
                         size_t instances, int threads, double* seconds) {
    return guarded([&] {
        auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        std::vector<MyVector<CKKSCiphertext>> inputs(instances);
        for (auto& bits : inputs)
            for (size_t k = 0; k < 8; ++k)
                bits.emplace_back(N, copy_in(in + (2 * k + 1) * n, n), copy_in(in + 2 * k * n, n),
                                  (long double)scale, level);
        std::vector<CKKSWalshSboxScratch> scratch(instances);
        std::exception_ptr first;
        if (threads > 0) omp_set_num_threads(threads);
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic)
        for (std::ptrdiff_t i = 0; i < (std::ptrdiff_t)instances; ++i) {
            try {
                auto res = ckks_walsh_sbox_complex_blocks_mask_packed(c, std::move(inputs[(size_t)i]), block_count,
                                                                      scratch[(size_t)i]);
                if (res.size() != 8) throw std::runtime_error("ref_walsh_sbox_layer: expected 8 output bits");
            } catch (...) {
#pragma omp critical
                if (!first) first = std::current_exception();
            }
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (first) std::rethrow_exception(first);
    });
}

// Timing samples of the XBOOT AES's two layers as the reference runs them: `instances` XBOOT
// S-boxes (sub_bytes_inplace, ckks_aes_ctr.cpp:474-509: OpenMP dynamic over byte positions; the
// S-box as restated in xboot_ref) on copies of the same 8 bits, or `pairs` pair bootstraps
// (xboot_state_inplace, :556-574: OpenMP dynamic over pairs) on copies of one pair, on `threads`
// threads.  *seconds = wall time of the loop; outputs are discarded.
int ref_xboot_sbox_layer(void* h, size_t level, double scale, const uint64_t* in, size_t instances, int threads,
                         double* seconds) {
    return guarded([&] {
        auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        std::vector<xboot_ref::Byte> inputs(instances);
        for (auto& bits : inputs)
            for (size_t k = 0; k < 8; ++k)
                bits.emplace_back(N, copy_in(in + (2 * k + 1) * n, n), copy_in(in + 2 * k * n, n),
                                  (long double)scale, level);
        std::exception_ptr first;
        if (threads > 0) omp_set_num_threads(threads);
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic)
        for (std::ptrdiff_t i = 0; i < (std::ptrdiff_t)instances; ++i) {
            try {
                auto res = xboot_ref::sbox(c, inputs[(size_t)i]);
                if (res.size() != 8) throw std::runtime_error("ref_xboot_sbox_layer: expected 8 output bits");
            } catch (...) {
#pragma omp critical
                if (!first) first = std::current_exception();
            }
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (first) std::rethrow_exception(first);
    });
}

int ref_bootstrap_pair_layer(void* h, size_t level, double scale, const uint64_t* b0, const uint64_t* a0,
                             const uint64_t* b1, const uint64_t* a1, size_t pairs, int threads, double* seconds) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        std::vector<CKKSCiphertext> x0, x1;
        for (size_t i = 0; i < pairs; ++i) {
            x0.emplace_back(N, copy_in(a0, n), copy_in(b0, n), (long double)scale, level);
            x1.emplace_back(N, copy_in(a1, n), copy_in(b1, n), (long double)scale, level);
        }
        std::exception_ptr first;
        if (threads > 0) omp_set_num_threads(threads);
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic)
        for (std::ptrdiff_t i = 0; i < (std::ptrdiff_t)pairs; ++i) {
            try {
                ckks_batch_bootstrap_evalmod_inplace(c, x0[(size_t)i], x1[(size_t)i]);
            } catch (...) {
#pragma omp critical
                if (!first) first = std::current_exception();
            }
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (first) std::rethrow_exception(first);
    });
}

// ckks_encode (coefficient form, eval = false) of N/2 slot values re[i] + i im[i].
int ref_encode(void* h, const double* re, const double* im, double scale, size_t level, uint64_t* out) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t slots = c.getParams().getSlots();
        MyVector<Complex> v(slots);
        for (size_t i = 0; i < slots; ++i) v[i] = Complex(re[i], im[i]);
        CKKSEncoding pt = ckks_encode(c, v, scale, level, /*eval=*/false);
        if (pt.isMontgomeryForm()) throw std::runtime_error("ref_encode: unexpected Montgomery plaintext");
        copy_out(pt.getPlaintext(), out);
    });
}

// The context's FFT twiddles (interleaved re, im) and one fft_dif of `data` (in place).
int ref_fft_probe(void* h, double* twiddles, double* data) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const auto& tw = c.getTwiddleFft();
        const size_t N = c.getParams().getN();
        for (size_t i = 0; i < N; ++i) {
            twiddles[2 * i] = tw[i].real();
            twiddles[2 * i + 1] = tw[i].imag();
        }
        MyVector<Complex> v(N);
        for (size_t i = 0; i < N; ++i) v[i] = Complex(data[2 * i], data[2 * i + 1]);
        fft_dif(v, tw, N);
        for (size_t i = 0; i < N; ++i) {
            data[2 * i] = v[i].real();
            data[2 * i + 1] = v[i].imag();
        }
    });
}

// ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks (ckks_aes_ctr_walsh_sbox.cpp:
// 981-1035): the 1408 encrypted round-key bits, each (b, a) at *key_level, back to back, with
// their scales.
int ref_aes_key_bits(void* h, const uint8_t* expanded_key, size_t active_blocks, uint64_t* out, double* scales,
                     size_t* key_level) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        std::array<uint8_t, 176> ek{};
        std::memcpy(ek.data(), expanded_key, 176);
        auto bits = ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks(c, ek, active_blocks);
        size_t off = 0;
        for (size_t k = 0; k < bits.size(); ++k) {
            copy_out(bits[k].getB(), out + off);
            off += bits[k].getB().size();
            copy_out(bits[k].getA(), out + off);
            off += bits[k].getA().size();
            scales[k] = (double)bits[k].getScale();
        }
        *key_level = bits.front().getLevel();
    });
}

// ckks_aes_ctr_walsh_sbox_complex_blocks (ckks_aes_ctr_walsh_sbox.cpp:1037-1051) on the given
// key-bit ciphertexts; the 128 output bits (b, a) back to back with their levels and scales.
int ref_aes_ctr(void* h, const uint64_t* key, const double* key_scales, size_t key_level, const uint8_t* counters,
                const uint8_t* ciphertexts, size_t active_blocks, uint64_t* out, size_t* out_levels,
                double* out_scales) {
    return guarded([&] {
        auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (key_level + 1) * N;
        MyVector<CKKSCiphertext> kb;
        for (size_t k = 0; k < 1408; ++k)
            kb.emplace_back(N, copy_in(key + (2 * k + 1) * n, n), copy_in(key + 2 * k * n, n),
                            (long double)key_scales[k], key_level);
        std::vector<std::array<uint8_t, 16>> ctr(2 * active_blocks), ctx(2 * active_blocks);
        for (size_t i = 0; i < 2 * active_blocks; ++i) {
            std::memcpy(ctr[i].data(), counters + 16 * i, 16);
            std::memcpy(ctx[i].data(), ciphertexts + 16 * i, 16);
        }
        auto res = ckks_aes_ctr_walsh_sbox_complex_blocks(c, kb, std::span<const std::array<uint8_t, 16>>(ctr),
                                                          std::span<const std::array<uint8_t, 16>>(ctx));
        size_t off = 0;
        for (size_t k = 0; k < res.size(); ++k) {
            out_levels[k] = res[k].getLevel();
            out_scales[k] = (double)res[k].getScale();
            copy_out(res[k].getB(), out + off);
            off += res[k].getB().size();
            copy_out(res[k].getA(), out + off);
            off += res[k].getA().size();
        }
    });
}

// ckks_decrypt (slots) of a 2-polynomial ciphertext: re / im of the N/2 slots.
int ref_decrypt(void* h, size_t level, double scale, const uint64_t* b, const uint64_t* a, double* re, double* im) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        CKKSCiphertext ct(N, copy_in(a, n), copy_in(b, n), (long double)scale, level);
        auto v = ckks_decrypt(c, ct);
        for (size_t i = 0; i < v.size(); ++i) {
            re[i] = v[i].real();
            im[i] = v[i].imag();
        }
    });
}

// The SlotToCoeff plan the EvalMod bootstrap uses for an input whose scale is `ratio` times the
// parameter scale, built from the same literal as get_scaled_s2c_plan
// (ckks_bootstrap_evalmod_inplace.cpp:115-154); afterwards plan index 100 + ratio selects it.
int ref_build_scaled_s2c(void* h, uint64_t ratio) {
    return guarded([&] {
        auto* r = static_cast<RefCtx*>(h);
        const auto& p = r->ctx.getParams();
        const size_t d = p.getBootstrapS2CDepth();
        CKKSBootstrapDftMatrixLiteral lit;
        lit.type = CKKSBootstrapDftType::SlotsToCoeffs;
        lit.level = d;
        lit.baby_step_count = p.getBootstrapLinearTransformBsgsBabyStepCounts()[0];
        lit.log_bsgs_ratio = p.getBootstrapS2CLogBsgsRatio();
        lit.stage_count = d;
        lit.log_plaintext_scale_groups = p.getBootstrapS2CLogPlaintextScales();
        lit.merge_depths = p.getBootstrapS2CMergeDepths();
        lit.active_slots = p.getBootstrapActiveSlotCount();
        lit.transform_scale = (static_cast<double>(p.getModuli()[0]) * 0.5) / (p.getScale() * static_cast<double>(ratio));
        lit.plaintext_scale = static_cast<double>(p.getModuli()[d]);
        lit.rescale_after_each_stage = true;
        r->scaled_s2c.insert_or_assign(ratio, ckks_generate_bootstrap_dft_plan(r->ctx, lit));
    });
}

static const CKKSLinearTransformPlan& plan_of(void* h, int which) {
    auto* r = static_cast<RefCtx*>(h);
    if (which >= 100) return r->scaled_s2c.at((uint64_t)(which - 100));
    return which == 0 ? r->ctx.getEvalModS2CPlan() : r->ctx.getEvalModScaledC2SPlan();
}

int ref_plan_stage_count(void* h, int which, size_t* stages, int* use_qp) {
    return guarded([&] {
        const auto& p = plan_of(h, which);
        *stages = p.stages.size();
        *use_qp = p.use_qp_evaluator ? 1 : 0;
    });
}

// Stage metadata: number of diagonals, baby-step count, rescale flag, QP limb count of the
// stored plaintexts, Montgomery flag, logical slot count.
int ref_plan_stage_info(void* h, int which, size_t stage, size_t* nterms, size_t* baby, int* rescale,
                        size_t* qp_limbs, int* montgomery, size_t* slot_count) {
    return guarded([&] {
        const auto& st = plan_of(h, which).stages.at(stage);
        *nterms = st.diagonal_qp_plaintexts.size();
        *baby = st.baby_step_count;
        *rescale = st.rescale_after ? 1 : 0;
        *qp_limbs = st.qp_limb_count;
        *montgomery = st.diagonal_qp_plaintexts_montgomery ? 1 : 0;
        *slot_count = st.slot_count;
    });
}

// Diagonal indices of a stage (one per term) and all QP plaintexts [term][qp_limbs][N].
int ref_plan_stage_data(void* h, int which, size_t stage, uint64_t* indices, uint64_t* diagonals) {
    return guarded([&] {
        const auto& st = plan_of(h, which).stages.at(stage);
        for (size_t t = 0; t < st.diagonal_qp_plaintexts.size(); ++t) {
            indices[t] = st.diagonal_indices.empty() ? t : st.diagonal_indices[t];
            if (diagonals) {
                const auto& d = st.diagonal_qp_plaintexts[t];
                std::memcpy(diagonals + t * d.size(), d.data(), d.size() * sizeof(uint64_t));
            }
        }
    });
}

// One stage of the reference's linear transform on (b, a) at `level`, through its QP
// evaluator (ckks_apply_linear_transform_owned_stage_qp).  Outputs (out_level+1)*N residues.
int ref_lt_stage(void* h, int which, size_t stage, size_t level, const uint64_t* b, const uint64_t* a,
                 uint64_t* out_b, uint64_t* out_a, size_t* out_level) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        CKKSCiphertext ct(N, copy_in(a, n), copy_in(b, n), c.getParams().getScale(), level);
        const auto& st = plan_of(h, which).stages.at(stage);
        CKKSCiphertext r = ckks_apply_linear_transform_owned_stage_qp(c, ct, st);
        copy_out(r.getB(), out_b);
        copy_out(r.getA(), out_a);
        *out_level = r.getLevel();
    });
}

// Timing sample of a whole plan (every stage in order, each through
// ckks_apply_linear_transform_owned_stage_qp) on `count` copies of (b, a) at `level`, OpenMP
// dynamic over ciphertexts on `threads` threads, the way the reference runs independent
// ciphertexts side by side.  *seconds = wall time of the loop; outputs are discarded.
int ref_lt_plan_seconds(void* h, int which, size_t level, const uint64_t* b, const uint64_t* a, size_t count,
                        int threads, double* seconds) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t N = c.getParams().getN();
        const size_t n = (level + 1) * N;
        const auto& plan = plan_of(h, which);
        std::vector<CKKSCiphertext> cts;
        for (size_t i = 0; i < count; ++i)
            cts.emplace_back(N, copy_in(a, n), copy_in(b, n), c.getParams().getScale(), level);
        std::exception_ptr first;
        if (threads > 0) omp_set_num_threads(threads);
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic)
        for (std::ptrdiff_t i = 0; i < (std::ptrdiff_t)count; ++i) {
            try {
                CKKSCiphertext x = std::move(cts[(size_t)i]);
                for (const auto& st : plan.stages) x = ckks_apply_linear_transform_owned_stage_qp(c, x, st);
            } catch (...) {
#pragma omp critical
                if (!first) first = std::current_exception();
            }
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (first) std::rethrow_exception(first);
    });
}

// Every rotation value with a key in the context.
int ref_ctx_rotations(void* h, int64_t* out, size_t* n) {
    return guarded([&] {
        const auto& c = static_cast<RefCtx*>(h)->ctx;
        const size_t slots = c.getParams().getSlots();
        size_t k = 0;
        for (size_t r = 1; r < slots; ++r)
            if (c.hasRotationKey((int64_t)r)) {
                if (out) out[k] = (int64_t)r;
                ++k;
            }
        *n = k;
    });
}

}  // extern "C"
