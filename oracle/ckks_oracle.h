/* CPU oracle for the CKKS residue path: a plain-C restatement of the reference's algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (aes-walsh-ckks_b200/) never includes, links or
 * calls anything in this directory; tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it as the checker.
 *
 * Every function names the reference file:line it restates.  Modular steps that can leave a
 * residue outside [0,q) in the reference (Barrett products, lazy adds) are restated with the
 * same formulas, so outputs are compared bit for bit, not modulo q.
 *
 * Layout conventions (identical to the reference and the device library):
 *   polynomial  = limb-major u64 array, poly[limb * N + coeff], NTT (evaluation) domain with
 *                 bit-reversed coefficient order unless a function says otherwise;
 *   switch key  = [part][0 = a, 1 = b][limb: key_level+1 Q limbs, then K P limbs][N],
 *                 folded (Q limbs x P^-1, P limbs x (P/p_j)^-1) and in Montgomery form.
 */
#ifndef WALSH_CKKS_ORACLE_H
#define WALSH_CKKS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* --- scalar helpers exposed for unit tests --- */
uint64_t orc_barrett_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t mu_lo, uint64_t mu_hi);
void orc_barrett_const(uint64_t q, uint64_t* mu_lo, uint64_t* mu_hi);
uint64_t orc_shoup_const(uint64_t w, uint64_t q);

/* --- parameters --- */
int orc_find_primes(const uint64_t* p_bits, size_t np, const uint64_t* q_bits, size_t nq,
                    uint64_t N, uint64_t* p_out, uint64_t* q_out);
int orc_ntt_tables(uint64_t N, uint64_t q, uint64_t* fwd, uint64_t* fwd_shoup, uint64_t* inv,
                   uint64_t* inv_shoup_np1, uint64_t* n_inv);

/* --- context: moduli, twiddles, ModUp / ModDown / rescale constants --- */
orc_ctx* orc_ctx_create(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np,
                        size_t dnum);
void orc_ctx_destroy(orc_ctx* c);
size_t orc_ctx_alpha(const orc_ctx* c);

/* In-place NTT of `limbs` consecutive limbs of modulus list `which` (0 = Q, 1 = P) starting
 * at modulus index `first`; lazy forward output in [0,4q), otherwise canonical. */
void orc_ntt(const orc_ctx* c, uint64_t* poly, size_t first, size_t limbs, int which,
             int inverse, int lazy);

/* Hybrid key switch (reference ckks_hybrid_key_switch_inplace). key_term is read only. */
int orc_keyswitch(const orc_ctx* c, size_t level, const uint64_t* key_term, const uint64_t* key,
                  size_t key_level, uint64_t* b, uint64_t* a, int b_add, int a_add);

/* NTT-domain automorphism map for galois element g (reference build_ntt_automorphism_map). */
void orc_automorphism_map(uint64_t N, uint64_t g, uint64_t* dst_to_src);
uint64_t orc_rotation_galois(uint64_t N, int64_t rotation);

int orc_rotate(const orc_ctx* c, size_t level, uint64_t* b, uint64_t* a, const uint64_t* key,
               size_t key_level, int64_t rotation);
int orc_conjugate(const orc_ctx* c, size_t level, uint64_t* b, uint64_t* a, const uint64_t* key,
                  size_t key_level);
int orc_mul(const orc_ctx* c, size_t level, uint64_t* b1, uint64_t* a1, const uint64_t* b2,
            const uint64_t* a2, uint64_t* c2);
int orc_relin(const orc_ctx* c, size_t level, uint64_t* c0, uint64_t* c1, const uint64_t* c2,
              const uint64_t* key, size_t key_level);
int orc_rescale(const orc_ctx* c, size_t level, size_t npolys, uint64_t* polys);
int orc_hoisted_rotations(const orc_ctx* c, size_t level, const uint64_t* b, const uint64_t* a,
                          const uint64_t* const* keys, size_t key_level, const int64_t* rots,
                          size_t nrot, uint64_t* out);

/* One QP baby-step / giant-step linear-transform stage (reference
 * ckks_apply_linear_transform_owned_stage_qp); diags [term][level+1+K][N] Montgomery; keys:
 * nkeys rotation keys with their rotations.  (b, a) updated in place (level-1 when rescale). */
int orc_lt_stage(const orc_ctx* c, size_t level, size_t nterms, const uint64_t* indices, const uint64_t* diags,
                 size_t baby, size_t slots, int rescale, const uint64_t* const* keys, const int64_t* key_rots,
                 size_t nkeys, size_t key_level, uint64_t* b, uint64_t* a);

/* --- bootstrapping boundary steps --- */
/* ModRaise (reference ckks_modraise_inplace): limb 0 of b and a lifted to target_level+1 limbs
 * in place (buffers hold (target_level+1)*N words). */
int orc_modraise(const orc_ctx* c, size_t target_level, uint64_t* b, uint64_t* a);
/* Level-0 dense-to-sparse switch through q0 and p0 only (reference
 * ckks_q0p0_key_switch_level0_inplace); key [a: q0, p0][b: q0, p0] x N, folded Montgomery. */
int orc_q0p0_switch(const orc_ctx* c, const uint64_t* key, uint64_t* b, uint64_t* a);

/* --- seeded key material and encryption (test data generation) --- */
void orc_sample_ternary(uint64_t N, size_t hamming_weight, uint64_t seed, int8_t* out);
/* Switch key from secret `src` (squared when src_square, for relinearization) to secret
 * `dst`, both in coefficient form; noise sigma; seeded.  Writes dnum parts at the top level. */
int orc_keygen_switch(const orc_ctx* c, const int8_t* src, int src_square, const int8_t* dst,
                      double sigma, uint64_t seed, uint64_t* key_out);
/* Secret transformed by the coefficient automorphism X -> X^g. */
void orc_secret_automorphism(uint64_t N, uint64_t g, const int8_t* s, int8_t* out);
/* Uniform residues in [0, q_i) for `limbs` Q limbs. */
void orc_uniform_poly(const orc_ctx* c, size_t limbs, uint64_t seed, uint64_t* out);
/* Symmetric encryption of a plaintext given in NTT form: b = -a s + m + e. */
int orc_encrypt(const orc_ctx* c, size_t level, const uint64_t* m_ntt, const int8_t* s,
                double sigma, uint64_t seed, uint64_t* b, uint64_t* a);
/* <ct, s> for a 2-polynomial ciphertext, returned in coefficient form, centered, as doubles of
 * the first limb only when level == 0 or combined by CRT when level >= 1 (first two limbs). */
int orc_decrypt_coeffs(const orc_ctx* c, size_t level, const uint64_t* b, const uint64_t* a,
                       const int8_t* s, double* out);

/* --- CPU baseline: the batched-ops workload (mul, relin, rescale, rotate) --- */
int orc_batched_ops(const orc_ctx* c, size_t count, const size_t* levels, uint64_t* x_b,
                    uint64_t* x_a, const uint64_t* y_b, const uint64_t* y_a,
                    const uint64_t* relin_key, const uint64_t* const* rot_keys,
                    const int64_t* rots, size_t key_level, size_t stride, int threads);

#ifdef __cplusplus
}
#endif
#endif
