/* walsh_gpu.h -- C ABI of the B200 CKKS residue engine (libwalshgpu.so).
 *
 * The engine replaces the CPU residue path of TrustworthyComputing/aes-walsh-ckks.  Every
 * entry point below names the reference interface it stands in for (path:line inside that
 * project).  Conventions shared by all calls:
 *
 *   - Polynomials are limb-major arrays of uint64 residues in DEVICE memory, limb l of a
 *     polynomial at poly + l*N, in the evaluation (NTT, bit-reversed) domain, exactly the
 *     reference's CKKSCiphertext poly layout (src/ckks/ciphertext/ckks_ciphertext.hpp:18-74).
 *     A ciphertext at level l has (l+1) Q limbs per polynomial; "b" is polynomial 0 and "a"
 *     polynomial 1 (src/ckks/ciphertext/ckks_ciphertext.cpp:20).
 *   - Switching keys are given in HOST memory in the layout
 *     [part][0 = a, 1 = b][key_level+1 Q limbs then K P limbs][N], folded and in Montgomery
 *     form as the reference stores them (hybrid_key_folding.hpp:50-77,
 *     hybrid_key_montgomery.hpp:12-36 under src/ckks/context/).
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls enqueue work and
 *     return; results are ready when the stream is synchronised.
 *   - Return 0 on success or a negative WG_ERR_* code; wg_last_error() describes the last
 *     failure of the calling thread.  WG_ERR_INVALID corresponds to the reference's
 *     std::invalid_argument, WG_ERR_RUNTIME to its std::runtime_error (missing key or table).
 *   - One context serves one stream per in-flight operation: each stream gets its own
 *     scratch on first use (wg_ctx_reserve allocates it ahead, e.g. before graph capture).
 */
#ifndef WALSH_GPU_H
#define WALSH_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WG_OK 0
#define WG_ERR_INVALID (-1)
#define WG_ERR_RUNTIME (-2)
#define WG_ERR_CUDA (-3)
#define WG_ERR_NOMEM (-4)
#define WG_NOT_READY 1 /* wg_serve_wait: the request has not finished within the timeout */

/* Switching-key kinds for wg_ctx_set_key / wg_keyswitch. */
#define WG_KEY_RELIN 0       /* s^2 -> s           (relinearization_key_generation.cpp:130-199) */
#define WG_KEY_CONJ 1        /* conj(s) -> s       (conjugation_key_generation.cpp:63-167) */
#define WG_KEY_ROTATION 2    /* s -> pi^-1(s)      (rotation_key_generation.cpp:92-199) */
/* dense s -> sparse s' at q0 * p0 only: compact key, one level-0 part whose a and b hold the
 * q0 limb then the p0 limb (2 x 2 x N words; parts = 1, key_level = 0).
 * generate_secret_key_switch_key_q0p0_hybrid, ckks_context.cpp:453. */
#define WG_KEY_DENSE_TO_SPARSE 3
/* sparse s' -> dense s, hybrid key (generate_secret_key_switch_key_hybrid, ckks_context.cpp:458) */
#define WG_KEY_SPARSE_TO_DENSE 4

typedef struct wg_context wg_context;

/* Last error message of the calling thread ("" when none). */
const char* wg_last_error(void);
/* ABI version (major * 100 + minor). */
int wg_version(void);

/* Prime chain: P primes for p_bits then Q primes for q_bits, each k*2N+1 searched downward
 * from 2^bits.  Replaces find_p_and_q_primes, src/util/random.cpp:115-131. */
int wg_find_primes(const uint64_t* p_bits, size_t np, const uint64_t* q_bits, size_t nq,
                   uint64_t N, uint64_t* p_out, uint64_t* q_out);

/* Host-side CKKS slot encoding (no GPU needed): the coefficient-form plaintext of the N/2 slot
 * values re[i] + i im[i] at `scale`, reduced modulo each of moduli[0..limbs), out[l*N + k].
 * Same residues as ckks_encode(..., eval = false), src/ckks/encoding/ckks_encoding.cpp:332-414. */
int wg_encode_slots(uint64_t N, const double* re, const double* im, double scale, const uint64_t* moduli,
                    size_t limbs, uint64_t* out);

/* Device-resident context for one parameter set: Q moduli q[0..nq), P moduli p[0..np), dnum
 * digits.  Builds twiddles, ModUp/ModDown and rescale tables on `device`.
 * Replaces the table-building part of CKKSContext::CKKSContext,
 * src/ckks/context/ckks_context.cpp:603-705 (keys are installed with wg_ctx_set_key). */
int wg_ctx_create(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np,
                  size_t dnum, int device, wg_context** out);
void wg_ctx_destroy(wg_context* ctx);

/* Install a switching key (copied to the device).  `rotation` is used for WG_KEY_ROTATION
 * only and is normalised modulo N/2.  Replaces the key storage behind
 * CKKSContext::getRelinHybrid / getConjugationKey / getRotationKey,
 * src/ckks/context/ckks_context.cpp:720-814. */
int wg_ctx_set_key(wg_context* ctx, int kind, int64_t rotation, const uint64_t* host_key,
                   size_t parts, size_t key_level);
/* 1 if the key is installed, else 0.  CKKSContext::hasRotationKey, ckks_context.cpp:769-775. */
/* Generate a rotation (WG_KEY_ROTATION, `rotation`), conjugation (WG_KEY_CONJ) or
 * relinearisation (WG_KEY_RELIN) switching key on the device from the ternary secret `secret`
 * (N coefficients, host memory) and install it like wg_ctx_set_key (all Q limbs, the context's
 * hybrid parts, folded, Montgomery form): replaces generate_rotation_key_hybrid
 * (src/ckks/context/rotation_key_generation.cpp:92-199), generate_conjugation_key_hybrid
 * (src/ckks/context/conjugation_key_generation.cpp:63-167) and encrypt_rlk_hybrid
 * (src/ckks/context/relinearization_key_generation.cpp:131-199).  a ([part][nq + np][N]
 * canonical residues, evaluation form) and e ([part][N] integers) are the mask and noise, both
 * given or both null; when null they are drawn on the device from `seed` (uniform mask; rounded
 * normal noise of deviation sigma; a statistical generator, so a deployment that needs
 * cryptographic randomness passes its own a and e).  out (optional, host) receives the key in
 * the wg_ctx_set_key layout. */
int wg_keygen_switch_key(wg_context* ctx, int kind, int64_t rotation, const int8_t* secret, const uint64_t* a,
                           const int64_t* e, uint64_t seed, double sigma, uint64_t* out, void* stream);
/* The bootstrapping secret switches generated the same way: WG_KEY_SPARSE_TO_DENSE from `source`
 * to `target` as a hybrid key (generate_secret_key_switch_key_hybrid,
 * src/ckks/context/secret_key_generation.cpp:227-300), WG_KEY_DENSE_TO_SPARSE as the compact
 * level-0 key over q0 and p0 (generate_secret_key_switch_key_q0p0_hybrid, :302-364; a [1][2][N],
 * e [1][N]).  Other arguments as for wg_keygen_switch_key. */
int wg_keygen_secret_switch(wg_context* ctx, int kind, const int8_t* source, const int8_t* target, const uint64_t* a,
                            const int64_t* e, uint64_t seed, double sigma, uint64_t* out, void* stream);
int wg_ctx_has_key(const wg_context* ctx, int kind, int64_t rotation);
/* Allocate the scratch of `stream` now (required before capturing the stream in a graph). */
int wg_ctx_reserve(wg_context* ctx, void* stream);
/* Give back the device memory the context holds for `stream` beyond its tables and keys (the
 * stream's scratch and staging buffers) and its cache of reusable scratch chunks, after the
 * stream's queued work finishes; the next call on the stream allocates again.  For processes
 * that keep several contexts on one device and use them in turn.  (No counterpart in the
 * reference, which allocates per operation.) */
int wg_ctx_trim(wg_context* ctx, void* stream);
/* Scratch words one in-flight operation uses (informational). */
size_t wg_ctx_workspace_words(const wg_context* ctx);

/* In-place negacyclic NTT of `polys` polynomials of `limbs` limbs, `poly_stride` words
 * apart; limb l uses Q modulus first+l (basis 0) or P modulus first+l (basis 1).  Output is
 * canonical.  Replaces ntt_forward_rns_flat_inplace / ntt_inverse_rns_flat_inplace,
 * src/math/ntt/ntt.cpp:416-447. */
int wg_ntt_forward(wg_context* ctx, uint64_t* poly, size_t limbs, size_t first, int basis,
                   size_t polys, size_t poly_stride, void* stream);
int wg_ntt_inverse(wg_context* ctx, uint64_t* poly, size_t limbs, size_t first, int basis,
                   size_t polys, size_t poly_stride, void* stream);

/* EvalMod polynomial fit on the host (no device needed): the Chebyshev series of
 * 1/2 - 1/2 cos(2 pi K u / 2^double_angle) over the 2K - 1 intervals of radius
 * interval_radius / K around the multiples of 1/(2K), in 256-bit arithmetic, odd coefficients
 * zeroed and those below prune_threshold dropped.  Replaces
 * binboot_han_ki_discrete_multi_interval_approximate (src/math/poly_approx.cpp:565-681), with
 * the same coefficients bit for bit.  coeffs: room for degree + 1 doubles (*ncoeffs receives
 * the count); max_error and interval (2 doubles: min, max) may be null. */
int wg_evalmod_fit(double K, size_t degree, size_t double_angle, double interval_radius,
                   size_t validation_points, double prune_threshold, double* coeffs, size_t* ncoeffs,
                   double* max_error, double* interval);
/* EvalMod K of a sparse secret of `hamming_weight` over `coefficients` coefficients at failure
 * probability 2^log2_failure (an integer exponent is exact): replaces required_binboot_k_bound
 * (src/math/binboot_k_bound.cpp:53-89), returning its evalmod_k. */
int wg_evalmod_k_bound(size_t coefficients, size_t hamming_weight, double log2_failure, size_t* k);

/* NTT geometry autotuner (no counterpart in the reference, whose transform has one loop
 * order, ntt.cpp:235-386).  Four geometries compute the same words: 0 = 8 residues per thread
 * with twiddles staged in shared memory, 1 = 8 residues, twiddles read from the table,
 * 2 = 16 residues, staged, 3 = 16 residues, from the table.  wg_ctx_create times each one per
 * direction and phase on the device (once per device and ring degree in the process) and
 * keeps the fastest.  wg_ntt_tuning reports chosen[direction][phase] (direction 0 forward,
 * 1 inverse; phase 0 rows = low index bits, 1 columns = high bits; 4 ints), the timings
 * ms[direction][phase][geometry] (16 floats, best of three launches over a batch of `limbs`
 * limb-transforms) and that batch size.  Either output pointer may be null. */
int wg_ntt_tuning(const wg_context* ctx, int* chosen, float* ms, int* limbs);
/* Pin the geometry of one (direction, phase) for this context (geometry < 0: restore the
 * tuned choice). */
int wg_ntt_set_geometry(wg_context* ctx, int direction, int phase, int geometry);
/* Batched key switches and rescales (every circuit entry point) run their base changes inside
 * the NTT column phases around them by default: one kernel finishes the inverse transform of the
 * source limbs, changes the basis (ModUp, ModDown, the rescale's rounded remainders) and starts
 * the forward transform of every output limb, so those limbs do not pass through device memory
 * in between; the final combine of a key switch and the rescale's finish step run as the
 * epilogue of the last forward row phase.  ckks_hybrid_key_switch_inplace
 * (src/ckks/operations/keyswitch/ckks_keyswitch.cpp:1330-1641) and ckks_rescale
 * (src/ckks/operations/arith/ckks_rescale.cpp:68-148) compute the same words step by step.
 * mode 1 (the default) fuses a step when its launch fills the device at least twice (the fused
 * kernels run one 128-thread block per job and 1024-coefficient column tile), so a single
 * ciphertext keeps the wider separate launches; mode 2 always fuses, mode 0 never.  The words
 * are identical in every mode. */
int wg_set_ntt_fusion(wg_context* ctx, int mode);

/* Hybrid key switch of key_term at `level` with the installed key (kind, rotation):
 * b = (b_add ? b + ks_b : ks_b), a = (a_add ? a + ks_a : ks_a).  key_term may alias a.
 * Replaces ckks_hybrid_key_switch_inplace (Montgomery, folded keys),
 * src/ckks/operations/keyswitch/ckks_keyswitch.cpp:1330-1641. */
int wg_keyswitch(wg_context* ctx, size_t level, const uint64_t* key_term, int kind,
                 int64_t rotation, uint64_t* b, uint64_t* a, int b_add, int a_add, void* stream);

/* Rotation by `rotation` slots (key switch to pi^-1(s), then the automorphism).
 * Replaces ckks_rotate_inplace, src/ckks/operations/keyswitch/ckks_rotation.cpp:41-96. */
int wg_rotate(wg_context* ctx, size_t level, uint64_t* b, uint64_t* a, int64_t rotation,
              void* stream);

/* Complex conjugation (automorphism X -> X^(2N-1), then the switch).
 * Replaces ckks_conjugate_inplace, src/ckks/operations/keyswitch/ckks_conjugate.cpp:16-61. */
int wg_conjugate(wg_context* ctx, size_t level, uint64_t* b, uint64_t* a, void* stream);

/* Several rotations of one ciphertext; out holds nrot ciphertexts laid out
 * [rot][b, a][level+1][N].  Replaces the hoisted path ckks_hoist_ciphertext_a_qp_eval +
 * ckks_hybrid_key_switch_hoisted_inplace, ckks_keyswitch.cpp:344-373 and 1072-1328. */
int wg_rotate_many(wg_context* ctx, size_t level, const uint64_t* b, const uint64_t* a,
                   const int64_t* rotations, size_t nrot, uint64_t* out, void* stream);

/* Tensor product: (b1, a1) <- (b1 b2, a1 b2 + b1 a2), c2 <- a1 a2 (Barrett products).
 * Replaces ckks_mul_inplace(ct, ct), src/ckks/operations/arith/ckks_mul.cpp:90-157. */
int wg_mul(wg_context* ctx, size_t level, uint64_t* b1, uint64_t* a1, const uint64_t* b2,
           const uint64_t* a2, uint64_t* c2, void* stream);

/* Relinearization of (c0, c1, c2) into (c0, c1).
 * Replaces ckks_relin_hybrid_inplace, src/ckks/operations/keyswitch/ckks_relin.cpp:8-44. */
int wg_relin(wg_context* ctx, size_t level, uint64_t* c0, uint64_t* c1, const uint64_t* c2,
             void* stream);

/* Rescale `npolys` polynomials (poly_stride words apart) from `level` to level-1; the first
 * level*N words of each polynomial hold the result, and the dropped limb's words are left as
 * scratch (here and in every batched entry point that rescales).
 * Replaces ckks_rescale, src/ckks/operations/arith/ckks_rescale.cpp:68-148. */
int wg_rescale(wg_context* ctx, size_t level, uint64_t* polys, size_t npolys,
               size_t poly_stride, void* stream);

/* x <- x + y / x <- x - y over npolys polynomials at `level`.
 * Replaces ckks_add_inplace / ckks_sub_inplace (ct, ct),
 * src/ckks/operations/arith/ckks_addition.cpp:62-139. */
int wg_add(wg_context* ctx, size_t level, uint64_t* x, const uint64_t* y, size_t npolys,
           size_t poly_stride, void* stream);
int wg_sub(wg_context* ctx, size_t level, uint64_t* x, const uint64_t* y, size_t npolys,
           size_t poly_stride, void* stream);

/* Batched multiply + relinearize + rescale + rotate over `count` ciphertexts at arbitrary
 * levels: for ciphertext i, (xb[i], xa[i]) <- rotate(rescale(relin(x_i * y_i)), rots[i]).
 * Pointer arrays are host arrays of device pointers; each x buffer must hold
 * (levels[i]+1)*N words per polynomial and receives levels[i]*N words (limb levels[i] is left as
 * scratch).  The workload the
 * reference runs as ckks_mul_inplace, ckks_relin_hybrid_inplace, ckks_rescale,
 * ckks_rotate_inplace per ciphertext with OpenMP over ciphertexts.  Every stage is one launch
 * over all ciphertexts, limbs and digits (job tables uploaded once per call). */
int wg_batch_mul_relin_rescale_rotate(wg_context* ctx, size_t count, const size_t* levels,
                                      uint64_t* const* xb, uint64_t* const* xa,
                                      const uint64_t* const* yb, const uint64_t* const* ya,
                                      const int64_t* rots, void* stream);

/* Bootstrapping boundary steps, batched over `count` ciphertexts (host arrays of device
 * pointers).
 * ModRaise: limb 0 (q0, evaluation form) of each b[i] / a[i] is lifted to target_level+1 limbs
 * in place (centered lift, then NTT); buffers hold (target_level+1)*N words.  Replaces
 * ckks_modraise_inplace, src/ckks/operations/bootstrap/ckks_modraise.cpp:103-110 (the caller
 * tracks the secret owner, which the reference checks).
 * Dense-to-sparse: level-0 key switch through q0 and p0 only with the WG_KEY_DENSE_TO_SPARSE
 * key (folded, Montgomery).  Replaces ckks_key_switch_dense_to_sparse_inplace /
 * ckks_q0p0_key_switch_level0_inplace, src/ckks/operations/keyswitch/ckks_keyswitch.cpp:1661-1856.
 * Sparse-to-dense: hybrid key switch of ciphertext i at levels[i] with the
 * WG_KEY_SPARSE_TO_DENSE key.  Replaces ckks_key_switch_sparse_to_dense_inplace,
 * ckks_keyswitch.cpp:1858-1869. */
int wg_modraise(wg_context* ctx, size_t count, size_t target_level, uint64_t* const* b, uint64_t* const* a,
                void* stream);
int wg_dense_to_sparse(wg_context* ctx, size_t count, uint64_t* const* b, uint64_t* const* a, void* stream);
int wg_sparse_to_dense(wg_context* ctx, size_t count, const size_t* levels, uint64_t* const* b,
                       uint64_t* const* a, void* stream);

/* Chebyshev polynomial evaluation of `count` ciphertexts that share `level` and `scale`
 * (device pointers b[i], a[i]; the inputs are read only): sum_k coeffs[k] T_k(x) with the
 * reference's power basis, scale-aware Paterson-Stockmeyer schedule and constant rounding, so
 * the residues equal those of ckks_evalchebyshev_preconditioned
 * (src/ckks/operations/evalpoly/ckks_evalpoly.cpp:1221-1256) for the same inputs.
 * target_scale <= 0 keeps `scale`; default_scale is the parameter set's scale
 * (CKKSParams::getScale, which decides how many moduli one rescale consumes).  The results go
 * to out_b[i], out_a[i] (room for level+1 limbs) at *out_level with scale *out_scale.  Needs
 * the relinearisation key.  Temporary ciphertexts come from the stream-ordered allocator. */
int wg_evalchebyshev(wg_context* ctx, size_t count, size_t level, double scale, const double* coeffs,
                     size_t ncoeffs, double target_scale, double default_scale, uint64_t* const* b,
                     uint64_t* const* a, uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level,
                     double* out_scale, void* stream);

/* The same batched pipeline planned once for fixed buffers and captured as a CUDA graph
 * (no counterpart in the reference, which plans nothing ahead).  Create takes the arguments
 * of wg_batch_mul_relin_rescale_rotate minus the stream, builds the job tables, uploads them
 * into memory the plan owns (with its own scratch) and captures the launch sequence; launch
 * replays it on `stream`, with no host planning or upload, reading and writing the buffers
 * given at creation, whose current contents are used.  Results equal those of
 * wg_batch_mul_relin_rescale_rotate.  Launches of one plan must not overlap (they share its
 * scratch); different plans are independent.  The plan refers to the context's tables and
 * to the switching keys installed at creation: destroy it before the context, and do not
 * replace those keys while it exists. */
typedef struct wg_batch_plan wg_batch_plan;
int wg_batch_plan_create(wg_context* ctx, size_t count, const size_t* levels, uint64_t* const* xb,
                         uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                         const int64_t* rots, wg_batch_plan** out);
int wg_batch_plan_launch(wg_batch_plan* plan, void* stream);
void wg_batch_plan_destroy(wg_batch_plan* plan);

/* One CoeffToSlot / SlotToCoeff stage: a baby-step / giant-step linear transform evaluated in
 * the QP basis (hoisted baby rotations without ModDown, one ModDown per giant step).
 * `diagonals` (host) holds the stage's nterms plaintexts [term][level+1+K limbs][N] in
 * Montgomery form, `indices` their diagonal indices, exactly as the reference's plan stores
 * them (CKKSLinearTransformOwnedStage, src/ckks/operations/bootstrap/
 * ckks_linear_transform_plan.hpp:29-44).  Rotation keys for the baby steps 1..baby-1 and giant
 * steps g*baby must be installed.  Apply replaces ckks_apply_linear_transform_owned_stage_qp
 * (src/ckks/operations/bootstrap/ckks_linear_transform.cpp:1174-1407) on `count` ciphertexts
 * at the stage's level at once (the diagonals are read once per batch); the result overwrites
 * (b[i], a[i]), one level lower when the stage rescales. */
typedef struct wg_lt_stage wg_lt_stage;
int wg_lt_stage_create(wg_context* ctx, size_t level, size_t nterms, const uint64_t* indices,
                       const uint64_t* diagonals, size_t baby_step_count, size_t slot_count,
                       int rescale_after, wg_lt_stage** out);
void wg_lt_stage_destroy(wg_lt_stage* stage);
/* Shape of a stage: level, term count, baby-step count, logical slots, rescale flag and the
 * plaintext scale of its diagonals (0 when the stage was made from caller-supplied words). */
int wg_lt_stage_info(const wg_lt_stage* stage, size_t* level, size_t* nterms, size_t* baby, size_t* slots,
                     int* rescale_after, double* plaintext_scale);
/* Copy a stage's diagonal indices (nterms) and QP diagonals ([term][level + 1 + P limbs][N],
 * Montgomery form) to host memory. */
int wg_lt_stage_download(wg_context* ctx, const wg_lt_stage* stage, uint64_t* indices, uint64_t* diagonals);

/* One homomorphic DFT to factorize into BSGS stages (the reference's
 * CKKSBootstrapDftMatrixLiteral, src/ckks/operations/bootstrap/ckks_bootstrap_dft.hpp). */
typedef struct wg_dft_literal {
    int coeffs_to_slots;        /* 1: CoeffsToSlots, 0: SlotsToCoeffs */
    size_t level;               /* level of the first stage */
    size_t baby_step_count;     /* 0: the cheapest split per stage */
    int log_bsgs_ratio;         /* giant steps weigh 2^log_bsgs_ratio baby steps */
    size_t stage_count;         /* factors when ngroups == 0 (then each stage rescales) */
    const size_t* group_sizes;  /* ngroups entries: factors per rescale group */
    const size_t* group_bits;   /* one log2 plaintext scale per factor, group after group */
    size_t ngroups;
    const size_t* merge_depths; /* FFT levels per factor (nmerge == 0: balanced) */
    size_t nmerge;
    size_t active_slots;        /* 0: N/2 */
    double transform_scale;
    size_t input_selector_start, input_selector_size; /* SlotsToCoeffs only; size 0: none */
} wg_dft_literal;
/* Generate the factorized DFT's stages on the context's device: diagonals on the host, encoded
 * on the device as QP plaintexts in Montgomery form.  Replaces ckks_generate_bootstrap_dft_plan
 * (src/ckks/operations/bootstrap/ckks_bootstrap_dft.cpp:961-1079), with the reference's
 * diagonal residues; the stages are ordinary wg_lt_stage handles (wg_lt_stage_destroy each).
 * *nstages receives the stage count (at most max_stages are written). */
int wg_dft_plan_create(wg_context* ctx, const wg_dft_literal* literal, wg_lt_stage** stages, size_t max_stages,
                       size_t* nstages, void* stream);
/* The same plan on the host only (no device): for stage `stage` of the plan of a ring of degree
 * N with Q moduli q[nq], its level, term count, baby steps, rescale flag, plaintext scale,
 * diagonal indices (nterms) and, when diagonals is not null, the diagonals before encoding
 * ([term][active slots] complex values as re, im pairs).  *nstages receives the stage count.
 * Pass null indices to query the sizes first. */
int wg_dft_plan_describe(uint64_t N, const uint64_t* q, size_t nq, const wg_dft_literal* literal, size_t stage,
                         size_t* nstages, size_t* level, size_t* nterms, size_t* baby, int* rescale_after,
                         double* plaintext_scale, uint64_t* indices, double* diagonals);
int wg_lt_stage_apply(wg_context* ctx, const wg_lt_stage* stage, size_t count, uint64_t* const* b,
                      uint64_t* const* a, void* stream);

/* EvalMod bootstrap of `count` packed ciphertexts (no counterpart as a batch: the reference
 * boots one packed ciphertext per call): replaces ckks_batch_bootstrap_evalmod_from_complex_packed
 * (src/ckks/operations/bootstrap/ckks_bootstrap_evalmod_inplace.cpp:416-434) -- SlotToCoeff
 * with the `s2c` stages, dense-to-sparse switch, ModRaise to params->depth, sparse-to-dense
 * switch, sparse-slot trace when active_slots < slots, CoeffToSlot with the `c2s` stages, the
 * conjugate split (ct + conj, -i (ct - conj)), and EvalMod on both halves (Chebyshev series
 * `coeffs` at scale 2^evalmod_log_scale, then double_angle doubling steps).  Inputs at level
 * s2c_depth with scale params->scale; b[i] / a[i] need room for depth+1 limbs and are
 * overwritten; the two results go to out0_* / out1_* (room for depth+1 limbs) at *out_level
 * with scale *out_scale.  Needs the relinearisation, conjugation, both secret-switch keys and
 * the stages' rotation keys. */
typedef struct wg_bootstrap_params {
    size_t s2c_depth, depth, evalmod_log_scale, double_angle, active_slots, slots;
    double scale;
} wg_bootstrap_params;
int wg_bootstrap_evalmod(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                         size_t ns2c, const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs,
                         size_t ncoeffs, size_t count, uint64_t* const* b, uint64_t* const* a,
                         uint64_t* const* out0_b, uint64_t* const* out0_a, uint64_t* const* out1_b,
                         uint64_t* const* out1_a, size_t* out_level, double* out_scale, void* stream);

/* The AES S-box on lazy bits through its Walsh expansion, mask-packed, for `count` S-box
 * instances at once (the reference runs one per call): replaces
 * ckks_walsh_sbox_complex_blocks_mask_packed (src/ckks/operations/circuits/
 * ckks_walsh_sbox.cpp:1286-1323).  in_b / in_a hold 8 * count device pointers, bit-major
 * (bit k of instance i at [k * count + i]), each a ciphertext at `level` (= s2c_depth) with
 * scale `scale` (= params->scale) and room for level+1 limbs; outputs likewise into out_b /
 * out_a (room for depth+1 limbs), with each output bit's level and scale in out_level[8] /
 * out_scale[8].  The bootstrap arguments are those of wg_bootstrap_evalmod; the rotation keys
 * +-k * block_count (k = 1..29) must be installed besides the bootstrap's keys. */
int wg_walsh_sbox(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                  const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                  size_t block_count, size_t count, size_t level, double scale, uint64_t* const* in_b,
                  uint64_t* const* in_a, uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level,
                  double* out_scale, void* stream);

/* AES-128 in CTR mode on lazy bits, evaluated on the device: replaces
 * ckks_aes_ctr_walsh_sbox_complex_blocks (src/ckks/operations/circuits/aes/
 * ckks_aes_ctr_walsh_sbox.cpp:1037-1051).  Each of the 128 state-bit ciphertexts carries, in
 * slot s < active_blocks, block s in its real part and block active_blocks + s in its
 * imaginary part.  key_b / key_a: the 1408 encrypted expanded-key bits (device pointers, level
 * key_level = s2c_depth + 1) with their scales; counters / ciphertexts: 2 * active_blocks public
 * 16-byte blocks (host memory).  Rounds 1..10 (active-slot mask, SubBytes by the mask-packed
 * Walsh S-box on all 16 bytes at once, ShiftRows, MixColumns except in round 10,
 * AddRoundKey), the public ciphertext XOR and the final binary refresh (packed bootstraps);
 * the 128 results go to out_b / out_a (room for depth+1 limbs) with levels and scales.
 * SlotToCoeff needs a plan per bootstrap input scale: s2c for inputs at the parameter scale,
 * s2c_x2 for inputs at twice it (the state after the first S-box); packing_block_count and
 * packed_segment_count are the parameter set's AES-Walsh packing (512 and 32 for walsh15).
 * Keys: relinearisation, conjugation, both secret switches, all plan rotations and
 * +-k * packing_block_count. */
int wg_aes_ctr_walsh(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                     size_t ns2c, const wg_lt_stage* const* s2c_x2, size_t ns2c_x2,
                     const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                     size_t packing_block_count, size_t packed_segment_count, const uint64_t* const* key_b,
                     const uint64_t* const* key_a, const double* key_scales, size_t key_level,
                     const uint8_t* counters, const uint8_t* ciphertexts, size_t active_blocks,
                     uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                     void* stream);
/* The same AES-CTR issued at the reference's call granularity (no counterpart in the reference
 * as an entry point): every S-box instance and every refresh bootstrap as its own call instead
 * of one batch per round, the plain per-operation GPU path the batched evaluation is measured
 * against.  Same arguments and the same output words as wg_aes_ctr_walsh. */
int wg_aes_ctr_walsh_plain(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                           size_t ns2c, const wg_lt_stage* const* s2c_x2, size_t ns2c_x2,
                           const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                           size_t packing_block_count, size_t packed_segment_count, const uint64_t* const* key_b,
                           const uint64_t* const* key_a, const double* key_scales, size_t key_level,
                           const uint8_t* counters, const uint8_t* ciphertexts, size_t active_blocks,
                           uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                           void* stream);

/* The XBOOT AES S-box on lazy bits (ckks_aes_xboot_sbox_impl,
 * src/ckks/operations/circuits/aes/ckks_aes_ctr.cpp:280-336, with its monomial tree :185-256
 * and coefficients :258-278) for `count` instances: in_b / in_a hold 8 x count ciphertexts
 * ([bit][instance], (level + 1) N words each) at `level` and `scale`; out_b / out_a receive the
 * 8 output bits (room for level + 1 limbs each) at out_level[bit], out_scale[bit] (three levels
 * lower, same scale).  Needs the relinearisation key; level >= 3. */
int wg_xboot_sbox(wg_context* ctx, size_t count, size_t level, double scale, uint64_t* const* in_b,
                  uint64_t* const* in_a, uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level,
                  double* out_scale, void* stream);
/* The integer coefficients of each S-box output bit over the monomials of the 8 input bits:
 * out[bit * 256 + mask] (mask 0 = constant term). */
int wg_xboot_sbox_coefficients(int64_t* out);

/* The XBOOT pair bootstrap for `count` pairs at once (the reference boots one pair per call):
 * replaces ckks_batch_bootstrap_evalmod_inplace (src/ckks/operations/bootstrap/
 * ckks_bootstrap_evalmod_inplace.cpp:393-414).  Pair i is (b0[i], a0[i]) and (b1[i], a1[i]) at
 * level s2c_depth; every first ciphertext has scale `scale`.  ct0 + i * ct1 (the slot constant
 * i encoded at scale 1) is bootstrapped as in wg_bootstrap_evalmod, and the two results
 * overwrite the pair's buffers (room for depth+1 limbs each) at *out_level with *out_scale. */
int wg_bootstrap_pair(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                      const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs, size_t count,
                      double scale, uint64_t* const* b0, uint64_t* const* a0, uint64_t* const* b1,
                      uint64_t* const* a1, size_t* out_level, double* out_scale, void* stream);

/* AES-128 in CTR mode on lazy bits with the XBOOT S-box, evaluated on the device: replaces
 * ckks_aes_ctr (src/ckks/operations/circuits/aes/ckks_aes_ctr.cpp:757-779).  Each of the 128
 * state-bit ciphertexts carries block (s mod active_slots) in slot s.  key_b / key_a: the 1408
 * encrypted expanded-key bits (device pointers, as ckks_aes128_encrypt_expanded_round_key_bits
 * makes them: round 0 at key_levels[0..127], the others at the S2C depth) with their scales and
 * levels; counters / ciphertexts: `blocks` public 16-byte blocks each (host memory, 1 <= blocks
 * <= params->active_slots).  Initial public XOR of the counter bits, rounds 1..10 (SubBytes by
 * the XBOOT S-box on all 16 bytes at once, ShiftRows, MixColumns except in round 10,
 * AddRoundKey, then, in rounds 1..9, the 64 pair bootstraps of the state), the public
 * ciphertext XOR and a last pair-bootstrap refresh; the 128 results go to out_b / out_a (room
 * for depth+1 limbs) with their levels and scales.  Keys: relinearisation, conjugation, both
 * secret switches and the plans' rotations. */
int wg_aes_ctr_xboot(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                     const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                     const uint64_t* const* key_b, const uint64_t* const* key_a, const double* key_scales,
                     const size_t* key_levels, const uint8_t* counters, const uint8_t* ciphertexts, size_t blocks,
                     uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                     void* stream);

/* Two steps of wg_aes_ctr_xboot on their own (file-internal in the reference, so no reference
 * interface is replaced): the initial public XOR of the counter bit planes
 * (make_batched_initial_counter_state, src/ckks/operations/circuits/aes/ckks_aes_ctr.cpp:576-683)
 * from the 128 round-0 key bits (key_b / key_a with their scales and levels, one common level
 * L >= 1) and `blocks` counter blocks; out_b / out_a need room for L + 1 limbs and receive the
 * state at *out_level = L - 1 with per-bit scales out_scale[128]. */
int wg_xboot_initial_state(wg_context* ctx, const wg_bootstrap_params* params, const uint64_t* const* key_b,
                           const uint64_t* const* key_a, const double* key_scales, const size_t* key_levels,
                           const uint8_t* counters, size_t blocks, uint64_t* const* out_b, uint64_t* const* out_a,
                           size_t* out_level, double* out_scale, void* stream);
/* ... and one round's linear layers (shift_rows_inplace, fmix_columns_inplace when `mix`,
 * add_round_key_lazy_inplace; ckks_aes_ctr.cpp:460-554) on 128 state bits at `level` with
 * scales in_scale[128], adding the 128 key bits key_b / key_a (levels >= level); results at
 * `level` in out_b / out_a (not aliasing the inputs) with the scales the reference's in-place
 * additions keep in out_scale[128]. */
int wg_xboot_linear_layer(wg_context* ctx, size_t level, const double* in_scale, uint64_t* const* in_b,
                          uint64_t* const* in_a, const uint64_t* const* key_b, const uint64_t* const* key_a,
                          const size_t* key_levels, int mix, uint64_t* const* out_b, uint64_t* const* out_a,
                          double* out_scale, void* stream);

/* Secret-key encryption on the device of `count` evaluation-form plaintexts (device pointers,
 * level + 1 limbs each) under the ternary `secret` (host, N coefficients): b = pt + e - a s into
 * out_b / out_a; replaces ckks_encrypt (src/ckks/encoding/ckks_encoding.cpp:522-566, through
 * ckks_encrypt_custom_eval :478-520).  a ([count][level + 1][N] canonical residues) and e
 * ([count][N] integers) both given or both null (then drawn from `seed`, as for
 * wg_keygen_switch_key; give each call its own seed). */
int wg_encrypt_symmetric(wg_context* ctx, size_t count, size_t level, const uint64_t* const* pts, const int8_t* secret,
                         const uint64_t* a, const int64_t* e, uint64_t seed, double sigma, uint64_t* const* out_b,
                         uint64_t* const* out_a, void* stream);
/* The XBOOT AES's encrypted round-key bits on the device: replaces
 * ckks_aes128_encrypt_expanded_round_key_bits (src/ckks/operations/circuits/aes/
 * ckks_aes_ctr.cpp:687-725).  Bit k of the 176-byte expanded key as the constant slot value at
 * params->scale, encrypted at params->s2c_depth (bits 0..127: first_round_key_level above it);
 * out_b / out_a: 1408 device buffers with room for their level + 1 limbs; their scales and
 * levels in out_scale[1408] / out_level[1408]. */
int wg_aes_xboot_encrypt_round_key_bits(wg_context* ctx, const wg_bootstrap_params* params,
                                        const uint8_t* expanded_key, size_t first_round_key_level,
                                        const int8_t* secret, uint64_t seed, double sigma, uint64_t* const* out_b,
                                        uint64_t* const* out_a, double* out_scale, size_t* out_level, void* stream);

/* CKKS slot encoding on the device of `count` slot vectors (re / im: host arrays [count][N/2])
 * at `scale` into out[c] (device, `limbs` Q limbs of N words), in evaluation form when `eval`,
 * else coefficient form: replaces ckks_encode (src/ckks/encoding/ckks_encoding.cpp:332-414).
 * The same FP64 operations as the reference's encoder (and as the host wg_encode_slots), so the
 * same residues. */
int wg_encode_slots_device(wg_context* ctx, size_t count, size_t limbs, double scale, const double* re, const double* im,
                    uint64_t* const* out, int eval, void* stream);

/* Keys and plans on disk (no counterpart in the reference, which rebuilds both in every
 * context constructor): wg_bundle_save writes the context's parameters, every installed
 * switching key and the given linear-transform stages to `path`; wg_bundle_load checks that the
 * file's ring degree, moduli and dnum are the context's, installs its keys (as wg_ctx_set_key)
 * and creates its stages (up to max_stages handles into stages, their number in *nstages).
 * Format: "WGB1", version, parameters, key records, stage records and a 64-bit FNV-1a checksum
 * (aes-walsh-ckks_b200/csrc/wg_bundle.hpp); a damaged or foreign file is rejected with
 * WG_ERR_INVALID.  Both hold the whole bundle in host memory while they run (about twice the
 * keys' and diagonals' size); keys installed before a failing record stay installed. */
int wg_bundle_save(wg_context* ctx, const char* path, const wg_lt_stage* const* stages, size_t nstages);
int wg_bundle_load(wg_context* ctx, const char* path, wg_lt_stage** stages, size_t max_stages, size_t* nstages);

/* Ciphertext wire format (host memory only; no counterpart in the reference, which keeps
 * ciphertexts in memory): a self-checking record of one ciphertext ("WGC1", version, N, level,
 * polynomial count, scale, secret owner and encoding labels, the level + 1 moduli, the
 * residues [poly][level + 1][N] in evaluation form, FNV-1a checksum).  wg_ct_wire_bytes gives
 * the record's size; wg_ct_wire_encode writes it from host residues `polys`; wg_ct_wire_decode
 * checks a record against the ring degree N and the Q moduli q[nq] of the receiving context
 * (same degree, the record's moduli a prefix of q, every residue below its modulus, checksum)
 * and copies out its residues (polys: room for cap_words words) and labels.  Move residues to
 * and from the device with wg_memcpy_dtoh / wg_memcpy_htod. */
size_t wg_ct_wire_bytes(uint64_t N, size_t level, size_t npolys);
int wg_ct_wire_encode(uint64_t N, const uint64_t* q, size_t level, size_t npolys, const uint64_t* polys, double scale,
                      int secret_owner, int encoding_state, uint8_t* out, size_t cap);
int wg_ct_wire_decode(const uint8_t* in, size_t len, uint64_t N, const uint64_t* q, size_t nq, uint64_t* polys,
                      size_t cap_words, size_t* level, size_t* npolys, double* scale, int* secret_owner,
                      int* encoding_state);

/* The Walsh AES's encrypted round-key bits on the device: replaces
 * ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks (src/ckks/operations/circuits/
 * aes/ckks_aes_ctr_walsh_sbox.cpp:981-1035).  Bit k of the 176-byte expanded key as (v, v) in the
 * first active_blocks slots (zero elsewhere) at params->scale for rounds 0 and 10 and a quarter
 * of it for rounds 1..9, encrypted under `secret` at params->s2c_depth + 1; out_b / out_a: 1408
 * device buffers with room for that level + 1 limbs; scales and levels in out_scale[1408] /
 * out_level[1408].  Mask and noise drawn on the device from `seed`. */
int wg_aes_walsh_encrypt_round_key_bits(wg_context* ctx, const wg_bootstrap_params* params,
                                        const uint8_t* expanded_key, size_t active_blocks, const int8_t* secret,
                                        uint64_t seed, double sigma, uint64_t* const* out_b, uint64_t* const* out_a,
                                        double* out_scale, size_t* out_level, void* stream);

/* Decryption and decoding on the device (client side): replaces ckks_decrypt
 * (src/ckks/encoding/ckks_encoding.cpp:89-171, 567-575) for `count` ciphertexts at `level`
 * (device pointers b[k], a[k], and c2[k] for three-polynomial ones or c2 null) with scales[k],
 * under the ternary `secret` (host, N coefficients); the N/2 slot values of each go to the host
 * arrays re / im ([count][N/2]).  Floating-point results agree with the reference's to FP64
 * rounding (a two-modulus CRT and another FFT evaluation order), not bit for bit. */
int wg_decrypt_decode(wg_context* ctx, size_t count, size_t level, const double* scales, const uint64_t* const* b,
                      const uint64_t* const* a, const uint64_t* const* c2, const int8_t* secret, double* re, double* im,
                      void* stream);

/* Continuous-batching AES-CTR transciphering service (no counterpart in the reference, whose
 * benchmark evaluates one AES-CTR batch at a time, bench/aes_bench.cpp:197-291).  Requests of
 * 2..max_blocks counter blocks (even counts) queue up; each of `workers` worker threads owns a
 * stream, takes every queued request, in arrival order, that still fits into one evaluation's
 * block slots (2 x packing_block_count by default; a request never splits), runs wg_aes_ctr_walsh on the
 * concatenated blocks padded with zero blocks to the full 2 x packing_block_count slots (the
 * walsh15 rotation keys serve that block count only) and copies the 128 output bit ciphertexts
 * into every request's buffers.
 * Evaluations of different workers run concurrently on the device; at most
 * max(1, hbm_budget_bytes / eval_bytes) of them at once when both are set.  The stages, keys,
 * coefficients and parameters passed to wg_serve_create must outlive the server.  Block b of an
 * evaluation sits in slot b mod active_blocks, real part for b < active_blocks, imaginary part
 * otherwise; a request's blocks are the evaluation blocks [block_offset, block_offset + blocks). */
typedef struct wg_server wg_server;
typedef struct wg_serve_config {
    size_t workers;          /* concurrent evaluations (>= 1) */
    size_t hbm_budget_bytes; /* device bytes the evaluations may take together (0: no limit) */
    size_t eval_bytes;       /* device bytes one evaluation takes (admission estimate; 0: none) */
    size_t max_blocks;       /* block slots per evaluation (0: 2 x packing_block_count) */
    double batch_window_ms;  /* a free worker waits up to this long after the oldest queued request
                                for more requests to fill its evaluation (0: start at once) */
    int priority;            /* 1: the workers' streams take the device's highest scheduling
                                priority, so this server's (short) evaluations are not queued behind
                                another server's long ones; 0: default */
    struct wg_serve_budget* budget; /* device bytes shared with other servers (null: none); each
                                evaluation holds eval_bytes of it while it runs */
} wg_serve_config;
/* A device-memory budget shared by several servers on one device (no counterpart in the
 * reference): an evaluation starts only when its eval_bytes fit beside the evaluations of every
 * server holding the budget.  Destroy it after the servers that use it. */
typedef struct wg_serve_budget wg_serve_budget;
int wg_serve_budget_create(size_t bytes, wg_serve_budget** out);
void wg_serve_budget_destroy(wg_serve_budget* budget);
typedef struct wg_serve_result {
    int status;              /* WG_OK, or the error code of the request's evaluation */
    size_t block_offset, active_blocks, batch_requests, batch_blocks;
    double queue_ms, latency_ms; /* submission to evaluation start / to completion */
    size_t out_level[128];
    double out_scale[128];
} wg_serve_result;
int wg_serve_create(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                    const wg_lt_stage* const* s2c_x2, size_t ns2c_x2, const wg_lt_stage* const* c2s, size_t nc2s,
                    const double* coeffs, size_t ncoeffs, size_t packing_block_count, size_t packed_segment_count,
                    const uint64_t* const* key_b, const uint64_t* const* key_a, const double* key_scales,
                    size_t key_level, const wg_serve_config* config, wg_server** out);
/* The same service over XBOOT evaluations (wg_aes_ctr_xboot) of an XBOOT parameter set: requests
 * of 1..max_blocks blocks (max_blocks 0: params->active_slots), concatenated in arrival order with
 * no padding; block b of an evaluation sits in slot b (real part), active_blocks reports the
 * active slot count.  Key bits with their scales and levels as for wg_aes_ctr_xboot.  A server
 * per parameter set on one device serves a mixed stream (e.g. walsh15 beside xboot15). */
int wg_serve_create_xboot(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                          size_t ns2c, const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs,
                          size_t ncoeffs, const uint64_t* const* key_b, const uint64_t* const* key_a,
                          const double* key_scales, const size_t* key_levels, const wg_serve_config* config,
                          wg_server** out);
/* Queue one request: `blocks` counter blocks and as many ciphertext blocks (16 bytes each,
 * copied at submission); out_b / out_a: 128 device buffers of (depth + 1) N words each. */
int wg_serve_submit(wg_server* server, const uint8_t* counters, const uint8_t* ciphertexts, size_t blocks,
                    uint64_t* const* out_b, uint64_t* const* out_a, uint64_t* id);
/* Wait up to timeout_s seconds (negative: no limit).  WG_OK with *result filled once the request
 * has finished (its status in result->status; the message of a failed evaluation in
 * wg_last_error()), WG_NOT_READY on timeout.  A finished request is collected once. */
int wg_serve_wait(wg_server* server, uint64_t id, double timeout_s, wg_serve_result* result);
/* Finishes every queued request, then stops the workers and frees the server. */
void wg_serve_destroy(wg_server* server);

/* Rotation that allocates no device memory (no counterpart in the reference, whose
 * operations all allocate host vectors).  For callers that cannot call cudaMalloc when they
 * rotate: memory reserved up front by another allocator, or loops that must not trigger the
 * synchronisation an allocation can cause.  Same result as wg_rotate.  The key-switch scratch is a file-scope static device
 * array of 32 MiB that every GPU loading the library holds until exit; a level needing more
 * returns WG_ERR_INVALID.  All calls share that array (nothing in it needs clearing between
 * calls), so calls that overlap on the GPU race: serialise them.  Every call makes the
 * context's device current and leaves it current.  The first call on a device looks up the
 * array's address; make it before any stream capture. */
int wg_rotate_noalloc(wg_context* ctx, size_t level, uint64_t* b, uint64_t* a, int64_t rotation,
                      void* stream);

/* The same workload issued op by op (one ciphertext after another, a few launches per op):
 * the plain per-operation GPU path the batched entry point is measured against.  Results
 * are identical to wg_batch_mul_relin_rescale_rotate. */
int wg_sequence_mul_relin_rescale_rotate(wg_context* ctx, size_t count, const size_t* levels,
                                         uint64_t* const* xb, uint64_t* const* xa,
                                         const uint64_t* const* yb, const uint64_t* const* ya,
                                         const int64_t* rots, void* stream);

/* Instrumentation (no counterpart in the reference, which has only one wall-clock span
 * around the AES evaluation, bench/aes_bench.cpp:264-271).  Kernel classes:
 * 0 NTT phases (the row phases with an epilogue included), 1 ModUp (fused or not), 2 key inner
 * product (BSGS baby steps included), 3 ModDown (fused or not), 4 combine/automorphism,
 * 5 elementwise (tensor, add/sub, rescale steps), 6 Walsh S-box products and sums,
 * 7 BSGS giant-step sums. */
#define WG_KCLASS_NTT 0
#define WG_KCLASS_MODUP 1
#define WG_KCLASS_KEYMAC 2
#define WG_KCLASS_MODDOWN 3
#define WG_KCLASS_COMBINE 4
#define WG_KCLASS_ELEMENTWISE 5
#define WG_KCLASS_WALSH 6
#define WG_KCLASS_GIANT 7
/* Kernel launches issued so far for a class (kernel_class < 0: all classes). */
uint64_t wg_launch_count(int kernel_class);
/* Bracket each following launch of `kernel_class` (up to max_launches) with CUDA events on
 * its stream; wg_probe_end synchronises them and returns the launch count, the summed
 * device time in ms and the summed algorithmic bytes (each input residue read once, each
 * output written once). */
int wg_probe_begin(int kernel_class, int max_launches);
int wg_probe_end(uint64_t* launches, double* total_ms, double* total_bytes);

/* Host-side counters: out[0] slot encodings, out[1] their wall time (ns), out[2] staged
 * host-to-device uploads, out[3] their bytes, out[4] time spent waiting for staging space (ns).
 * Writes the first n of them. */
int wg_host_stats(uint64_t* out, size_t n);

/* Plain device-memory helpers for C callers without another allocator. */
int wg_malloc(void** ptr, size_t bytes);
int wg_free(void* ptr);
int wg_memcpy_htod(void* dst, const void* src, size_t bytes, void* stream);
int wg_memcpy_dtoh(void* dst, const void* src, size_t bytes, void* stream);
int wg_stream_synchronize(void* stream);

#ifdef __cplusplus
}
#endif
#endif /* WALSH_GPU_H */
