// Batched execution over many ciphertexts (wg_batch.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <array>
#include <vector>

#include "wg_bundle.hpp"
#include "wg_internal.hpp"

namespace wg {

// One key switch of a batch: b = (b_add ? b_in + ks_b : ks_b), a likewise, then the
// automorphism `galois` (0 = none) on both outputs.
struct KsItem {
    size_t level = 0;
    const uint64_t* key_term = nullptr;
    const KeyEntry* key = nullptr;
    const uint64_t* b_in = nullptr;
    const uint64_t* a_in = nullptr;
    uint64_t* b = nullptr;
    uint64_t* a = nullptr;
    int b_add = 1;
    int a_add = 0;
    uint64_t galois = 0;
};

// Host image of the job tables of one call; pointers returned by add() are byte offsets
// until upload() places the image in device memory, at() turns them into device pointers.
struct JobTable {
    std::vector<unsigned char> bytes;
    std::vector<size_t> offsets;
    void* base = nullptr;
    template <class J>
    const J* add(const std::vector<J>& v) {
        const size_t off = (bytes.size() + 15) & ~size_t{15};
        bytes.resize(off + v.size() * sizeof(J));
        if (!v.empty()) std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(J));
        offsets.push_back(off);
        return reinterpret_cast<const J*>(off);  // resolved against the device base by at()
    }
    template <class J>
    const J* at(const J* off) const {
        return reinterpret_cast<const J*>(static_cast<unsigned char*>(base) + reinterpret_cast<size_t>(off));
    }
    void upload(Context& c, cudaStream_t s);
};

size_t batch_keyswitch_words(const Context& c, const KsItem* items, size_t n);
void batch_keyswitch(Context& c, const KsItem* items, size_t n, cudaStream_t s);
void batch_mul_relin_rescale_rotate(Context& c, size_t count, const size_t* levels, uint64_t* const* xb,
                                    uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                                    const int64_t* rots, const uint64_t* galois, const KeyEntry* relin,
                                    const KeyEntry* const* rot_keys, cudaStream_t s);

// A batched mul + relin + rescale + rotate pipeline planned once for fixed buffers and captured
// as a CUDA graph: launching it replays every stage with no host-side planning or upload.  It
// owns its job table and scratch; the ciphertext buffers stay the caller's.
struct BatchGraph {
    uint64_t* d_jobs = nullptr;
    uint64_t* d_arena = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches[kClsCount] = {};
    ~BatchGraph();
};
BatchGraph* batch_graph_create(Context& c, size_t count, const size_t* levels, uint64_t* const* xb,
                               uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                               const uint64_t* galois, const KeyEntry* relin, const KeyEntry* const* rot_keys);
void batch_graph_launch(BatchGraph& g, cudaStream_t s);

// One baby-step / giant-step linear-transform stage (wg_bsgs.cu).
struct LtStage;
// diags == nullptr: allocate the diagonal store only (filled by the caller through lt_stage_data).
LtStage* lt_stage_create(Context& c, size_t level, size_t nterms, const uint64_t* indices, const uint64_t* diags,
                         size_t baby, size_t slots, bool rescale);
void lt_stage_destroy(LtStage* st);
uint64_t* lt_stage_data(LtStage& st);  // [term][QP limbs][N], Montgomery form
void lt_stage_set_plaintext_scale(LtStage& st, double scale);
// level, term count, baby steps, logical slots, rescale flag, plaintext scale (0 if not known)
void lt_stage_info(const LtStage& st, size_t& level, size_t& nterms, size_t& baby, size_t& slots, bool& rescale,
                   double& pt_scale);
const std::vector<size_t>& lt_stage_indices(const LtStage& st);
namespace dft {
struct Literal;
}
// The factorized DFT's stages generated and encoded on the context's device (wg_dftplan_dev.cu).
std::vector<LtStage*> dft_plan_create(Context& c, const dft::Literal& lit, cudaStream_t s);
void lt_stage_apply(Context& c, const LtStage& st, size_t count, uint64_t* const* b, uint64_t* const* a,
                    cudaStream_t s);

// Bootstrapping boundary steps (wg_boot.cu): ModRaise of level-0 ciphertexts to target_level,
// and the level-0 dense-to-sparse switch through q0 and p0 with the compact key.
void modraise(Context& c, size_t count, size_t target_level, uint64_t* const* b, uint64_t* const* a,
              cudaStream_t s);
void q0p0_switch(Context& c, size_t count, uint64_t* const* b, uint64_t* const* a, const KeyEntry& key,
                 cudaStream_t s);

// Chebyshev evaluation (wg_evalpoly.cu) of `count` ciphertexts sharing level and scale.
void evalchebyshev(Context& c, size_t count, size_t level, double scale, const double* coeffs, size_t ncoeffs,
                   double target_scale, double default_scale, uint64_t* const* b, uint64_t* const* a,
                   uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                   cudaStream_t s);

// EvalMod bootstrap of packed ciphertexts (wg_evalpoly.cu).
struct BootstrapParams {
    size_t s2c_depth = 0, depth = 0, evalmod_log_scale = 0, double_angle = 0, active_slots = 0, slots = 0;
    double scale = 0.0;
};
// A SlotToCoeff plan for inputs whose scale is `ratio` times the parameter scale.
struct S2cPlan {
    uint64_t ratio = 1;
    const LtStage* const* stages = nullptr;
    size_t n = 0;
};
size_t lt_stage_level(const LtStage& st);
// A stage's shape and diagonals (downloaded) for a bundle file.
void lt_stage_export(const Context& c, const LtStage& st, BundleStage& out);
bool lt_stage_rescales(const LtStage& st);
void bootstrap_evalmod(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans,
                       const LtStage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs, size_t count,
                       double in_scale, uint64_t* const* b, uint64_t* const* a, uint64_t* const* out0_b,
                       uint64_t* const* out0_a, uint64_t* const* out1_b, uint64_t* const* out1_a, size_t* out_level,
                       double* out_scale, cudaStream_t s);

// Mask-packed Walsh S-box over `count` instances (wg_sbox.cu); in/out are bit-major arrays of
// 8 * count ciphertext pointers.
// The AES S-box from the FIPS-197 definition (GF(2^8) inverse, then the affine map).
std::array<uint8_t, 256> aes_sbox_table();

// The XBOOT S-box (wg_xboot.cu) on `count` instances of 8 bit ciphertexts ([bit][instance]) at
// `level` and `scale`; outputs at out_level[bit] and out_scale[bit].
void xboot_sbox(Context& c, size_t count, size_t level, double scale, uint64_t* const* in_b, uint64_t* const* in_a,
                uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s);
// Integer coefficients of each S-box output bit over the 256 monomials of the input bits.
std::array<std::array<int64_t, 256>, 8> xboot_sbox_coefficients();

// ckks_batch_bootstrap_evalmod_inplace for `count` pairs at once (wg_xboot.cu): ct0 + i ct1
// labelled with `scale` (ct0's), bootstrapped; the two results overwrite (b0, a0) and (b1, a1),
// which hold s2c_depth + 1 limbs on entry and need room for depth + 1.
void bootstrap_pair(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                    size_t nc2s, const double* coeffs, size_t ncoeffs, size_t count, double scale, uint64_t* const* b0,
                    uint64_t* const* a0, uint64_t* const* b1, uint64_t* const* a1, size_t* out_level, double* out_scale,
                    cudaStream_t s);

// A rotation (kind WG_KEY_ROTATION), conjugation (WG_KEY_CONJ) or relinearisation
// (WG_KEY_RELIN) switching key of the secret
// `secret` (N ternary coefficients) generated on the device and installed in the context
// (wg_keygen.cu); mask a ([part][QP limb][N]) and noise e ([part][N]) from the caller, or drawn
// from `seed` when both are null; out_host (optional) receives the key as stored.
void keygen_switch_key(Context& c, int kind, int64_t rotation, const int8_t* secret, const uint64_t* a_host,
                       const int64_t* e_host, uint64_t seed, double sigma, uint64_t* out_host, cudaStream_t s);
// Secret-key encryption (ckks_encrypt_custom_eval) of `count` evaluation-form plaintexts at
// `level` under the ternary `secret` (wg_keygen.cu): b = pt + e - a s into out_b / out_a (level +
// 1 limbs each); mask a ([count][level+1][N]) and noise e ([count][N]) given, or drawn from
// `seed` when both are null.
void encrypt_symmetric(Context& c, size_t count, size_t level, const uint64_t* const* pts, const int8_t* secret,
                       const uint64_t* a_host, const int64_t* e_host, uint64_t seed, double sigma,
                       uint64_t* const* out_b, uint64_t* const* out_a, cudaStream_t s);
// ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks on the device (wg_aes.cu):
// the 1408 bits as (v, v) in the first active_blocks slots, rounds 1..9 at a quarter of the
// parameter scale, all at the S2C depth + 1; out_b / out_a need room for that level + 1 limbs.
void walsh_encrypt_round_key_bits(Context& c, const BootstrapParams& p, const uint8_t* expanded_key,
                                  size_t active_blocks, const int8_t* secret, uint64_t seed, double sigma,
                                  uint64_t* const* out_b, uint64_t* const* out_a, double* out_scale,
                                  size_t* out_level, cudaStream_t s);
// ckks_aes128_encrypt_expanded_round_key_bits on the device (wg_xboot.cu): the 1408 bits of the
// expanded key as constant-slot plaintexts at the parameter scale, encrypted under `secret` at
// the S2C depth (round 0: first_round_key_level above it); out_b / out_a need room for the
// level + 1 limbs of each bit.
void xboot_encrypt_round_key_bits(Context& c, const BootstrapParams& p, const uint8_t* expanded_key,
                                  size_t first_round_key_level, const int8_t* secret, uint64_t seed, double sigma,
                                  uint64_t* const* out_b, uint64_t* const* out_a, double* out_scale,
                                  size_t* out_level, cudaStream_t s);

// CKKS slot encoding of `count` slot vectors (re / im host arrays [count][N/2]) at `scale` into
// out[c] (limbs limbs), evaluation form when `eval`, else coefficient form (wg_encode_dev.cu).
void encode_slots_device(Context& c, size_t count, size_t limbs, double scale, const double* re, const double* im,
                         uint64_t* const* out, bool eval, cudaStream_t s);
// The same encoding into an arbitrary basis (modulus index per limb: Q moduli 0..nq-1, P moduli
// nq..), optionally converted to Montgomery form after the NTT.
void encode_slots_device_basis(Context& c, size_t count, const std::vector<int>& mods, double scale, const double* re,
                               const double* im, uint64_t* const* out, bool eval, bool montgomery, cudaStream_t s);
// ckks_decrypt on the device (wg_encode_dev.cu): slots of `count` ciphertexts at `level` (b, a
// and optional c2 per ciphertext; scales[k] each) under the ternary `secret`, into host arrays
// re / im [count][N/2].
void decrypt_decode_device(Context& c, size_t count, size_t level, const double* scales, const uint64_t* const* b,
                           const uint64_t* const* a, const uint64_t* const* c2, const int8_t* secret, double* re,
                           double* im, cudaStream_t s);
// The bootstrapping secret switches (wg_keygen.cu): WG_KEY_SPARSE_TO_DENSE as a hybrid key from
// `source` to `target`, WG_KEY_DENSE_TO_SPARSE as the compact level-0 key over (q0, p0).
void keygen_secret_switch(Context& c, int kind, const int8_t* source, const int8_t* target, const uint64_t* a_host,
                          const int64_t* e_host, uint64_t seed, double sigma, uint64_t* out_host, cudaStream_t s);

// AES-128-CTR on lazy bits with the XBOOT S-box and pair bootstraps (wg_xboot.cu).
struct XbootAesArgs {
    const uint64_t* const* key_b = nullptr;  // 1408 round-key bit ciphertexts
    const uint64_t* const* key_a = nullptr;
    const double* key_scales = nullptr;
    const size_t* key_levels = nullptr;
    const uint8_t* counters = nullptr;       // `blocks` public 16-byte blocks each
    const uint8_t* ciphertexts = nullptr;
    size_t blocks = 0;
    size_t pair_batch = 32;                  // pair bootstraps per batched call
};
void aes_ctr_xboot(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                   size_t nc2s, const double* coeffs, size_t ncoeffs, const XbootAesArgs& a, uint64_t* const* out_b,
                   uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s);
// Its steps on their own: the initial public XOR of the counter bits (key bits 0..127 of `a`,
// outputs with room for their level + 1 limbs), and ShiftRows + MixColumns (when `mix`) +
// AddRoundKey of 128 state bits at `level` with the key bits 0..127 of `a`.
void xboot_initial_state(Context& c, const BootstrapParams& p, const XbootAesArgs& a, uint64_t* const* out_b,
                         uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s);
void xboot_linear_layer(Context& c, size_t level, const double* in_scale, uint64_t* const* in_b,
                        uint64_t* const* in_a, const XbootAesArgs& a, bool mix, uint64_t* const* out_b,
                        uint64_t* const* out_a, double* out_scale, cudaStream_t s);

void walsh_sbox(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                size_t nc2s, const double* coeffs, size_t ncoeffs, size_t block_count, size_t count, size_t level,
                double scale, uint64_t* const* in_b, uint64_t* const* in_a, uint64_t* const* out_b,
                uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s);

// AES-128-CTR on lazy bits with the mask-packed Walsh S-box (wg_aes.cu).
struct AesArgs {
    const uint64_t* const* key_b = nullptr;  // 1408 round-key bit ciphertexts at key_level
    const uint64_t* const* key_a = nullptr;
    const double* key_scales = nullptr;
    size_t key_level = 0;
    const uint8_t* counters = nullptr;       // 2 * active_blocks blocks of 16 bytes
    const uint8_t* ciphertexts = nullptr;
    size_t active_blocks = 0;
    size_t packing_block_count = 0, packed_segment_count = 0;
    // the reference's call granularity: each S-box instance and each refresh bootstrap as its
    // own call (the plain per-operation path; same words as the batched one)
    bool per_instance = false;
};
void aes_ctr_walsh(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                   size_t nc2s, const double* coeffs, size_t ncoeffs, const AesArgs& args, uint64_t* const* out_b,
                   uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s);

// Hoisted rotations of one ciphertext; out [rotation][b, a][level+1][N] (wg_bsgs.cu).
void rotate_many(Context& c, size_t level, const uint64_t* b, const uint64_t* a, const int64_t* rots, size_t nrot,
                 uint64_t* out, cudaStream_t s);
// ... for `count` ciphertexts at once; outs[i] as `out` above for ciphertext i.
void rotate_many_batch(Context& c, size_t level, size_t count, const uint64_t* const* bs, const uint64_t* const* as,
                       const int64_t* rots, size_t nrot, uint64_t* const* outs, cudaStream_t s);

}  // namespace wg
