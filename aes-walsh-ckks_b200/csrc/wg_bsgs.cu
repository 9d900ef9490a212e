// Baby-step / giant-step linear transform in the QP domain (one CoeffToSlot or SlotToCoeff
// stage), batched over ciphertexts that share the stage's diagonals.
//
// Reference: ckks_apply_linear_transform_owned_stage_qp,
// src/ckks/operations/bootstrap/ckks_linear_transform.cpp:1174-1407, with its helpers
// make_direct_input_qp :487, ckks_hybrid_key_switch_hoisted_qp_rotated (ckks_keyswitch.cpp:675),
// multiply_qp_plaintext_accumulate_pair :418, moddown_qp_poly_to_q_eval :581,
// ckks_hybrid_key_switch_qp_from_key_term (ckks_keyswitch.cpp:854),
// automorphism_qp_pair_accumulate :373 and moddown_qp_pair_to_q_eval :641.
//
// Per stage, for a batch of C ciphertexts at level l (L = l+1 Q limbs, T = L+K QP limbs):
//   1. hoist a: iNTT, HPS ModUp per digit, NTT                       (one launch per step)
//   2. baby steps in QP: baby 0 = (a, b) with zero P limbs; baby r = key inner product of the
//      hoisted digits with the rotation-r key, b added on the Q limbs, automorphism applied
//      by scattering each coefficient to its rotated slot                (one launch)
//   3. giant inner sums: sum over the giant's diagonals of REDC(baby * diagonal), all
//      ciphertexts in the same thread so each diagonal word is read once per batch
//   4. giants g >= 1: single ModDown of the inner a (alpha as multiply + add, like the
//      reference's single-polynomial ModDown), then a QP key switch of that key term with
//      the rotation-(g * baby) key (no ModDown)
//   5. accumulate: out = inner_0 + sum_g automorphism_g(switch_g + (0, inner_g.b))
//   6. pair ModDown of out (alpha fused), optional rescale.
// Every addition is an exact modular addition of canonical residues, so the order of
// accumulation (raw sums with periodic reduction in the reference) does not change any word.
#include <algorithm>
#include <map>

#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_internal.hpp"
#include "wg_keyswitch.cuh"

namespace wg {
using namespace bk;

struct LtStage {
    size_t level = 0;
    size_t nterms = 0;
    size_t baby = 0;
    size_t slots = 0;
    bool rescale = false;
    double pt_scale = 0.0;       // plaintext scale of the diagonals (0: not known)
    std::vector<size_t> indices;
    uint64_t* d_diag = nullptr;  // [term][QP limbs][N], Montgomery form
    ~LtStage() { cudaFree(d_diag); }
};

uint64_t* lt_stage_data(LtStage& st) { return st.d_diag; }
void lt_stage_set_plaintext_scale(LtStage& st, double scale) { st.pt_scale = scale; }
void lt_stage_info(const LtStage& st, size_t& level, size_t& nterms, size_t& baby, size_t& slots, bool& rescale,
                   double& pt_scale) {
    level = st.level;
    nterms = st.nterms;
    baby = st.baby;
    slots = st.slots;
    rescale = st.rescale;
    pt_scale = st.pt_scale;
}
const std::vector<size_t>& lt_stage_indices(const LtStage& st) { return st.indices; }

namespace {


// Baby rotation `slot` of QP limb i for ciphertexts [c0, c0 + nc) of the batch: the key words
// of a coefficient are loaded once and used for every ciphertext of the group.
struct BabyJob {
    const uint64_t* key;
    uint64_t galois_inv;
    int key_level, i, slot, c0, nc, pad;
};

struct CtRef {
    const uint64_t* a;
    const uint64_t* b;
};

struct CopyPair {
    uint64_t* dst;
    const uint64_t* src;
};

constexpr int kGiantBatch = 8;  // ciphertexts per thread in the baby-step kernel (key words reused)

struct TermRef {
    const uint64_t* diag;  // QP plaintext of the term (limb 0)
    int slot;              // baby slot
    int g;                 // giant step within its group
};

constexpr int kGiantGroup = 8;  // giant steps accumulated per thread

// One ciphertext, one QP limb, a group of up to kGiantGroup giant steps: terms
// [term0, term0 + nterms) of the term table, sorted by baby slot, so every baby-step value is
// loaded once for all giant steps of the group.
struct GiantJob {
    const uint64_t* babies;  // batch base: [C][slots][2][T][N]
    uint64_t* inner;         // batch base: [C][giants][2][T][N]
    int term0, nterms, i, g0, ng, c;
};

struct SubJob {
    const uint64_t* x;
    const uint64_t* y;
    uint64_t* out;
    int mod;
    int pad;
};

struct GiantInfo {
    uint64_t galois;  // automorphism of the giant rotation (0 for giant 0)
    int g;
    int pad;
};

struct AccumJob {
    const uint64_t* inner;   // this ciphertext's [giants][2][T][N]
    const uint64_t* sw;      // this ciphertext's switch outputs [giants][2][T][N] (g >= 1 used)
    uint64_t* out;           // [2][T][N]
    int ngiants, i, pad0, pad1;
};

// NC (the ciphertexts of the job) is a compile-time count so that every digit load of a part is
// unconditional and all of them are in flight at once.
template <int NC>
__device__ __forceinline__ void baby_step(const BabyJob* j, const CtRef* __restrict__ cts,
                                          const uint64_t* __restrict__ digits, uint64_t* __restrict__ babies,
                                          const Modulus* mods, int nq, int L, int K, int parts, int alpha,
                                          int nslots, int logN) {
    const size_t N = size_t{1} << logN;
    const uint32_t x = blockIdx.x * kT + threadIdx.x;
    const int i = j->i;
    const int T = L + K;
    const bool is_p = i >= L;
    const Modulus& m = mods[is_p ? nq + (i - L) : i];
    const uint64_t q = m.q, qninv = m.qninv;
    const size_t key_limbs = (size_t)j->key_level + 1 + K;
    const size_t klimb = is_p ? (size_t)j->key_level + 1 + (i - L) : (size_t)i;
    const size_t part_stride = (size_t)T * N;
    const size_t limb = (size_t)i * N + x;
    const CtRef* ct = cts + j->c0;
    uint64_t acc_a[NC], acc_b[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        acc_a[c] = 0;
        acc_b[c] = is_p ? 0 : ct[c].b[limb];
    }
    for (int p = 0; p < parts; ++p) {
        const int s0 = p * alpha, s1 = s0 + alpha < L ? s0 + alpha : L;
        const bool own = !is_p && i >= s0 && i < s1;  // source limb: the key term itself
        const uint64_t ka = j->key[(((size_t)p * 2 + 0) * key_limbs + klimb) * N + x];
        const uint64_t kb = j->key[(((size_t)p * 2 + 1) * key_limbs + klimb) * N + x];
        uint64_t d[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c)
            d[c] = own ? ct[c].a[limb] : digits[((size_t)(j->c0 + c) * parts + p) * part_stride + limb];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            acc_a[c] = add_mod(acc_a[c], mont_mul(d[c], ka, q, qninv), q);
            acc_b[c] = add_mod(acc_b[c], mont_mul(d[c], kb, q, qninv), q);
        }
    }
    const uint32_t dst = automorphism_src(x, j->galois_inv, logN);
    const size_t slot_words = 2 * (size_t)T * N;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        uint64_t* o = babies + ((size_t)(j->c0 + c) * nslots + j->slot) * slot_words + (size_t)i * N;
        o[dst] = acc_a[c];
        o[(size_t)T * N + dst] = acc_b[c];
    }
}

__global__ void __launch_bounds__(kT, 3) kb_baby(const BabyJob* jobs, int n, const CtRef* __restrict__ cts,
                                                 const uint64_t* __restrict__ digits, uint64_t* __restrict__ babies,
                                                 const Modulus* mods, int nq, int L, int K, int parts, int alpha,
                                                 int nslots, int logN) {
    const BabyJob* j = job_of(jobs, n);
    if (!j) return;
    static_assert(kGiantBatch == 8, "one case per batch size");
#define WG_BABY(NC) baby_step<NC>(j, cts, digits, babies, mods, nq, L, K, parts, alpha, nslots, logN)
    switch (j->nc) {  // the same for every thread of the block
        case 1: WG_BABY(1); break;
        case 2: WG_BABY(2); break;
        case 3: WG_BABY(3); break;
        case 4: WG_BABY(4); break;
        case 5: WG_BABY(5); break;
        case 6: WG_BABY(6); break;
        case 7: WG_BABY(7); break;
        default: WG_BABY(8); break;
    }
#undef WG_BABY
}

// Adds one term's products to the accumulator pair of its giant step.  g is the same for every
// thread of the block (one job per block), so this is a uniform branch to that pair; the
// accumulators keep constant indices and stay in registers.
__device__ __forceinline__ void giant_add(int g, uint64_t pa, uint64_t pb, uint64_t q, uint64_t* acc_a,
                                          uint64_t* acc_b) {
    static_assert(kGiantGroup == 8, "one case per giant step of a group");
    switch (g) {
#define WG_GIANT_ADD(G)                          \
    case G:                                      \
        acc_a[G] = add_mod(acc_a[G], pa, q);     \
        acc_b[G] = add_mod(acc_b[G], pb, q);     \
        break;
        WG_GIANT_ADD(0)
        WG_GIANT_ADD(1)
        WG_GIANT_ADD(2)
        WG_GIANT_ADD(3)
        WG_GIANT_ADD(4)
        WG_GIANT_ADD(5)
        WG_GIANT_ADD(6)
        WG_GIANT_ADD(7)
#undef WG_GIANT_ADD
        default:
            break;
    }
}

// Giant-step inner sums: inner[c][g] = sum over the terms (g, slot) of diag x baby[c][slot], in
// QP.  Montgomery products and modular additions of canonical residues, so the order of the
// terms does not change the canonical sums.
// The terms go kGiantUnroll at a time: their table entries, then all their diagonal and baby-step
// words, then the products, so each warp has that many HBM loads in flight rather than one
// dependent chain per term (a baby-step word shared by consecutive terms is read again from L1).
constexpr int kGiantUnroll = 4;

__global__ void __launch_bounds__(kT, 3) kb_giant(const GiantJob* jobs, int n, const TermRef* __restrict__ term_table,
                                                  const Modulus* mods, int nq, int L, int T, int nslots, int ngiants,
                                                  size_t N) {
    const GiantJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t x = (size_t)blockIdx.x * kT + threadIdx.x;
    const int i = j->i;
    const Modulus& m = mods[i < L ? i : nq + (i - L)];
    const uint64_t q = m.q, qninv = m.qninv;
    const size_t limb = (size_t)i * N + x;
    const size_t slot_words = 2 * (size_t)T * N;
    uint64_t acc_a[kGiantGroup], acc_b[kGiantGroup];
#pragma unroll
    for (int g = 0; g < kGiantGroup; ++g) acc_a[g] = acc_b[g] = 0;
    const uint64_t* babies = j->babies + (size_t)j->c * nslots * slot_words + limb;
    const TermRef* terms = term_table + j->term0;
    const int nterms = j->nterms;
    int t = 0;
    for (; t + kGiantUnroll <= nterms; t += kGiantUnroll) {
        TermRef tr[kGiantUnroll];
        uint64_t d[kGiantUnroll], ba[kGiantUnroll], bb[kGiantUnroll];
#pragma unroll
        for (int u = 0; u < kGiantUnroll; ++u) tr[u] = terms[t + u];
#pragma unroll
        for (int u = 0; u < kGiantUnroll; ++u) {
            const uint64_t* bs = babies + (size_t)tr[u].slot * slot_words;
            d[u] = tr[u].diag[limb];
            ba[u] = bs[0];
            bb[u] = bs[(size_t)T * N];
        }
#pragma unroll
        for (int u = 0; u < kGiantUnroll; ++u)
            giant_add(tr[u].g, mont_mul(ba[u], d[u], q, qninv), mont_mul(bb[u], d[u], q, qninv), q, acc_a, acc_b);
    }
    for (; t < nterms; ++t) {
        const TermRef tr = terms[t];
        const uint64_t* bs = babies + (size_t)tr.slot * slot_words;
        const uint64_t d = tr.diag[limb];
        giant_add(tr.g, mont_mul(bs[0], d, q, qninv), mont_mul(bs[(size_t)T * N], d, q, qninv), q, acc_a, acc_b);
    }
#pragma unroll
    for (int g = 0; g < kGiantGroup; ++g) {
        if (g >= j->ng) break;
        uint64_t* o = j->inner + ((size_t)j->c * ngiants + j->g0 + g) * slot_words;
        o[limb] = acc_a[g];
        o[(size_t)T * N + limb] = acc_b[g];
    }
}

__global__ void __launch_bounds__(kT) kb_moddown_single(const ModDownJob* jobs, int n, const Modulus* mods, int nq,
                                                        int K, size_t N) {
    const ModDownJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t coeff = (size_t)blockIdx.x * kT + threadIdx.x;
    moddown_all_limbs<false>(mods, nq, j->L, K, j->src_p, N, coeff, j->inv, j->inv_s, j->out);
}

__global__ void __launch_bounds__(kT) kb_sub(const SubJob* jobs, int n, const Modulus* mods) {
    const SubJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    j->out[k] = sub_mod(j->x[k], j->y[k], mods[j->mod].q);
}

__global__ void __launch_bounds__(kT) kb_accumulate(const AccumJob* jobs, int n, const GiantInfo* __restrict__ giants,
                                                    const Modulus* mods, int nq, int L, int T, int logN) {
    const AccumJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t N = size_t{1} << logN;
    const uint32_t x = blockIdx.x * kT + threadIdx.x;
    const int i = j->i;
    const uint64_t q = mods[i < L ? i : nq + (i - L)].q;
    const size_t slot_words = 2 * (size_t)T * N;
    const size_t limb = (size_t)i * N;
    uint64_t oa = 0, ob = 0;
    for (int k = 0; k < j->ngiants; ++k) {
        const GiantInfo gi = giants[k];
        const uint64_t* in = j->inner + (size_t)gi.g * slot_words;
        if (gi.galois == 0) {
            oa = add_mod(oa, in[limb + x], q);
            ob = add_mod(ob, in[(size_t)T * N + limb + x], q);
        } else {
            const uint32_t s = automorphism_src(x, gi.galois, logN);
            const uint64_t* sw = j->sw + (size_t)gi.g * slot_words;
            oa = add_mod(oa, sw[limb + s], q);
            ob = add_mod(ob, add_mod(sw[(size_t)T * N + limb + s], in[(size_t)T * N + limb + s], q), q);
        }
    }
    j->out[limb + x] = oa;
    j->out[(size_t)T * N + limb + x] = ob;
}

}  // namespace

void lt_stage_export(const Context& c, const LtStage& st, BundleStage& out) {
    out.level = st.level;
    out.baby = st.baby;
    out.slots = st.slots;
    out.rescale = st.rescale ? 1 : 0;
    out.indices.assign(st.indices.begin(), st.indices.end());
    out.diagonals.resize(st.nterms * (st.level + 1 + c.np) * c.N);
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    check_cuda(cudaMemcpy(out.diagonals.data(), st.d_diag, out.diagonals.size() * 8, cudaMemcpyDeviceToHost),
               "linear transform: diagonal download");
}

size_t lt_stage_level(const LtStage& st) { return st.level; }
bool lt_stage_rescales(const LtStage& st) { return st.rescale; }

LtStage* lt_stage_create(Context& c, size_t level, size_t nterms, const uint64_t* indices, const uint64_t* diags,
                         size_t baby, size_t slots, bool rescale) {
    if (level >= c.nq) fail(kInvalid, "ckks_linear_transform: invalid stage level");
    if (nterms == 0) fail(kInvalid, "ckks_linear_transform: empty stage");
    const size_t full = c.N / 2;
    if (slots == 0) slots = full;
    if (slots > full || full % slots || (slots & (slots - 1)))
        fail(kInvalid, "ckks_linear_transform: invalid logical stage slot count");
    if (baby == 0 || baby > slots) fail(kInvalid, "ckks_linear_transform: invalid compiled stage input");
    for (size_t t = 0; t < nterms; ++t)
        if (indices[t] >= slots) fail(kInvalid, "ckks_linear_transform: diagonal index out of range");
    auto st = std::make_unique<LtStage>();
    st->level = level;
    st->nterms = nterms;
    st->baby = baby;
    st->slots = slots;
    st->rescale = rescale;
    st->indices.assign(indices, indices + nterms);
    const size_t words = nterms * (level + 1 + c.np) * c.N;
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    if (cudaMalloc(&st->d_diag, words * 8) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "linear transform: diagonal allocation failed");
    }
    if (diags) check_cuda(cudaMemcpy(st->d_diag, diags, words * 8, cudaMemcpyHostToDevice), "upload diagonals");
    return st.release();
}

void lt_stage_destroy(LtStage* st) { delete st; }

// Rotation keys a stage needs: baby rotations 1..baby-1 and giant rotations g * baby.
static void stage_rotations(const LtStage& st, std::vector<size_t>& babies, std::vector<size_t>& giants,
                            std::vector<std::vector<size_t>>& terms_by_giant) {
    std::vector<char> baby_needed(st.baby, 0);
    const size_t ngiants = (st.slots + st.baby - 1) / st.baby;
    terms_by_giant.assign(ngiants, {});
    for (size_t t = 0; t < st.nterms; ++t) {
        baby_needed[st.indices[t] % st.baby] = 1;
        terms_by_giant[st.indices[t] / st.baby].push_back(t);
    }
    babies.clear();
    giants.clear();
    for (size_t r = 0; r < st.baby; ++r)
        if (baby_needed[r]) babies.push_back(r);
    for (size_t g = 0; g < ngiants; ++g)
        if (!terms_by_giant[g].empty()) giants.push_back(g);
}

void lt_stage_apply(Context& c, const LtStage& st, size_t count, uint64_t* const* b, uint64_t* const* a,
                    cudaStream_t s) {
    if (count == 0) return;
    const size_t N = c.N, level = st.level, L = level + 1, K = c.np, T = L + K, nq = c.nq;
    const size_t B = c.parts_at(level);
    const size_t slots_full = N / 2;
    std::vector<size_t> babies, giants;
    std::vector<std::vector<size_t>> terms_by_giant;
    stage_rotations(st, babies, giants, terms_by_giant);
    auto rot_key = [&](size_t r) -> const KeyEntry& {
        const int64_t rr = (int64_t)(r % slots_full);
        if (rr == 0) fail(kInvalid, "ckks_linear_transform: zero rotation");
        auto it = c.keys.find({WG_KEY_ROTATION, rr});
        if (it == c.keys.end()) fail(kInvalid, "ckks_linear_transform: missing baby-step or giant-step rotation key");
        if (it->second.key_level < level || it->second.parts < B) fail(kRuntime, "keyswitch: unusable rotation key");
        return it->second;
    };
    auto galois_of = [&](size_t r) { return host::powmod(5, (uint64_t)(r % slots_full), 2 * N); };
    // Slot of each needed baby value and the giants with terms.
    std::map<size_t, int> slot_of;
    for (size_t k = 0; k < babies.size(); ++k) slot_of[babies[k]] = (int)k;
    const size_t ns = babies.size(), ng = giants.size();
    std::map<size_t, int> gidx;
    for (size_t k = 0; k < ng; ++k) gidx[giants[k]] = (int)k;

    // Arena layout.
    const size_t w_coeff = count * L * N;
    const size_t w_digits = count * B * T * N;
    const size_t w_babies = count * ns * 2 * T * N;
    const size_t w_inner = count * ng * 2 * T * N;
    const size_t w_csingle = count * ng * L * N;
    const size_t w_coeff2 = count * ng * L * N;
    const size_t w_digits2 = count * ng * B * T * N;
    const size_t w_switch = count * ng * 2 * T * N;
    const size_t w_out = count * 2 * T * N;
    const size_t w_cfinal = count * 2 * L * N;
    const size_t w_rem = count * 2 * L * N;
    uint64_t* base = c.batch_buffers(s).arena(c, w_coeff + w_digits + w_babies + w_inner + w_csingle + w_coeff2 +
                                                     w_digits2 + w_switch + w_out + w_cfinal + w_rem, s);
    uint64_t* coeff = base;
    uint64_t* digits = coeff + w_coeff;
    uint64_t* babybuf = digits + w_digits;
    uint64_t* inner = babybuf + w_babies;
    uint64_t* csingle = inner + w_inner;
    uint64_t* coeff2 = csingle + w_csingle;
    uint64_t* digits2 = coeff2 + w_coeff2;
    uint64_t* sw = digits2 + w_digits2;
    uint64_t* out = sw + w_switch;
    uint64_t* cfinal = out + w_out;
    uint64_t* rem = cfinal + w_cfinal;
    const size_t slotw = 2 * T * N;
    auto modq = [&](size_t limb) { return (int)(limb < L ? limb : nq + (limb - L)); };

    JobTable t;
    // 1. hoist
    const bool fused = c.fuse(2 * count);  // the pair ModDown launch: two jobs per ciphertext
    int max_src = 1;
    for (size_t j = 0; j < B; ++j) max_src = std::max(max_src, c.modup[level][j].src_count);
    std::vector<NttJob> intt_a, ntt_dig;
    std::vector<ModUpJob> modup;
    for (size_t ci = 0; ci < count; ++ci) {
        uint64_t* cf = coeff + ci * L * N;
        uint64_t* dg = digits + ci * B * T * N;
        for (size_t l = 0; l < L; ++l) intt_a.push_back({a[ci] + l * N, cf + l * N, (int)l, 0});
        for (size_t j = 0; j < B; ++j) {
            modup.push_back({c.d_modup + level * c.dnum + j, cf, dg + j * T * N});
            const size_t s0 = j * c.alpha, s1 = std::min(s0 + c.alpha, L);
            for (size_t l = 0; l < T; ++l)
                if (l < s0 || l >= s1) ntt_dig.push_back({dg + j * T * N + l * N, dg + j * T * N + l * N, modq(l), 0});
        }
    }
    // 2. babies: baby 0 as a copy (P limbs zeroed below), others by MAC + scatter
    std::vector<BabyJob> baby_jobs;
    std::vector<CtRef> ct_refs;
    for (size_t ci = 0; ci < count; ++ci) ct_refs.push_back({a[ci], b[ci]});
    const bool baby0 = !babies.empty() && babies[0] == 0;
    // limb-outer, baby-step-inner: the blocks of consecutive jobs read the same hoisted digit
    // limbs (one ciphertext group's, limb i) with different keys, so the digits come from HBM
    // once per stage instead of once per baby step
    std::vector<const KeyEntry*> baby_keys(ns, nullptr);
    std::vector<uint64_t> baby_ginv(ns, 0);
    for (size_t k = 0; k < ns; ++k) {
        if (babies[k] == 0) continue;
        baby_keys[k] = &rot_key(babies[k]);
        baby_ginv[k] = host::powmod(galois_of(babies[k]), N - 1, 2 * N);
    }
    for (size_t i = 0; i < T; ++i)
        for (size_t c0 = 0; c0 < count; c0 += kGiantBatch)
            for (size_t k = 0; k < ns; ++k) {
                if (!baby_keys[k]) continue;
                baby_jobs.push_back({baby_keys[k]->d_data, baby_ginv[k], (int)baby_keys[k]->key_level, (int)i, (int)k,
                                     (int)c0, (int)std::min<size_t>(kGiantBatch, count - c0), 0});
            }
    // 3. giant sums
    std::vector<TermRef> terms;
    std::vector<GiantJob> giant_jobs;
    const size_t qp_words = T * N;
    for (size_t g0 = 0; g0 < ng; g0 += kGiantGroup) {
        const size_t gn = std::min<size_t>(kGiantGroup, ng - g0);
        std::vector<TermRef> group;
        for (size_t gk = g0; gk < g0 + gn; ++gk)
            for (size_t term : terms_by_giant[giants[gk]])
                group.push_back({st.d_diag + term * qp_words, slot_of[st.indices[term] % st.baby], (int)(gk - g0)});
        std::stable_sort(group.begin(), group.end(), [](const TermRef& x, const TermRef& y) { return x.slot < y.slot; });
        const size_t off = terms.size();
        terms.insert(terms.end(), group.begin(), group.end());
        // limb-outer, ciphertext-inner: the blocks of consecutive jobs read the same diagonal
        // words (this group's terms on limb i), so each diagonal limb comes from HBM once per
        // batch and from L2 for the other ciphertexts
        for (size_t i = 0; i < T; ++i)
            for (size_t ci = 0; ci < count; ++ci)
                giant_jobs.push_back({babybuf, inner, (int)off, (int)group.size(), (int)i, (int)g0, (int)gn, (int)ci});
    }
    // 4. giants >= 1: single ModDown of inner a, then QP key switch from that key term
    std::vector<NttJob> intt_pg, ntt_cs, intt_kt, ntt_dig2;
    std::vector<NttEpiJob> cs_epi, cf_epi;
    std::vector<ModDownJob> md_single;
    std::vector<SubJob> kt_sub;
    std::vector<ModUpJob> modup2;
    std::vector<MacGroupJob> mac2;
    for (size_t ci = 0; ci < count; ++ci)
        for (size_t gk = 0; gk < ng; ++gk) {
            if (giants[gk] == 0) continue;
            const KeyEntry& key = rot_key(giants[gk] * st.baby);
            uint64_t* in_a = inner + (ci * ng + gk) * slotw;
            uint64_t* cs = csingle + (ci * ng + gk) * L * N;
            for (size_t pi = 0; pi < K; ++pi) {
                uint64_t* p = in_a + (L + pi) * N;
                intt_pg.push_back({p, p, (int)(nq + pi), 0});
            }
            md_single.push_back({in_a + L * N, cs, c.fold_inv[level], c.fold_inv_s[level], (int)L, 0});
            for (size_t qi = 0; qi < L; ++qi) {
                if (fused) {
                    // key term = inner a - ModDown: the subtraction as the row phase's epilogue
                    cs_epi.push_back({cs + qi * N, in_a + qi * N, nullptr, in_a + qi * N, 0, 0, (int)qi, kEpiCombine});
                } else {
                    ntt_cs.push_back({cs + qi * N, cs + qi * N, (int)qi, 0});
                    kt_sub.push_back({in_a + qi * N, cs + qi * N, in_a + qi * N, (int)qi, 0});
                }
            }
            uint64_t* cf2 = coeff2 + (ci * ng + gk) * L * N;
            uint64_t* dg2 = digits2 + (ci * ng + gk) * B * T * N;
            uint64_t* acc = sw + (ci * ng + gk) * slotw;
            for (size_t l = 0; l < L; ++l) intt_kt.push_back({in_a + l * N, cf2 + l * N, (int)l, 0});
            for (size_t j = 0; j < B; ++j) {
                modup2.push_back({c.d_modup + level * c.dnum + j, cf2, dg2 + j * T * N});
                const size_t s0 = j * c.alpha, s1 = std::min(s0 + c.alpha, L);
                for (size_t l = 0; l < T; ++l)
                    if (l < s0 || l >= s1)
                        ntt_dig2.push_back({dg2 + j * T * N + l * N, dg2 + j * T * N + l * N, modq(l), 0});
            }
        }
    // the giant's key inner products, up to kMacGroup ciphertexts per job so each key word is
    // loaded once for all of them
    double mac2_bytes = 0.0;
    for (size_t gk = 0; gk < ng; ++gk) {
        if (giants[gk] == 0) continue;
        const KeyEntry& key = rot_key(giants[gk] * st.baby);
        for (size_t c0 = 0; c0 < count; c0 += kMacGroup) {
            const size_t n = std::min<size_t>(kMacGroup, count - c0);
            for (size_t i = 0; i < T; ++i) {
                MacGroupJob jb{};
                jb.key = key.d_data;
                jb.part_stride = T * N;
                jb.L = (int)L;
                jb.K = (int)K;
                jb.parts = (int)B;
                jb.alpha = (int)c.alpha;
                jb.key_level = (int)key.key_level;
                jb.i = (int)i;
                jb.n = (int)n;
                for (size_t k = 0; k < n; ++k) {
                    const size_t slot = (c0 + k) * ng + gk;
                    jb.key_term[k] = inner + slot * slotw;
                    jb.digits[k] = digits2 + slot * B * T * N;
                    jb.acc[k] = sw + slot * slotw;
                }
                mac2.push_back(jb);
            }
            mac2_bytes += 8.0 * N * T * (2.0 * B + (double)n * (B + 2.0));
        }
    }
    // 5. accumulation
    std::vector<GiantInfo> ginfo;
    for (size_t gk = 0; gk < ng; ++gk)
        ginfo.push_back({giants[gk] == 0 ? 0 : galois_of(giants[gk] * st.baby), (int)gk, 0});
    std::vector<AccumJob> accum;
    for (size_t ci = 0; ci < count; ++ci)
        for (size_t i = 0; i < T; ++i)
            accum.push_back({inner + ci * ng * slotw, sw + ci * ng * slotw, out + ci * slotw, (int)ng, (int)i, 0, 0});
    // 6. pair ModDown, then into the ciphertext (and rescale)
    std::vector<NttJob> intt_po, ntt_cf;
    std::vector<ModDownJob> md_pair;
    std::vector<SubJob> final_sub;
    for (size_t ci = 0; ci < count; ++ci) {
        for (int poly = 0; poly < 2; ++poly) {
            uint64_t* o = out + ci * slotw + poly * T * N;
            uint64_t* cf = cfinal + (ci * 2 + poly) * L * N;
            for (size_t pi = 0; pi < K; ++pi) intt_po.push_back({o + (L + pi) * N, o + (L + pi) * N, (int)(nq + pi), 0});
            md_pair.push_back({o + L * N, cf, c.fold_inv[level], c.fold_inv_s[level], (int)L, 0});
            uint64_t* dst = poly ? b[ci] : a[ci];  // out holds a at offset 0, b at T*N
            for (size_t qi = 0; qi < L; ++qi) {
                if (fused) {
                    cf_epi.push_back({cf + qi * N, o + qi * N, nullptr, dst + qi * N, 0, 0, (int)qi, kEpiCombine});
                    continue;
                }
                ntt_cf.push_back({cf + qi * N, cf + qi * N, (int)qi, 0});
                final_sub.push_back({o + qi * N, cf + qi * N, dst + qi * N, (int)qi, 0});
            }
        }
    }
    RescaleJobs rescale_jobs;
    if (st.rescale) {
        if (level == 0) fail(kInvalid, "ckks_rescale: invalid level");
        for (size_t ci = 0; ci < count; ++ci)
            for (int poly = 0; poly < 2; ++poly)
                rescale_jobs.add(poly ? a[ci] : b[ci], level, rem + (ci * 2 + poly) * level * N);
    }

    // Baby slot 0 holds (a, b) with zero P limbs: copy Q limbs, clear P limbs.
    for (size_t ci = 0; ci < count && baby0; ++ci) {
        uint64_t* slot = babybuf + (ci * ns + 0) * slotw;
        check_cuda(cudaMemcpyAsync(slot, a[ci], L * N * 8, cudaMemcpyDeviceToDevice, s), "baby 0");
        check_cuda(cudaMemcpyAsync(slot + T * N, b[ci], L * N * 8, cudaMemcpyDeviceToDevice, s), "baby 0");
        check_cuda(cudaMemsetAsync(slot + L * N, 0, K * N * 8, s), "baby 0");
        check_cuda(cudaMemsetAsync(slot + T * N + L * N, 0, K * N * 8, s), "baby 0");
    }

    const NttJob* j_intt_a = t.add(intt_a);
    const ModUpJob* j_modup = t.add(modup);
    const NttJob* j_ntt_dig = t.add(ntt_dig);
    const BabyJob* j_baby = t.add(baby_jobs);
    const CtRef* j_cts = t.add(ct_refs);
    const TermRef* j_terms = t.add(terms);
    const GiantJob* j_giant = t.add(giant_jobs);
    const NttJob* j_intt_pg = t.add(intt_pg);
    const ModDownJob* j_mds = t.add(md_single);
    const NttJob* j_ntt_cs = t.add(ntt_cs);
    const SubJob* j_kt_sub = t.add(kt_sub);
    const NttJob* j_intt_kt = t.add(intt_kt);
    const ModUpJob* j_modup2 = t.add(modup2);
    const NttJob* j_ntt_dig2 = t.add(ntt_dig2);
    const MacGroupJob* j_mac2 = t.add(mac2);
    const GiantInfo* j_ginfo = t.add(ginfo);
    const AccumJob* j_accum = t.add(accum);
    const NttJob* j_intt_po = t.add(intt_po);
    const ModDownJob* j_mdp = t.add(md_pair);
    const NttJob* j_ntt_cf = t.add(ntt_cf);
    const SubJob* j_final = t.add(final_sub);
    const NttEpiJob* j_cs_epi = t.add(cs_epi);
    const NttEpiJob* j_cf_epi = t.add(cf_epi);
    rescale_jobs.plan(c, t);
    t.upload(c, s);
    // 1.
    if (fused) {
        // inverse row phase, [inverse columns, ModUp, forward columns], forward row phase
        ntt_jobs_phase(c, t.at(j_intt_a), (int)intt_a.size(), false, false, s);
        modup_ntt_jobs(c, t.at(j_modup), (int)modup.size(), max_src, 8.0 * N * (double)(count * B * T), s);
        ntt_jobs_phase(c, t.at(j_ntt_dig), (int)ntt_dig.size(), true, false, s);
    } else {
        ntt_jobs(c, t.at(j_intt_a), (int)intt_a.size(), false, s);
        {
            Probe probe(kClsModUp, 8.0 * N * (double)(count * B * T), s);
            kb_modup<<<grid_for(c, modup.size()), kT, 0, s>>>(t.at(j_modup), (int)modup.size(), c.d_mod, N);
        }
        ntt_jobs(c, t.at(j_ntt_dig), (int)ntt_dig.size(), true, s);
    }
    // 2.
    if (!baby_jobs.empty()) {
        double bytes = 0;
        for (const BabyJob& bj : baby_jobs) bytes += 8.0 * N * (2.0 * B + bj.nc * (B + 3.0));
        Probe probe(kClsKeyMac, bytes, s);
        kb_baby<<<grid_for(c, baby_jobs.size()), kT, 0, s>>>(t.at(j_baby), (int)baby_jobs.size(), t.at(j_cts), digits,
                                                             babybuf, c.d_mod, (int)nq, (int)L, (int)K, (int)B,
                                                             (int)c.alpha, (int)ns, c.logN);
    }
    // 3.
    {
        Probe probe(kClsGiant, 8.0 * N * (double)(st.nterms * T + count * (ns + ng) * 2 * T), s);
        kb_giant<<<grid_for(c, giant_jobs.size()), kT, 0, s>>>(t.at(j_giant), (int)giant_jobs.size(), t.at(j_terms),
                                                               c.d_mod, (int)nq, (int)L, (int)T, (int)ns, (int)ng, N);
    }
    // 4.
    if (!md_single.empty() && fused) {
        ntt_jobs_phase(c, t.at(j_intt_pg), (int)intt_pg.size(), false, false, s);
        moddown_ntt_jobs(c, t.at(j_mds), (int)md_single.size(), 8.0 * N * (K + L) * md_single.size(), s, false);
        ntt_rows_epilogue_jobs(c, t.at(j_cs_epi), (int)cs_epi.size(), ntt_epilogue_bytes(cs_epi, N), s);
        ntt_jobs_phase(c, t.at(j_intt_kt), (int)intt_kt.size(), false, false, s);
        modup_ntt_jobs(c, t.at(j_modup2), (int)modup2.size(), max_src, 8.0 * N * (double)(md_single.size() * B * T),
                       s);
        ntt_jobs_phase(c, t.at(j_ntt_dig2), (int)ntt_dig2.size(), true, false, s);
        Probe probe(kClsKeyMac, mac2_bytes, s);
        kb_mac_group<<<grid_for(c, mac2.size()), kT, 0, s>>>(t.at(j_mac2), (int)mac2.size(), c.d_mod, (int)nq, N);
    } else if (!md_single.empty()) {
        ntt_jobs(c, t.at(j_intt_pg), (int)intt_pg.size(), false, s);
        {
            Probe probe(kClsModDown, 8.0 * N * (K + L) * md_single.size(), s);
            kb_moddown_single<<<grid_for(c, md_single.size()), kT, 0, s>>>(t.at(j_mds), (int)md_single.size(),
                                                                           c.d_mod, (int)nq, (int)K, N);
        }
        ntt_jobs(c, t.at(j_ntt_cs), (int)ntt_cs.size(), true, s);
        {
            Probe probe(kClsElementwise, 8.0 * N * 3.0 * kt_sub.size(), s);
            kb_sub<<<grid_for(c, kt_sub.size()), kT, 0, s>>>(t.at(j_kt_sub), (int)kt_sub.size(), c.d_mod);
        }
        ntt_jobs(c, t.at(j_intt_kt), (int)intt_kt.size(), false, s);
        {
            Probe probe(kClsModUp, 8.0 * N * (double)(md_single.size() * B * T), s);
            kb_modup<<<grid_for(c, modup2.size()), kT, 0, s>>>(t.at(j_modup2), (int)modup2.size(), c.d_mod, N);
        }
        ntt_jobs(c, t.at(j_ntt_dig2), (int)ntt_dig2.size(), true, s);
        Probe probe(kClsKeyMac, mac2_bytes, s);
        kb_mac_group<<<grid_for(c, mac2.size()), kT, 0, s>>>(t.at(j_mac2), (int)mac2.size(), c.d_mod, (int)nq, N);
    }
    // 5.
    {
        Probe probe(kClsCombine, 8.0 * N * (double)(count * (2 * ng + 1) * 2 * T), s);
        kb_accumulate<<<grid_for(c, accum.size()), kT, 0, s>>>(t.at(j_accum), (int)accum.size(), t.at(j_ginfo),
                                                               c.d_mod, (int)nq, (int)L, (int)T, c.logN);
    }
    // 6.
    if (fused) {
        ntt_jobs_phase(c, t.at(j_intt_po), (int)intt_po.size(), false, false, s);
        moddown_ntt_jobs(c, t.at(j_mdp), (int)md_pair.size(), 8.0 * N * (K + L) * md_pair.size(), s);
        ntt_rows_epilogue_jobs(c, t.at(j_cf_epi), (int)cf_epi.size(), ntt_epilogue_bytes(cf_epi, N), s);
    } else {
        ntt_jobs(c, t.at(j_intt_po), (int)intt_po.size(), false, s);
        {
            Probe probe(kClsModDown, 8.0 * N * (K + L) * md_pair.size(), s);
            kb_moddown<<<grid_for(c, md_pair.size()), kT, 0, s>>>(t.at(j_mdp), (int)md_pair.size(), c.d_mod,
                                                                  (int)nq, (int)K, N);
        }
        ntt_jobs(c, t.at(j_ntt_cf), (int)ntt_cf.size(), true, s);
        {
            Probe probe(kClsElementwise, 8.0 * N * 3.0 * final_sub.size(), s);
            kb_sub<<<grid_for(c, final_sub.size()), kT, 0, s>>>(t.at(j_final), (int)final_sub.size(), c.d_mod);
        }
    }
    rescale_jobs.run(c, t, s);
    check_cuda(cudaGetLastError(), "linear transform launch");
}

// Hoisted rotations of one ciphertext (ckks_hoist_ciphertext_a_qp_eval + per rotation
// ckks_hybrid_key_switch_hoisted_inplace, ckks_keyswitch.cpp:344-373 and 1072-1328): the
// iNTT / ModUp / NTT of `a` is done once; each rotation then costs a key inner product, a
// pair ModDown, the combine and the automorphism, all rotations batched per step.
// out: [rotation][b, a][level+1][N].
void rotate_many(Context& c, size_t level, const uint64_t* b, const uint64_t* a, const int64_t* rots, size_t nrot,
                 uint64_t* out, cudaStream_t s) {
    rotate_many_batch(c, level, 1, &b, &a, rots, nrot, &out, s);
}

// The same for `count` ciphertexts at one level, every step one launch over all of them:
// out[i] receives ciphertext i's rotations, [rotation][b, a][level+1][N].
void rotate_many_batch(Context& c, size_t level, size_t count, const uint64_t* const* bs, const uint64_t* const* as,
                       const int64_t* rots, size_t nrot, uint64_t* const* outs, cudaStream_t s) {
    if (nrot == 0 || count == 0) return;
    const size_t N = c.N, L = level + 1, K = c.np, T = L + K, nq = c.nq;
    const size_t B = c.parts_at(level);
    const size_t slots = N / 2;
    std::vector<const KeyEntry*> keys(nrot, nullptr);
    std::vector<uint64_t> gal(nrot, 0);
    for (size_t r = 0; r < nrot; ++r) {
        int64_t rr = rots[r] % (int64_t)slots;
        if (rr < 0) rr += (int64_t)slots;
        if (rr == 0) continue;
        const KeyEntry& k = c.key(WG_KEY_ROTATION, rr);
        if (k.key_level < level) fail(kRuntime, "keyswitch: switch key level is below ciphertext level");
        if (k.parts < B) fail(kRuntime, "keyswitch: insufficient key partitions");
        keys[r] = &k;
        gal[r] = host::powmod(5, (uint64_t)rr, 2 * N);
    }
    const size_t w_coeff = L * N, w_digits = B * T * N, w_acc = nrot * 2 * T * N, w_contrib = nrot * 2 * L * N;
    const size_t per_ct = w_coeff + w_digits + w_acc + w_contrib;
    uint64_t* arena = c.batch_buffers(s).arena(c, count * per_ct, s);
    auto modq = [&](size_t limb) { return (int)(limb < L ? limb : nq + (limb - L)); };

    const bool fused = c.fuse(count * B);  // the ModUp launch: one job per digit
    int max_src = 1;
    for (size_t j = 0; j < B; ++j) max_src = std::max(max_src, c.modup[level][j].src_count);
    std::vector<NttJob> intt_a, ntt_dig, intt_p, ntt_c;
    std::vector<NttEpiJob> c_epi;
    std::vector<ModUpJob> modup;
    std::vector<MacJob> mac;
    std::vector<ModDownJob> md;
    std::vector<CombineJob> comb;
    std::vector<GatherJob> gath;
    std::vector<CopyPair> copies;
    for (size_t ci = 0; ci < count; ++ci) {
        const uint64_t* b = bs[ci];
        const uint64_t* a = as[ci];
        uint64_t* out = outs[ci];
        uint64_t* coeff = arena + ci * per_ct;
        uint64_t* digits = coeff + w_coeff;
        uint64_t* accb = digits + w_digits;
        uint64_t* contrib = accb + w_acc;
        for (size_t l = 0; l < L; ++l) intt_a.push_back({a + l * N, coeff + l * N, (int)l, 0});
        for (size_t j = 0; j < B; ++j) {
            modup.push_back({c.d_modup + level * c.dnum + j, coeff, digits + j * T * N});
            const size_t s0 = j * c.alpha, s1 = std::min(s0 + c.alpha, L);
            for (size_t l = 0; l < T; ++l)
                if (l < s0 || l >= s1)
                    ntt_dig.push_back({digits + j * T * N + l * N, digits + j * T * N + l * N, modq(l), 0});
        }
        for (size_t r = 0; r < nrot; ++r) {
            uint64_t* ob = out + (2 * r) * L * N;
            uint64_t* oa = ob + L * N;
            if (!keys[r]) {  // rotation by a multiple of the slot count: the ciphertext itself
                copies.push_back({ob, b});
                copies.push_back({oa, a});
                continue;
            }
            uint64_t* acc = accb + r * 2 * T * N;
            uint64_t* cr = contrib + r * 2 * L * N;
            for (size_t i = 0; i < T; ++i)
                mac.push_back({keys[r]->d_data, a, digits, acc, T * N, (int)L, (int)K, (int)B, (int)c.alpha,
                               (int)keys[r]->key_level, (int)i});
            for (int poly = 0; poly < 2; ++poly) {
                for (size_t pi = 0; pi < K; ++pi) {
                    uint64_t* p = acc + (poly * T + L + pi) * N;
                    intt_p.push_back({p, p, (int)(nq + pi), 0});
                }
                md.push_back({acc + (poly * T + L) * N, cr + poly * L * N, c.fold_inv[level], c.fold_inv_s[level],
                              (int)L, 0});
                if (!fused)
                    for (size_t qi = 0; qi < L; ++qi)
                        ntt_c.push_back({cr + (poly * L + qi) * N, cr + (poly * L + qi) * N, (int)qi, 0});
            }
            for (size_t qi = 0; qi < L; ++qi) {
                // combine in place of the accumulators, then gather into the output slot
                if (fused) {
                    c_epi.push_back({cr + qi * N, acc + qi * N, nullptr, acc + qi * N, 0, 0, (int)qi, kEpiCombine});
                    c_epi.push_back({cr + (L + qi) * N, acc + (T + qi) * N, b + qi * N, acc + (T + qi) * N, 1, 0,
                                     (int)qi, kEpiCombine});
                } else {
                    comb.push_back({acc, cr, b, a, acc + T * N, acc, (int)L, (int)K, (int)qi, 1, 0, 0});
                }
                gath.push_back({acc + T * N + qi * N, acc + qi * N, ob + qi * N, oa + qi * N, gal[r]});
            }
        }
    }
    for (const CopyPair& cp : copies)
        check_cuda(cudaMemcpyAsync(cp.dst, cp.src, L * N * 8, cudaMemcpyDeviceToDevice, s), "rotate_many copy");
    JobTable t;
    const NttJob* j1 = t.add(intt_a);
    const ModUpJob* j2 = t.add(modup);
    const NttJob* j3 = t.add(ntt_dig);
    const MacJob* j4 = t.add(mac);
    const NttJob* j5 = t.add(intt_p);
    const ModDownJob* j6 = t.add(md);
    const NttJob* j7 = t.add(ntt_c);
    const CombineJob* j8 = t.add(comb);
    const GatherJob* j9 = t.add(gath);
    const NttEpiJob* j10 = t.add(c_epi);
    t.upload(c, s);
    double modup_bytes = 0;
    for (size_t j = 0; j < B; ++j) modup_bytes += 8.0 * N * (c.modup[level][j].src_count + c.modup[level][j].dst_count);
    modup_bytes *= count;
    if (fused) {
        ntt_jobs_phase(c, t.at(j1), (int)intt_a.size(), false, false, s);
        modup_ntt_jobs(c, t.at(j2), (int)modup.size(), max_src, modup_bytes, s);
        ntt_jobs_phase(c, t.at(j3), (int)ntt_dig.size(), true, false, s);
    } else {
        ntt_jobs(c, t.at(j1), (int)intt_a.size(), false, s);
        {
            Probe probe(kClsModUp, modup_bytes, s);
            kb_modup<<<grid_for(c, modup.size()), kT, 0, s>>>(t.at(j2), (int)modup.size(), c.d_mod, N);
        }
        ntt_jobs(c, t.at(j3), (int)ntt_dig.size(), true, s);
    }
    if (!mac.empty()) {
        {
            Probe probe(kClsKeyMac, 8.0 * N * mac.size() * (3.0 * B + 2.0), s);
            kb_mac<<<grid_for(c, mac.size()), kT, 0, s>>>(t.at(j4), (int)mac.size(), c.d_mod, (int)nq, N);
        }
        if (fused) {
            ntt_jobs_phase(c, t.at(j5), (int)intt_p.size(), false, false, s);
            moddown_ntt_jobs(c, t.at(j6), (int)md.size(), 8.0 * N * (K + L) * md.size(), s);
            ntt_rows_epilogue_jobs(c, t.at(j10), (int)c_epi.size(), ntt_epilogue_bytes(c_epi, N), s);
            Probe probe(kClsCombine, 8.0 * N * 4.0 * gath.size(), s);
            kb_gather<<<grid_for(c, gath.size()), kT, 0, s>>>(t.at(j9), (int)gath.size(), c.logN);
        } else {
            ntt_jobs(c, t.at(j5), (int)intt_p.size(), false, s);
            {
                Probe probe(kClsModDown, 8.0 * N * (K + L) * md.size(), s);
                kb_moddown<<<grid_for(c, md.size()), kT, 0, s>>>(t.at(j6), (int)md.size(), c.d_mod, (int)nq, (int)K,
                                                                 N);
            }
            ntt_jobs(c, t.at(j7), (int)ntt_c.size(), true, s);
            Probe probe(kClsCombine, 8.0 * N * L * 12.0 * (mac.size() / T), s);
            kb_combine<<<grid_for(c, comb.size()), kT, 0, s>>>(t.at(j8), (int)comb.size(), c.d_mod, N);
            kb_gather<<<grid_for(c, gath.size()), kT, 0, s>>>(t.at(j9), (int)gath.size(), c.logN);
        }
    }
    check_cuda(cudaGetLastError(), "rotate_many launch");
}

}  // namespace wg
