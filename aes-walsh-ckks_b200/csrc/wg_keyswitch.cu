// Hybrid key switching on the device: iNTT -> HPS ModUp -> NTT -> Montgomery key MAC ->
// P-limb iNTT -> folded HPS ModDown -> NTT -> combine (+ optional automorphism).
//
// Reference: ckks_hybrid_key_switch_inplace, src/ckks/operations/keyswitch/ckks_keyswitch.cpp:
// 1330-1641, with folded keys in Montgomery form (the reference defaults).  Each stage is one
// launch that covers every limb and every digit of the switch, so a switch costs a fixed
// number of launches regardless of level or dnum.
//
// Workspace layout for level l (L = l+1 Q limbs, K P limbs, T = L+K, B digits):
//   coeff   [L][N]      coefficient-domain copy of the key term
//   digits  [B][T][N]   ModUp output per digit (source limbs left unused)
//   acc     [2][T][N]   key inner products for a (0) and b (1)
//   contrib [2][L][N]   ModDown contributions
#include <algorithm>

#include "wg_internal.hpp"
#include "wg_keyswitch.cuh"

namespace wg {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxParts = 16;

struct ModUpBatch {
    ModUpDesc d[kMaxParts];
};

__global__ void __launch_bounds__(kThreads)
    k_modup(ModUpBatch batch, const Modulus* __restrict__ mods, const uint64_t* __restrict__ src,
            uint64_t* __restrict__ digits, size_t part_stride, size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    const int part = blockIdx.y;
    modup_coeff(batch.d[part], mods, src, digits + part * part_stride, N, coeff);
}

__global__ void __launch_bounds__(kThreads)
    k_key_mac(const Modulus* __restrict__ mods, int nq, int L, int K, int parts, int alpha,
              const uint64_t* __restrict__ key, int key_level, const uint64_t* __restrict__ key_term,
              const uint64_t* __restrict__ digits, size_t part_stride, uint64_t* __restrict__ acc, size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    mac_coeff(mods, nq, L, K, parts, alpha, key, key_level, key_term, digits, part_stride, acc, N, blockIdx.y, coeff);
}

__global__ void __launch_bounds__(kThreads)
    k_moddown(const Modulus* __restrict__ mods, int nq, int L, int K, const uint64_t* __restrict__ acc,
              const uint64_t* __restrict__ inv, const uint64_t* __restrict__ inv_s,
              uint64_t* __restrict__ contrib, size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    const int poly = blockIdx.y;
    const int T = L + K;
    const uint64_t* src_p = acc + ((size_t)poly * T + L) * N;
    moddown_all_limbs(mods, nq, L, K, src_p, N, coeff, inv, inv_s, contrib + (size_t)poly * L * N);
}

// Combine; written in place of acc when an automorphism follows (so the gather reads a
// stable buffer), else straight to the outputs.
__global__ void __launch_bounds__(kThreads)
    k_combine(const Modulus* __restrict__ mods, int L, int K, uint64_t* acc, const uint64_t* __restrict__ contrib,
              const uint64_t* b_in, const uint64_t* a_in, uint64_t* b_out, uint64_t* a_out, int b_add, int a_add,
              size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    const int qi = blockIdx.y;
    combine_coeff(mods[qi].q, L, K, acc, contrib, b_in, a_in, b_out, a_out, b_add, a_add, N, qi, coeff);
}

__global__ void __launch_bounds__(kThreads)
    k_gather_pair(const uint64_t* __restrict__ src_b, const uint64_t* __restrict__ src_a,
                  uint64_t* __restrict__ b, uint64_t* __restrict__ a, uint64_t galois, int logN) {
    const size_t N = size_t{1} << logN;
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    const size_t off = (size_t)blockIdx.y * N;
    const uint32_t s = automorphism_src(i, galois, logN);
    b[off + i] = src_b[off + s];
    a[off + i] = src_a[off + s];
}

}  // namespace

size_t keyswitch_workspace_words(const Context& c, size_t level) {
    const size_t L = level + 1, T = L + c.np, B = c.parts_at(level);
    return c.N * (L + B * T + 2 * T + 2 * L);
}

void keyswitch(const Context& c, size_t level, const uint64_t* key_term, const KeyEntry& k, const uint64_t* b_in,
               const uint64_t* a_in, uint64_t* b, uint64_t* a, bool b_add, bool a_add, uint64_t galois,
               uint64_t* ws, cudaStream_t s) {
    const size_t N = c.N, L = level + 1, K = c.np, T = L + K;
    const size_t B = c.parts_at(level);
    if (level >= c.nq) fail(kInvalid, "keyswitch: invalid ciphertext level");
    if (k.key_level < level) fail(kRuntime, "keyswitch: switch key level is below ciphertext level");
    if (k.parts < B) fail(kRuntime, "keyswitch: insufficient key partitions");
    if (B > (size_t)kMaxParts || c.alpha > (size_t)kMaxDigitWidth || K > (size_t)kMaxPLimbs)
        fail(kInvalid, "keyswitch: parameter set exceeds kernel limits");

    uint64_t* coeff = ws;
    uint64_t* digits = coeff + L * N;
    uint64_t* acc = digits + B * T * N;
    uint64_t* contrib = acc + 2 * T * N;
    const dim3 blk(kThreads);
    const unsigned gx = (unsigned)(N / kThreads);

    // 1. key term to coefficient form.
    check_cuda(cudaMemcpyAsync(coeff, key_term, L * N * 8, cudaMemcpyDeviceToDevice, s), "keyswitch copy");
    ntt_inverse(c, coeff, (int)L, 1, 0, LimbMap{(int)L, 0, 0}, s);

    // 2. ModUp of every digit.
    ModUpBatch batch;
    for (size_t j = 0; j < B; ++j) batch.d[j] = c.modup[level][j];
    {
        size_t words = 0;  // each digit reads its source limbs and writes every other QP limb
        for (size_t j = 0; j < B; ++j) words += (size_t)(c.modup[level][j].src_count + c.modup[level][j].dst_count) * N;
        Probe probe(kClsModUp, 8.0 * words, s);
        k_modup<<<dim3(gx, (unsigned)B), blk, 0, s>>>(batch, c.d_mod, coeff, digits, T * N, N);
    }

    // 3. Forward NTT of every ModUp output limb: per digit, the Q limbs after the digit and
    //    the P limbs form one contiguous run, the Q limbs before it another.
    for (size_t j = 0; j < B; ++j) {
        const size_t s0 = j * c.alpha, s1 = std::min(s0 + c.alpha, L);
        uint64_t* dj = digits + j * T * N;
        if (s0 > 0) ntt_forward(c, dj, (int)s0, 1, 0, LimbMap{(int)s0, 0, 0}, s);
        ntt_forward(c, dj + s1 * N, (int)(T - s1), 1, 0, LimbMap{(int)(L - s1), (int)s1, (int)c.nq}, s);
    }

    // 4. Key inner product over digits, all QP limbs.
    {
        // per QP limb: B digit limbs + 2B key limbs read, 2 accumulator limbs written
        Probe probe(kClsKeyMac, 8.0 * N * T * (3.0 * B + 2.0), s);
        k_key_mac<<<dim3(gx, (unsigned)T), blk, 0, s>>>(c.d_mod, (int)c.nq, (int)L, (int)K, (int)B, (int)c.alpha,
                                                        k.d_data, (int)k.key_level, key_term, digits, T * N, acc, N);
    }

    // 5. P limbs of both accumulators back to coefficient form.
    ntt_inverse(c, acc + L * N, (int)K, 2, T * N, LimbMap{0, 0, (int)c.nq}, s);

    // 6. Folded ModDown contributions, then to evaluation form.
    {
        Probe probe(kClsModDown, 8.0 * N * 2.0 * (K + L), s);
        k_moddown<<<dim3(gx, 2), blk, 0, s>>>(c.d_mod, (int)c.nq, (int)L, (int)K, acc,
                                                            c.fold_inv[level], c.fold_inv_s[level], contrib, N);
    }
    ntt_forward(c, contrib, (int)L, 2, L * N, LimbMap{(int)L, 0, 0}, s);

    // 7. Combine (and apply the automorphism for rotations).
    if (galois == 0) {
        Probe probe(kClsCombine, 8.0 * N * L * (b_add + a_add + 6.0), s);
        k_combine<<<dim3(gx, (unsigned)L), blk, 0, s>>>(c.d_mod, (int)L, (int)K, acc, contrib, b_in, a_in, b, a,
                                                         b_add, a_add, N);
    } else {
        uint64_t* tb = acc + (size_t)T * N;  // b result staged in place of acc_b
        uint64_t* ta = acc;
        {
            Probe probe(kClsCombine, 8.0 * N * L * (b_add + a_add + 6.0), s);
            k_combine<<<dim3(gx, (unsigned)L), blk, 0, s>>>(c.d_mod, (int)L, (int)K, acc, contrib, b_in, a_in, tb, ta,
                                                             b_add, a_add, N);
        }
        Probe probe(kClsCombine, 8.0 * N * L * 4.0, s);
        k_gather_pair<<<dim3(gx, (unsigned)L), blk, 0, s>>>(tb, ta, b, a, galois, c.logN);
    }
    check_cuda(cudaGetLastError(), "keyswitch launch");
}

}  // namespace wg
