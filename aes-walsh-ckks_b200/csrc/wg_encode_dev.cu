// CKKS slot encoding on the device (FP64), batched over plaintexts.
//
// Reference: ckks_encode / encode_slots_custom_basis, src/ckks/encoding/ckks_encoding.cpp:332-414
// (Hermitian embedding :29-43, the DIF transform of src/math/fft/fft.cpp:36-97, the slot
// permutation of src/ckks/context/ckks_context.cpp:56-68).  The coefficients are
// llrint(Re(FFT) * scale / N) and the FFT's rounding decides the coefficients next to a
// rounding boundary, so every operation is the host encoder's (wg_encode.cpp) one for one: the
// same tables (computed on the host by that encoder), the butterfly sums as separate roundings,
// the twiddle product as fma(a, c, -(b d)) and fma(a, d, b c) in IEEE double with explicit
// round-to-nearest intrinsics (no contraction), and the same final multiply and llrint.  Each
// IEEE operation is correctly rounded on both sides, so the device values equal the host's.
//
// One launch per DIF stage over all plaintexts of the batch (log2 N launches): the transform is
// a few MB per plaintext and bound by memory traffic; the stages with strides below 2048 could
// run in shared memory, which matters only for far larger batches than the AES circuits use.
//
// Decryption and decoding (ckks_decrypt, ckks_encoding.cpp:89-171, 567-575) run the other way:
// m = b + a s per limb, inverse NTT, the coefficients' signed values, then the conjugate
// transpose of the encoder's transform (its stages in reverse order, each butterfly transposed,
// twiddles conjugated), divided by the scale, read at the slot permutation.  The signed value of
// a coefficient comes from its residues mod q0 and q1 (Garner's two-modulus CRT, exact while
// |m| < q0 q1 / 2, which decryptable messages are far below) instead of the reference's CRT over
// all limbs in long double, and the transform is a different FP64 evaluation order, so decoded
// values agree with the reference's to FP64 rounding (about 1e-15 relative), not bit for bit.
#include <stdexcept>
#include <vector>

#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_encode.hpp"
#include "wg_internal.hpp"

namespace wg {
using namespace bk;

namespace {

// ev[c][perm[i]] = slot i, ev[c][N - 1 - perm[i]] = its conjugate
__global__ void __launch_bounds__(kT) kb_embed(const double* __restrict__ re, const double* __restrict__ im,
                                               const uint32_t* __restrict__ perm, double2* __restrict__ ev,
                                               size_t N, size_t count) {
    const size_t half = N >> 1;
    const size_t t = (size_t)blockIdx.x * kT + threadIdx.x;
    if (t >= count * half) return;
    const size_t c = t / half, i = t % half;
    const double vr = re[t], vi = im[t];
    const size_t d = perm[i];
    ev[c * N + d] = make_double2(vr, vi);
    ev[c * N + N - 1 - d] = make_double2(vr, -vi);
}

// one DIF stage: blocks of 2k, twiddle tw[m + i] for block i (m = N / 2k)
__global__ void __launch_bounds__(kT) kb_dif_stage(double2* __restrict__ ev, const double2* __restrict__ tw,
                                                   size_t N, size_t count, size_t m, size_t k) {
    const size_t half = N >> 1;
    const size_t t = (size_t)blockIdx.x * kT + threadIdx.x;
    if (t >= count * half) return;
    const size_t c = t / half, u = t % half;
    const size_t i = u / k, j = u % k;
    double2* x0 = ev + c * N + 2 * i * k + j;
    double2* x1 = x0 + k;
    const double2 a = *x0, b = *x1, w = tw[m + i];
    *x0 = make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
    const double dr = __dsub_rn(a.x, b.x), di = __dsub_rn(a.y, b.y);
    *x1 = make_double2(__fma_rn(dr, w.x, -__dmul_rn(di, w.y)), __fma_rn(dr, w.y, __dmul_rn(di, w.x)));
}

struct EncodeOutJob {
    uint64_t* out;  // limb of plaintext c
    int c, mod;
};

// out[i] = llrint(Re(ev[c][i]) * s) mod q
__global__ void __launch_bounds__(kT) kb_encode_out(const EncodeOutJob* jobs, int n, const double2* __restrict__ ev,
                                                    double s, size_t N, const Modulus* mods) {
    const EncodeOutJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t i = (size_t)blockIdx.x * kT + threadIdx.x;
    const int64_t q = (int64_t)mods[j->mod].q;
    const int64_t v = llrint(__dmul_rn(ev[(size_t)j->c * N + i].x, s));
    const int64_t r = v % q;
    j->out[i] = (uint64_t)(r + (q & (r >> 63)));
}

struct DecryptJob {
    uint64_t* m;          // out: b + a s (+ c2 s^2), this limb
    const uint64_t* b;
    const uint64_t* a;
    const uint64_t* c2;   // null for two-polynomial ciphertexts
    const uint64_t* s;    // secret limb (evaluation form)
    int mod, pad;
};

__global__ void __launch_bounds__(kT) kb_decrypt(const DecryptJob* jobs, int n, const Modulus* mods) {
    const DecryptJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const Modulus m = mods[j->mod];
    const uint64_t q = m.q, sv = j->s[k];
    uint64_t v = add_mod(barrett_mul(j->a[k], sv, m), j->b[k], q);
    if (j->c2) v = add_mod(v, barrett_mul(j->c2[k], barrett_mul(sv, sv, m), m), q);
    j->m[k] = v;
}

struct SecretLimbJob {
    const int8_t* src;
    uint64_t* dst;
    int mod, pad;
};

__global__ void __launch_bounds__(kT) kb_secret_to_limb(const SecretLimbJob* jobs, int n, const Modulus* mods) {
    const SecretLimbJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q = mods[j->mod].q;
    const int v = j->src[k];
    j->dst[k] = v >= 0 ? (uint64_t)v % q : (q - (uint64_t)(-v) % q) % q;
}

// signed coefficient values from limbs 0 (and 1): ev[c][i] = (value, 0)
__global__ void __launch_bounds__(kT) kb_signed_coeffs(const uint64_t* __restrict__ m, size_t N, size_t count,
                                                       size_t limbs, uint64_t q0, uint64_t q1, uint64_t q0_inv_q1,
                                                       double2* __restrict__ ev) {
    const size_t t = (size_t)blockIdx.x * kT + threadIdx.x;
    if (t >= count * N) return;
    const size_t c = t / N, i = t % N;
    const uint64_t r0 = m[(c * limbs) * N + i];
    double v;
    if (limbs == 1) {
        v = r0 > (q0 >> 1) ? -(double)(q0 - r0) : (double)r0;
    } else {
        const uint64_t r1 = m[(c * limbs + 1) * N + i];
        const uint64_t r0m = r0 % q1;
        const uint64_t d = r1 >= r0m ? r1 - r0m : r1 + q1 - r0m;
        const uint64_t tq = (uint64_t)(((unsigned __int128)d * q0_inv_q1) % q1);
        const unsigned __int128 x = (unsigned __int128)r0 + (unsigned __int128)q0 * tq;  // in [0, q0 q1)
        const unsigned __int128 Q = (unsigned __int128)q0 * q1;
        const bool neg = x > (Q >> 1);
        const unsigned __int128 mag = neg ? Q - x : x;
        const double dv = (double)(uint64_t)(mag >> 64) * 0x1p64 + (double)(uint64_t)mag;
        v = neg ? -dv : dv;
    }
    ev[t] = make_double2(v, 0.0);
}

// one stage of the transposed transform: (x0, x1) -> (x0 + conj(w) x1, x0 - conj(w) x1)
__global__ void __launch_bounds__(kT) kb_dit_stage(double2* __restrict__ ev, const double2* __restrict__ tw,
                                                   size_t N, size_t count, size_t m, size_t k) {
    const size_t half = N >> 1;
    const size_t t = (size_t)blockIdx.x * kT + threadIdx.x;
    if (t >= count * half) return;
    const size_t c = t / half, u = t % half;
    const size_t i = u / k, j = u % k;
    double2* x0 = ev + c * N + 2 * i * k + j;
    double2* x1 = x0 + k;
    const double2 a = *x0, b = *x1, w = tw[m + i];
    // b * conj(w)
    const double pr = b.x * w.x + b.y * w.y, pi = b.y * w.x - b.x * w.y;
    *x0 = make_double2(a.x + pr, a.y + pi);
    *x1 = make_double2(a.x - pr, a.y - pi);
}

// slot i of plaintext c = ev[c][perm[i]] / scale[c]
__global__ void __launch_bounds__(kT) kb_extract_slots(const double2* __restrict__ ev, const uint32_t* __restrict__ perm,
                                                       const double* __restrict__ scale, size_t N, size_t count,
                                                       double* __restrict__ re, double* __restrict__ im) {
    const size_t half = N >> 1;
    const size_t t = (size_t)blockIdx.x * kT + threadIdx.x;
    if (t >= count * half) return;
    const size_t c = t / half, i = t % half;
    const double2 v = ev[c * N + perm[i]];
    re[t] = v.x / scale[c];
    im[t] = v.y / scale[c];
}

// x = x * (2^64 mod q) with the Barrett product, limb by limb (the Montgomery form of the
// reference's precomputed plaintexts, ckks_convert_plaintext_to_montgomery_inplace,
// src/ckks/encoding/ckks_encoding.cpp:177-194).
struct MontJob {
    uint64_t* x;
    uint64_t r;  // 2^64 mod q
    int mod, pad;
};

__global__ void __launch_bounds__(kT) kb_to_montgomery(const MontJob* jobs, int n, const Modulus* mods) {
    const MontJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    j->x[k] = barrett_mul(j->x[k], j->r, mods[j->mod]);
}

}  // namespace

void encode_slots_device(Context& c, size_t count, size_t limbs, double scale, const double* re, const double* im,
                         uint64_t* const* out, bool eval, cudaStream_t s) {
    if (limbs == 0 || limbs > c.nq) throw std::invalid_argument("ckks_encode: invalid level");
    std::vector<int> mods(limbs);
    for (size_t l = 0; l < limbs; ++l) mods[l] = (int)l;
    encode_slots_device_basis(c, count, mods, scale, re, im, out, eval, false, s);
}

void encode_slots_device_basis(Context& c, size_t count, const std::vector<int>& mods, double scale, const double* re,
                               const double* im, uint64_t* const* out, bool eval, bool montgomery, cudaStream_t s) {
    if (count == 0) return;
    if (!(scale > 0.0)) throw std::invalid_argument("ckks_encode: scale must be positive");
    const size_t limbs = mods.size();
    if (limbs == 0) throw std::invalid_argument("ckks_encode: invalid level");
    for (int m : mods)
        if (m < 0 || m >= (int)(c.nq + c.np)) throw std::invalid_argument("ckks_encode: invalid modulus index");
    if (!re || !im) throw std::invalid_argument("ckks_encode: null slot values");
    const size_t N = c.N, half = N >> 1;
    std::vector<double> tw;
    std::vector<uint32_t> perm;
    host::encode_tables(N, tw, perm);
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    // scratch: twiddles [N] double2, permutation [N/2] u32, slot values [2][count][N/2], the
    // transform [count][N] double2
    const size_t bytes = N * 16 + half * 4 + 2 * count * half * 8 + count * N * 16 + 256;
    unsigned char* ws = nullptr;
    if (cudaMallocAsync((void**)&ws, bytes, s) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "ckks_encode: scratch allocation failed");
    }
    auto* dtw = reinterpret_cast<double2*>(ws);
    auto* dev = dtw + N;
    auto* dre = reinterpret_cast<double*>(dev + count * N);
    auto* dim = dre + count * half;
    auto* dperm = reinterpret_cast<uint32_t*>(dim + count * half);
    try {
        check_cuda(cudaMemcpyAsync(dtw, tw.data(), N * 16, cudaMemcpyHostToDevice, s), "encode upload");
        check_cuda(cudaMemcpyAsync(dperm, perm.data(), half * 4, cudaMemcpyHostToDevice, s), "encode upload");
        check_cuda(cudaMemcpyAsync(dre, re, count * half * 8, cudaMemcpyHostToDevice, s), "encode upload");
        check_cuda(cudaMemcpyAsync(dim, im, count * half * 8, cudaMemcpyHostToDevice, s), "encode upload");
        const unsigned grid = (unsigned)((count * half + kT - 1) / kT);
        kb_embed<<<grid, kT, 0, s>>>(dre, dim, dperm, dev, N, count);
        for (size_t m = half, k = 1; m > 0; m >>= 1, k <<= 1) kb_dif_stage<<<grid, kT, 0, s>>>(dev, dtw, N, count, m, k);
        check_cuda(cudaGetLastError(), "encode transform");
        std::vector<EncodeOutJob> jobs;
        std::vector<NttJob> ntt;
        std::vector<MontJob> mont;
        for (size_t ci = 0; ci < count; ++ci)
            for (size_t l = 0; l < limbs; ++l) {
                jobs.push_back({out[ci] + l * N, (int)ci, mods[l]});
                ntt.push_back({out[ci] + l * N, out[ci] + l * N, mods[l], 0});
                const uint64_t q = c.mods[mods[l]].q;
                mont.push_back({out[ci] + l * N, (uint64_t)(((unsigned __int128)1 << 64) % q), mods[l], 0});
            }
        JobTable t;
        const EncodeOutJob* jo = t.add(jobs);
        const NttJob* jn = t.add(ntt);
        const MontJob* jm = t.add(mont);
        t.upload(c, s);
        {
            Probe probe(kClsElementwise, (16.0 + 8.0) * N * jobs.size(), s);
            kb_encode_out<<<grid_for(c, jobs.size()), kT, 0, s>>>(t.at(jo), (int)jobs.size(), dev,
                                                                  scale / static_cast<double>(N), N, c.d_mod);
        }
        if (eval) ntt_jobs(c, t.at(jn), (int)ntt.size(), true, s);
        if (montgomery) {
            Probe probe(kClsElementwise, 16.0 * N * mont.size(), s);
            kb_to_montgomery<<<grid_for(c, mont.size()), kT, 0, s>>>(t.at(jm), (int)mont.size(), c.d_mod);
        }
        check_cuda(cudaGetLastError(), "encode output");
        check_cuda(cudaFreeAsync(ws, s), "encode scratch");
        ws = nullptr;
        check_cuda(cudaStreamSynchronize(s), "encode");
    } catch (...) {
        if (ws) cudaFreeAsync(ws, s);
        cudaStreamSynchronize(s);
        throw;
    }
}

void decrypt_decode_device(Context& c, size_t count, size_t level, const double* scales, const uint64_t* const* b,
                           const uint64_t* const* a, const uint64_t* const* c2, const int8_t* secret, double* re,
                           double* im, cudaStream_t s) {
    if (count == 0) return;
    if (level >= c.nq) throw std::invalid_argument("ckks_decrypt: invalid level");
    if (!secret || !scales || !re || !im) throw std::invalid_argument("ckks_decrypt: null argument");
    const size_t N = c.N, half = N >> 1, L = level + 1;
    for (size_t i = 0; i < N; ++i)
        if (secret[i] < -1 || secret[i] > 1) throw std::invalid_argument("ckks_decrypt: secret must be ternary");
    for (size_t k = 0; k < count; ++k)
        if (!(scales[k] > 0.0)) throw std::invalid_argument("ckks_decrypt: scale must be positive");
    std::vector<double> tw;
    std::vector<uint32_t> perm;
    host::encode_tables(N, tw, perm);
    const uint64_t q0 = c.q[0], q1 = L > 1 ? c.q[1] : 1;
    const uint64_t q0_inv_q1 = L > 1 ? host::powmod(q0 % q1, q1 - 2, q1) : 0;
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    // scratch: m [count][L][N] u64, secret limbs [L][N], transform [count][N] double2, twiddles
    // [N] double2, slot values [2][count][N/2], scales [count], permutation [N/2], secret bytes
    const size_t bytes = count * L * N * 8 + L * N * 8 + count * N * 16 + N * 16 + 2 * count * half * 8 +
                         count * 8 + half * 4 + N + 256;
    unsigned char* ws = nullptr;
    if (cudaMallocAsync((void**)&ws, bytes, s) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "ckks_decrypt: scratch allocation failed");
    }
    auto* dev = reinterpret_cast<double2*>(ws);
    auto* dtw = dev + count * N;
    auto* dm = reinterpret_cast<uint64_t*>(dtw + N);
    auto* ds = dm + count * L * N;
    auto* dre = reinterpret_cast<double*>(ds + L * N);
    auto* dim = dre + count * half;
    auto* dscale = dim + count * half;
    auto* dperm = reinterpret_cast<uint32_t*>(dscale + count);
    auto* dsec = reinterpret_cast<int8_t*>(dperm + half);
    try {
        check_cuda(cudaMemcpyAsync(dtw, tw.data(), N * 16, cudaMemcpyHostToDevice, s), "decode upload");
        check_cuda(cudaMemcpyAsync(dperm, perm.data(), half * 4, cudaMemcpyHostToDevice, s), "decode upload");
        check_cuda(cudaMemcpyAsync(dscale, scales, count * 8, cudaMemcpyHostToDevice, s), "decode upload");
        check_cuda(cudaMemcpyAsync(dsec, secret, N, cudaMemcpyHostToDevice, s), "decode upload");
        std::vector<SecretLimbJob> sec;
        std::vector<NttJob> sntt, mntt;
        std::vector<DecryptJob> dec;
        for (size_t l = 0; l < L; ++l) {
            sec.push_back({dsec, ds + l * N, (int)l, 0});
            sntt.push_back({ds + l * N, ds + l * N, (int)l, 0});
        }
        for (size_t k = 0; k < count; ++k)
            for (size_t l = 0; l < L; ++l) {
                dec.push_back({dm + (k * L + l) * N, b[k] + l * N, a[k] + l * N, c2 && c2[k] ? c2[k] + l * N : nullptr,
                               ds + l * N, (int)l, 0});
                mntt.push_back({dm + (k * L + l) * N, dm + (k * L + l) * N, (int)l, 0});
            }
        JobTable t;
        const SecretLimbJob* j1 = t.add(sec);
        const NttJob* j2 = t.add(sntt);
        const DecryptJob* j3 = t.add(dec);
        const NttJob* j4 = t.add(mntt);
        t.upload(c, s);
        kb_secret_to_limb<<<grid_for(c, sec.size()), kT, 0, s>>>(t.at(j1), (int)sec.size(), c.d_mod);
        ntt_jobs(c, t.at(j2), (int)sntt.size(), true, s);
        kb_decrypt<<<grid_for(c, dec.size()), kT, 0, s>>>(t.at(j3), (int)dec.size(), c.d_mod);
        ntt_jobs(c, t.at(j4), (int)mntt.size(), false, s);
        const unsigned gridN = (unsigned)((count * N + kT - 1) / kT);
        const unsigned gridH = (unsigned)((count * half + kT - 1) / kT);
        kb_signed_coeffs<<<gridN, kT, 0, s>>>(dm, N, count, L, q0, q1, q0_inv_q1, dev);
        for (size_t m = 1, k = half; m < N; m <<= 1, k >>= 1) kb_dit_stage<<<gridH, kT, 0, s>>>(dev, dtw, N, count, m, k);
        kb_extract_slots<<<gridH, kT, 0, s>>>(dev, dperm, dscale, N, count, dre, dim);
        check_cuda(cudaGetLastError(), "decode");
        check_cuda(cudaMemcpyAsync(re, dre, count * half * 8, cudaMemcpyDeviceToHost, s), "decode download");
        check_cuda(cudaMemcpyAsync(im, dim, count * half * 8, cudaMemcpyDeviceToHost, s), "decode download");
        check_cuda(cudaFreeAsync(ws, s), "decode scratch");
        ws = nullptr;
        check_cuda(cudaStreamSynchronize(s), "decode");
    } catch (...) {
        if (ws) cudaFreeAsync(ws, s);
        cudaStreamSynchronize(s);
        throw;
    }
}

}  // namespace wg
