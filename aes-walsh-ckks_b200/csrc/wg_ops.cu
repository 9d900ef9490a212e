// Elementwise and structural ciphertext kernels: tensor product, add/sub, rescale and the
// evaluation-domain automorphism.
//
// References (src/ckks/operations/):
//   tensor      arith/ckks_mul.cpp:90-157   (Barrett products, c1 = a1*b2 + b1*a2)
//   add / sub   arith/ckks_addition.cpp, src/math/polynomial.cpp:1-32
//   rescale     arith/ckks_rescale.cpp:68-148
//   automorphism keyswitch/ckks_rotation.cpp:13-31 with the map of
//               src/ckks/context/rotation_key_generation.cpp:80-90, computed in the kernel.
#include "wg_internal.hpp"
#include "wg_keyswitch.cuh"

namespace wg {
namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads)
    k_automorphism(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst, size_t poly_stride,
                   uint64_t galois, int logN) {
    const size_t N = size_t{1} << logN;
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    const size_t off = (size_t)blockIdx.z * poly_stride + (size_t)blockIdx.y * N;
    dst[off + i] = src[off + automorphism_src(i, galois, logN)];
}

// c2 = a1 a2, c0 = b1 b2 (into b1), c1 = a1 b2 + b1 a2 (into a1), all Barrett products with
// the reference's exact reduction so representations match bit for bit.
__global__ void __launch_bounds__(kThreads)
    k_tensor(const Modulus* __restrict__ mods, uint64_t* __restrict__ b1, uint64_t* __restrict__ a1,
             const uint64_t* __restrict__ b2, const uint64_t* __restrict__ a2, uint64_t* __restrict__ c2,
             size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    const Modulus m = mods[blockIdx.y];
    const size_t k = (size_t)blockIdx.y * N + coeff;
    const uint64_t xa = a1[k], xb = b1[k], ya = a2[k], yb = b2[k];
    c2[k] = barrett_mul(xa, ya, m);
    const uint64_t tmp = barrett_mul(xb, ya, m);
    b1[k] = barrett_mul(xb, yb, m);
    a1[k] = add_mod(barrett_mul(xa, yb, m), tmp, m.q);
}

__global__ void __launch_bounds__(kThreads)
    k_add_sub(const Modulus* __restrict__ mods, uint64_t* __restrict__ x, const uint64_t* __restrict__ y,
              size_t poly_stride, int subtract, size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    const uint64_t q = mods[blockIdx.y].q;
    const size_t k = (size_t)blockIdx.z * poly_stride + (size_t)blockIdx.y * N + coeff;
    x[k] = subtract ? sub_mod(x[k], y[k], q) : add_mod(x[k], y[k], q);
}

// Rescale, step 1: from the dropped limb r (coefficient form, canonical mod p) build, per
// remaining limb i, (((r + floor(p/2)) mod p) mod q_i) - floor(p/2) mod q_i.  The reference
// adds NTT(floor(p/2)) to the limb and subtracts NTT((r + floor(p/2)) mod p); by linearity
// subtracting the NTT of this single difference gives the same canonical result.
__global__ void __launch_bounds__(kThreads)
    k_rescale_prep(const Modulus* __restrict__ mods, const uint64_t* __restrict__ polys, size_t poly_stride,
                   int level, const uint64_t* __restrict__ one_s, const uint64_t* __restrict__ half_mod,
                   uint64_t* __restrict__ rem, size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    const int i = blockIdx.y, poly = blockIdx.z;
    const uint64_t p = mods[level].q, half_p = p >> 1;
    const uint64_t q = mods[i].q;
    uint64_t shift = polys[(size_t)poly * poly_stride + (size_t)level * N + coeff] + half_p;
    if (shift >= p) shift -= p;
    const uint64_t r = reduce_shoup(shift, q, one_s[i]);
    rem[((size_t)poly * level + i) * N + coeff] = sub_mod(r, half_mod[i], q);
}

// Rescale, step 2: x_i = (x_i - NTT(rem_i)) * p^-1 mod q_i.
__global__ void __launch_bounds__(kThreads)
    k_rescale_finish(const Modulus* __restrict__ mods, uint64_t* __restrict__ polys, size_t poly_stride, int level,
                     const uint64_t* __restrict__ inv_p, const uint64_t* __restrict__ inv_p_s,
                     const uint64_t* __restrict__ rem, size_t N) {
    const size_t coeff = (size_t)blockIdx.x * kThreads + threadIdx.x;
    const int i = blockIdx.y, poly = blockIdx.z;
    const uint64_t q = mods[i].q;
    const size_t k = (size_t)poly * poly_stride + (size_t)i * N + coeff;
    uint64_t x = polys[k];
    if (x >= q) x -= q;
    const uint64_t d = sub_mod(x, rem[((size_t)poly * level + i) * N + coeff], q);
    polys[k] = mul_shoup(d, inv_p[i], inv_p_s[i], q);
}

}  // namespace

void automorphism(const Context& c, const uint64_t* src, uint64_t* dst, int limbs, int polys, size_t poly_stride,
                  uint64_t galois, cudaStream_t s) {
    if (limbs <= 0 || polys <= 0) return;
    Probe probe(kClsCombine, 16.0 * c.N * limbs * polys, s);
    k_automorphism<<<dim3((unsigned)(c.N / kThreads), limbs, polys), kThreads, 0, s>>>(src, dst, poly_stride, galois,
                                                                                      c.logN);
    check_cuda(cudaGetLastError(), "automorphism launch");
}

void tensor(const Context& c, size_t level, uint64_t* b1, uint64_t* a1, const uint64_t* b2, const uint64_t* a2,
            uint64_t* c2, cudaStream_t s) {
    Probe probe(kClsElementwise, 8.0 * c.N * (level + 1) * 7.0, s);
    k_tensor<<<dim3((unsigned)(c.N / kThreads), (unsigned)(level + 1)), kThreads, 0, s>>>(c.d_mod, b1, a1, b2, a2,
                                                                                          c2, c.N);
    check_cuda(cudaGetLastError(), "tensor launch");
}

void add_sub(const Context& c, size_t level, uint64_t* x, const uint64_t* y, int npolys, size_t poly_stride,
             bool subtract, cudaStream_t s) {
    Probe probe(kClsElementwise, 8.0 * c.N * (level + 1) * npolys * 3.0, s);
    k_add_sub<<<dim3((unsigned)(c.N / kThreads), (unsigned)(level + 1), npolys), kThreads, 0, s>>>(
        c.d_mod, x, y, poly_stride, subtract ? 1 : 0, c.N);
    check_cuda(cudaGetLastError(), "add/sub launch");
}

void rescale(const Context& c, size_t level, uint64_t* polys, int npolys, size_t poly_stride, uint64_t* ws,
             cudaStream_t s) {
    if (level == 0 || level >= c.nq) fail(kInvalid, "ckks_rescale: invalid level");
    const unsigned gx = (unsigned)(c.N / kThreads);
    // Dropped limb to coefficient form (in place; it is discarded afterwards).
    ntt_inverse(c, polys + level * c.N, 1, npolys, poly_stride, LimbMap{1, (int)level, 0}, s);
    {
        Probe probe(kClsElementwise, 8.0 * c.N * npolys * (1.0 + level), s);
        k_rescale_prep<<<dim3(gx, (unsigned)level, npolys), kThreads, 0, s>>>(
            c.d_mod, polys, poly_stride, (int)level, c.rs_one_s[level], c.rs_half[level], ws, c.N);
    }
    ntt_forward(c, ws, (int)level, npolys, level * c.N, LimbMap{(int)level, 0, 0}, s);
    Probe probe(kClsElementwise, 8.0 * c.N * npolys * 3.0 * level, s);
    k_rescale_finish<<<dim3(gx, (unsigned)level, npolys), kThreads, 0, s>>>(
        c.d_mod, polys, poly_stride, (int)level, c.rs_inv_p[level], c.rs_inv_p_s[level], ws, c.N);
    check_cuda(cudaGetLastError(), "rescale launch");
}

}  // namespace wg
