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

}  // namespace

void encode_slots_device(Context& c, size_t count, size_t limbs, double scale, const double* re, const double* im,
                         uint64_t* const* out, bool eval, cudaStream_t s) {
    if (count == 0) return;
    if (!(scale > 0.0)) throw std::invalid_argument("ckks_encode: scale must be positive");
    if (limbs == 0 || limbs > c.nq) throw std::invalid_argument("ckks_encode: invalid level");
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
        for (size_t ci = 0; ci < count; ++ci)
            for (size_t l = 0; l < limbs; ++l) {
                jobs.push_back({out[ci] + l * N, (int)ci, (int)l});
                ntt.push_back({out[ci] + l * N, out[ci] + l * N, (int)l, 0});
            }
        JobTable t;
        const EncodeOutJob* jo = t.add(jobs);
        const NttJob* jn = t.add(ntt);
        t.upload(c, s);
        {
            Probe probe(kClsElementwise, (16.0 + 8.0) * N * jobs.size(), s);
            kb_encode_out<<<grid_for(c, jobs.size()), kT, 0, s>>>(t.at(jo), (int)jobs.size(), dev,
                                                                  scale / static_cast<double>(N), N, c.d_mod);
        }
        if (eval) ntt_jobs(c, t.at(jn), (int)ntt.size(), true, s);
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

}  // namespace wg
