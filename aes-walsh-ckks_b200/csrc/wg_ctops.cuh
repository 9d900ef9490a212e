// Ciphertext-level device operations over batches of ciphertexts that share metadata, used by
// the host-orchestrated evaluators (Chebyshev series, EvalMod bootstrap, Walsh S-box).  Every
// operation is one set of batched launches for the whole batch.  Included by several
// translation units: everything here has internal linkage.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <stdexcept>
#include <vector>

#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_internal.hpp"

namespace wg {
namespace {
using namespace bk;

enum ScalarOp : int { kScalarMul = 0, kScalarMulAdd = 1, kScalarAdd = 2 };

struct ScalarJob {
    uint64_t* x;
    const uint64_t* y;
    uint64_t s, s_shoup;
    int mod, op;
};

// x = x * s, x = x + y * s or x = x + s (mod q), s < q; canonical in, canonical out.
__global__ void __launch_bounds__(kT) kb_scalar(const ScalarJob* jobs, int n, const Modulus* mods) {
    const ScalarJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q = mods[j->mod].q;
    if (j->op == kScalarMul)
        j->x[k] = mul_shoup(j->x[k], j->s, j->s_shoup, q);
    else if (j->op == kScalarMulAdd)
        j->x[k] = add_mod(j->x[k], mul_shoup(j->y[k], j->s, j->s_shoup, q), q);
    else
        j->x[k] = add_mod(j->x[k], j->s, q);
}

struct PmulJob {
    uint64_t* x;
    const uint64_t* p;
    int mod, pad;
};

// x = x * p (mod q), pointwise (Barrett product of canonical residues)
__global__ void __launch_bounds__(kT) kb_pmul(const PmulJob* jobs, int n, const Modulus* mods) {
    const PmulJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    j->x[k] = barrett_mul(j->x[k], j->p[k], mods[j->mod]);
}

// A batch of ciphertexts with common metadata.  Polynomial k of ciphertext i lives at p[i][k]
// with room for `cap` limbs; limbs [0, level] are live.
struct CtBatch {
    std::vector<std::array<uint64_t*, 3>> p;
    int np = 2;
    size_t level = 0;
    size_t cap = 0;
    long double scale = 0.0L;
};

class DeviceOps {
public:
    DeviceOps(Context& c, size_t count, cudaStream_t s) : c_(c), count_(count), s_(s) {}
    ~DeviceOps() {
        for (uint64_t* p : owned_) cudaFreeAsync(p, s_);
    }
    DeviceOps(const DeviceOps&) = delete;
    DeviceOps& operator=(const DeviceOps&) = delete;

    size_t count() const { return count_; }

    CtBatch wrap(uint64_t* const* b, uint64_t* const* a, size_t level, long double scale) {
        CtBatch x;
        x.p.resize(count_);
        for (size_t i = 0; i < count_; ++i) x.p[i] = {b[i], a[i], nullptr};
        x.np = 2;
        x.level = level;
        x.cap = level + 1;
        x.scale = scale;
        return x;
    }

    CtBatch zeros(size_t level, long double scale) {
        CtBatch x;
        x.p.resize(count_);
        for (size_t i = 0; i < count_; ++i) x.p[i] = {buffer(level + 1, true), buffer(level + 1, true), nullptr};
        x.np = 2;
        x.level = level;
        x.cap = level + 1;
        x.scale = scale;
        return x;
    }

    CtBatch clone(const CtBatch& x) {
        CtBatch y = x;
        y.cap = x.level + 1;
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k) {
                y.p[i][k] = buffer(y.cap, false);
                check_cuda(cudaMemcpyAsync(y.p[i][k], x.p[i][k], y.cap * c_.N * 8, cudaMemcpyDeviceToDevice, s_),
                           "evalpoly copy");
            }
        return y;
    }

    void pad(CtBatch& x, int np) {
        if (np < x.np) throw std::invalid_argument("ckks_evalchebyshev: cannot shrink ciphertext degree by padding");
        while (x.np < np) {
            for (size_t i = 0; i < count_; ++i) x.p[i][x.np] = buffer(x.cap, true);
            ++x.np;
        }
    }

    // (b, a) x (b', a') -> (b b', a b' + b a', a a'); y must not alias x.
    void tensor(CtBatch& x, const CtBatch& y) {
        const size_t N = c_.N;
        pad(x, 3);
        std::vector<TensorJob> jobs;
        for (size_t i = 0; i < count_; ++i)
            for (size_t l = 0; l <= x.level; ++l)
                jobs.push_back({x.p[i][0] + l * N, x.p[i][1] + l * N, y.p[i][0] + l * N, y.p[i][1] + l * N,
                                x.p[i][2] + l * N, (int)l, 0});
        JobTable t;
        const TensorJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 8.0 * N * jobs.size() * 7.0, s_);
        kb_tensor<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "evalpoly tensor");
    }

    void relin(CtBatch& x) {
        if (x.np != 3) return;
        const KeyEntry& k = c_.key(WG_KEY_RELIN, 0);
        std::vector<KsItem> items(count_);
        for (size_t i = 0; i < count_; ++i) {
            KsItem& it = items[i];
            it.level = x.level;
            it.key_term = x.p[i][2];
            it.key = &k;
            it.b_in = x.p[i][0];
            it.a_in = x.p[i][1];
            it.b = x.p[i][0];
            it.a = x.p[i][1];
            it.b_add = 1;
            it.a_add = 1;
            it.galois = 0;
        }
        batch_keyswitch(c_, items.data(), count_, s_);
        x.np = 2;
    }

    // ckks_rescale on every polynomial; scale /= q_level.
    void rescale(CtBatch& x) {
        const size_t N = c_.N, lv = x.level;
        if (lv == 0) throw std::invalid_argument("ckks_rescale: invalid level");
        uint64_t* rem = scratch(count_ * x.np * lv);
        const uint64_t* rc = c_.rs_host.data() + c_.rs_host_off[lv];
        std::vector<NttJob> drop_intt, rem_ntt;
        std::vector<RescalePrepJob> prep;
        std::vector<RescaleFinishJob> fin;
        uint64_t* r = rem;
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k) {
                uint64_t* poly = x.p[i][k];
                uint64_t* drop = poly + lv * N;
                drop_intt.push_back({drop, drop, (int)lv, 0});
                for (size_t q = 0; q < lv; ++q) {
                    prep.push_back({drop, r + q * N, rc[q], rc[3 * lv + q], (int)lv, (int)q});
                    rem_ntt.push_back({r + q * N, r + q * N, (int)q, 0});
                    fin.push_back({poly + q * N, r + q * N, rc[lv + q], rc[2 * lv + q], (int)q, 0});
                }
                r += lv * N;
            }
        JobTable t;
        const NttJob* jd = t.add(drop_intt);
        const RescalePrepJob* jp = t.add(prep);
        const NttJob* jr = t.add(rem_ntt);
        const RescaleFinishJob* jf = t.add(fin);
        t.upload(c_, s_);
        ntt_jobs(c_, t.at(jd), (int)drop_intt.size(), false, s_);
        {
            Probe probe(kClsElementwise, 8.0 * N * prep.size() * 2.0, s_);
            kb_rescale_prep<<<grid_for(c_, prep.size()), kT, 0, s_>>>(t.at(jp), (int)prep.size(), c_.d_mod);
        }
        ntt_jobs(c_, t.at(jr), (int)rem_ntt.size(), true, s_);
        {
            Probe probe(kClsElementwise, 8.0 * N * fin.size() * 3.0, s_);
            kb_rescale_finish<<<grid_for(c_, fin.size()), kT, 0, s_>>>(t.at(jf), (int)fin.size(), c_.d_mod);
        }
        check_cuda(cudaGetLastError(), "evalpoly rescale");
        x.scale = x.scale / static_cast<long double>(c_.q[lv]);
        x.level = lv - 1;
    }

    void add(CtBatch& x, const CtBatch& y, bool subtract) {
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k) add_sub(c_, x.level, x.p[i][k], y.p[i][k], 1, 0, subtract, s_);
    }

    // op per limb: scalars[l] < q_l.  kScalarMul / kScalarMulAdd touch every polynomial,
    // kScalarAdd the b polynomial only; zero scalars of a multiply-add are skipped.
    void scalar(CtBatch& x, const CtBatch* y, const std::vector<uint64_t>& scalars, int op) {
        const size_t N = c_.N;
        std::vector<ScalarJob> jobs;
        for (size_t l = 0; l <= x.level; ++l) {
            const uint64_t q = c_.q[l], sv = scalars[l];
            if (op == kScalarMulAdd && sv == 0) continue;
            const uint64_t ss = host::shoup(sv, q);
            for (size_t i = 0; i < count_; ++i) {
                const int polys = op == kScalarAdd ? 1 : (op == kScalarMulAdd ? y->np : x.np);
                for (int k = 0; k < polys; ++k)
                    jobs.push_back({x.p[i][k] + l * N, y ? y->p[i][k] + l * N : nullptr, sv, ss, (int)l, op});
            }
        }
        if (jobs.empty()) return;
        JobTable t;
        const ScalarJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 8.0 * N * jobs.size() * (op == kScalarMulAdd ? 3.0 : 2.0), s_);
        kb_scalar<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "evalpoly scalar");
    }

    // ckks_conjugate: automorphism X -> X^(2N-1) of (b, a), then key switch of the permuted a.
    CtBatch conjugate(const CtBatch& x) {
        const size_t N = c_.N, L = x.level + 1;
        const KeyEntry& k = c_.key(WG_KEY_CONJ, 0);
        CtBatch perm = alloc(x.level, 2);
        CtBatch out = alloc(x.level, 2);
        out.scale = x.scale;
        std::vector<KsItem> items(count_);
        for (size_t i = 0; i < count_; ++i) {
            for (int poly = 0; poly < 2; ++poly)
                automorphism(c_, x.p[i][poly], perm.p[i][poly], (int)L, 1, 0, 2 * N - 1, s_);
            KsItem& it = items[i];
            it.level = x.level;
            it.key_term = perm.p[i][1];
            it.key = &k;
            it.b_in = perm.p[i][0];
            it.a_in = perm.p[i][1];
            it.b = out.p[i][0];
            it.a = out.p[i][1];
            it.b_add = 1;
            it.a_add = 0;
            it.galois = 0;
        }
        batch_keyswitch(c_, items.data(), count_, s_);
        return out;
    }

    // ckks_mul_inplace(ct, Complex, scale): the slot-constant re + i im encodes (at scale
    // `scale`) to round(scale re) + round(scale im) X^(N/2); multiply every polynomial by it.
    // Evaluation-form plaintext of the slot constant re + i im at `scale`:
    // round(scale re) + round(scale im) X^(N/2), reduced per limb, then NTT.
    uint64_t* constant_plaintext(size_t L, double re, double im, double scale) {
        const size_t N = c_.N;
        const long double r0 = std::round(static_cast<long double>(scale) * re);
        const long double r1 = std::round(static_cast<long double>(scale) * im);
        std::vector<uint64_t> host(L * N, 0);
        for (size_t l = 0; l < L; ++l) {
            const uint64_t q = c_.q[l];
            auto modq = [q](long double v) {
                long double m = std::fmod(v, static_cast<long double>(q));
                if (m < 0.0L) m += static_cast<long double>(q);
                uint64_t r = static_cast<uint64_t>(m);
                return r >= q ? r % q : r;
            };
            host[l * N] = modq(r0);
            host[l * N + N / 2] = modq(r1);
        }
        uint64_t* pt = buffer(L, false);
        check_cuda(cudaMemcpyAsync(pt, host.data(), L * N * 8, cudaMemcpyHostToDevice, s_), "constant plaintext");
        check_cuda(cudaStreamSynchronize(s_), "constant plaintext");
        ntt_forward(c_, pt, (int)L, 1, 0, LimbMap{0, 0, 0}, s_);
        return pt;
    }

    // Evaluation-form plaintext from coefficient-form residues (L limbs): upload, then NTT.
    uint64_t* upload_plain(const uint64_t* coeff, size_t L) {
        uint64_t* pt = buffer(L, false);
        check_cuda(cudaMemcpyAsync(pt, coeff, L * c_.N * 8, cudaMemcpyHostToDevice, s_), "plaintext upload");
        check_cuda(cudaStreamSynchronize(s_), "plaintext upload");
        ntt_forward(c_, pt, (int)L, 1, 0, LimbMap{0, 0, 0}, s_);
        return pt;
    }

    // b += pt (evaluation form, x.level+1 limbs) on every ciphertext (ckks_add_inplace(ct, pt))
    void add_plain(CtBatch& x, const uint64_t* pt) {
        for (size_t i = 0; i < count_; ++i) add_sub(c_, x.level, x.p[i][0], pt, 1, 0, false, s_);
    }

    // every polynomial *= pt pointwise (ckks_mul_inplace(ct, pt)); scale left to the caller
    void mul_plain(CtBatch& x, const uint64_t* pt) {
        const size_t N = c_.N, L = x.level + 1;
        std::vector<PmulJob> jobs;
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k)
                for (size_t l = 0; l < L; ++l) jobs.push_back({x.p[i][k] + l * N, pt + l * N, (int)l, 0});
        JobTable t;
        const PmulJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 8.0 * N * jobs.size() * 3.0, s_);
        kb_pmul<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "plaintext multiply");
    }

    void mul_complex_constant(CtBatch& x, double re, double im, double scale) {
        const size_t N = c_.N, L = x.level + 1;
        uint64_t* pt = constant_plaintext(L, re, im, scale);
        std::vector<PmulJob> jobs;
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k)
                for (size_t l = 0; l < L; ++l) jobs.push_back({x.p[i][k] + l * N, pt + l * N, (int)l, 0});
        JobTable t;
        const PmulJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 8.0 * N * jobs.size() * 3.0, s_);
        kb_pmul<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "evalpoly plaintext multiply");
    }

    // b += the encoding of the slot constant re + i im at `scale` (closed form, as in
    // mul_complex_constant), on every ciphertext of the batch.
    void add_complex_constant(CtBatch& x, double re, double im, double scale) {
        const size_t N = c_.N, L = x.level + 1;
        uint64_t* pt = constant_plaintext(L, re, im, scale);
        for (size_t i = 0; i < count_; ++i) add_sub(c_, x.level, x.p[i][0], pt, 1, 0, false, s_);
    }

    // x *= k (mod q) on every polynomial (ckks_mul_inplace(ct, int64_t)); scale unchanged.
    void mul_int(CtBatch& x, int64_t k) {
        if (k == 1) return;
        if (k == 0) {
            for (size_t i = 0; i < count_; ++i)
                for (int j = 0; j < x.np; ++j)
                    check_cuda(cudaMemsetAsync(x.p[i][j], 0, (x.level + 1) * c_.N * 8, s_), "zero");
            return;
        }
        std::vector<uint64_t> v(x.level + 1);
        for (size_t l = 0; l <= x.level; ++l) {
            const int64_t q = (int64_t)c_.q[l];
            int64_t r = k % q;
            if (r < 0) r += q;
            v[l] = (uint64_t)r;
        }
        scalar(x, nullptr, v, kScalarMul);
    }

    uint64_t* raw(size_t limbs) { return buffer(limbs, false); }

    // ckks_rotate_inplace by r on every ciphertext of the batch (key switch, then automorphism)
    void rotate(CtBatch& x, int64_t r) {
        const int64_t slots = (int64_t)(c_.N / 2);
        int64_t n = r % slots;
        if (n < 0) n += slots;
        if (n == 0) return;
        const KeyEntry& k = c_.key(WG_KEY_ROTATION, n);
        std::vector<KsItem> items(count_);
        for (size_t i = 0; i < count_; ++i) {
            KsItem& it = items[i];
            it.level = x.level;
            it.key_term = x.p[i][1];
            it.key = &k;
            it.b_in = x.p[i][0];
            it.a_in = x.p[i][1];
            it.b = x.p[i][0];
            it.a = x.p[i][1];
            it.b_add = 1;
            it.a_add = 0;
            it.galois = host::powmod(5, (uint64_t)n, 2 * c_.N);
        }
        batch_keyswitch(c_, items.data(), count_, s_);
    }

    CtBatch alloc(size_t level, int np) {
        CtBatch x;
        x.p.resize(count_);
        for (size_t i = 0; i < count_; ++i) {
            x.p[i] = {nullptr, nullptr, nullptr};
            for (int k = 0; k < np; ++k) x.p[i][k] = buffer(level + 1, false);
        }
        x.np = np;
        x.level = level;
        x.cap = level + 1;
        return x;
    }

    void copy_out(const CtBatch& x, uint64_t* const* b, uint64_t* const* a) {
        for (size_t i = 0; i < count_; ++i) {
            if (x.p[i][0] != b[i])
                check_cuda(cudaMemcpyAsync(b[i], x.p[i][0], (x.level + 1) * c_.N * 8, cudaMemcpyDeviceToDevice, s_),
                           "evalpoly output");
            if (x.p[i][1] != a[i])
                check_cuda(cudaMemcpyAsync(a[i], x.p[i][1], (x.level + 1) * c_.N * 8, cudaMemcpyDeviceToDevice, s_),
                           "evalpoly output");
        }
    }

private:
    uint64_t* buffer(size_t limbs, bool zero) {
        uint64_t* p = nullptr;
        const size_t bytes = std::max<size_t>(limbs, 1) * c_.N * 8;
        if (cudaMallocAsync((void**)&p, bytes, s_) != cudaSuccess) {
            cudaGetLastError();
            fail(kNoMemory, "ckks_evalchebyshev: device allocation failed");
        }
        owned_.push_back(p);
        if (zero) check_cuda(cudaMemsetAsync(p, 0, bytes, s_), "evalpoly zero");
        return p;
    }
    uint64_t* scratch(size_t limbs) { return buffer(limbs, false); }

    Context& c_;
    size_t count_;
    cudaStream_t s_;
    std::vector<uint64_t*> owned_;
};

}  // namespace
}  // namespace wg
