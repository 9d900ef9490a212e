// Ciphertext-level device operations over batches of ciphertexts that share metadata, used by
// the host-orchestrated evaluators (Chebyshev series, EvalMod bootstrap, Walsh S-box).  Every
// operation is one set of batched launches for the whole batch.  Included by several
// translation units: everything here has internal linkage.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <stdexcept>
#include <vector>

#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_internal.hpp"
#include "wg_encode.hpp"

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
    const uint64_t q = mods[j->mod].q, s = j->s, ss = j->s_shoup;
    uint64_t x[kWide], y[kWide];
    if (j->op == kScalarMul) {
#pragma unroll
        for (int r = 0; r < kWide; ++r) x[r] = j->x[wide_index(r)];
#pragma unroll
        for (int r = 0; r < kWide; ++r) j->x[wide_index(r)] = mul_shoup(x[r], s, ss, q);
    } else if (j->op == kScalarMulAdd) {
#pragma unroll
        for (int r = 0; r < kWide; ++r) x[r] = j->x[wide_index(r)], y[r] = j->y[wide_index(r)];
#pragma unroll
        for (int r = 0; r < kWide; ++r) j->x[wide_index(r)] = add_mod(x[r], mul_shoup(y[r], s, ss, q), q);
    } else {
#pragma unroll
        for (int r = 0; r < kWide; ++r) x[r] = j->x[wide_index(r)];
#pragma unroll
        for (int r = 0; r < kWide; ++r) j->x[wide_index(r)] = add_mod(x[r], s, q);
    }
}

constexpr int kMaxLincombTerms = 16;

struct LincombJob {
    uint64_t* out;
    const uint64_t* src[kMaxLincombTerms];
    uint64_t c[kMaxLincombTerms], cs[kMaxLincombTerms];
    uint64_t add;
    int n, mod, accumulate, pad;
};

// out = (accumulate ? out : 0) + add + sum_t c_t src_t (mod q).  Shoup products and modular
// additions of canonical residues: the value is the canonical residue of the sum, whatever the
// order of the terms, equal to adding the scaled terms one multiply-add at a time.
__global__ void __launch_bounds__(kT) kb_lincomb(const LincombJob* jobs, int n, const Modulus* mods) {
    const LincombJob* j = job_of(jobs, n);
    if (!j) return;
    const uint64_t q = mods[j->mod].q;
    uint64_t acc[kWide];
#pragma unroll
    for (int r = 0; r < kWide; ++r) acc[r] = j->accumulate ? j->out[wide_index(r)] : 0;
#pragma unroll
    for (int r = 0; r < kWide; ++r) acc[r] = add_mod(acc[r], j->add, q);
    for (int t = 0; t < j->n; ++t) {
        const uint64_t* src = j->src[t];
        const uint64_t c = j->c[t], cs = j->cs[t];
        uint64_t v[kWide];
#pragma unroll
        for (int r = 0; r < kWide; ++r) v[r] = src[wide_index(r)];
#pragma unroll
        for (int r = 0; r < kWide; ++r) acc[r] = add_mod(acc[r], mul_shoup(v[r], c, cs, q), q);
    }
#pragma unroll
    for (int r = 0; r < kWide; ++r) j->out[wide_index(r)] = acc[r];
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
    const Modulus m = mods[j->mod];
    uint64_t x[kWide], p[kWide];
#pragma unroll
    for (int r = 0; r < kWide; ++r) x[r] = j->x[wide_index(r)], p[r] = j->p[wide_index(r)];
#pragma unroll
    for (int r = 0; r < kWide; ++r) j->x[wide_index(r)] = barrett_mul(x[r], p[r], m);
}

struct CopyJob {
    uint64_t* dst;
    const uint64_t* src;
};

__global__ void __launch_bounds__(kT) kb_copy(const CopyJob* jobs, int n) {
    const CopyJob* j = job_of(jobs, n);
    if (!j) return;
    uint64_t v[kWide];
#pragma unroll
    for (int r = 0; r < kWide; ++r) v[r] = j->src[wide_index(r)];
#pragma unroll
    for (int r = 0; r < kWide; ++r) j->dst[wide_index(r)] = v[r];
}

struct AddJob {
    uint64_t* x;
    const uint64_t* y;
    int mod, sub;
};

// x = x +- y (mod q), canonical
__global__ void __launch_bounds__(kT) kb_add(const AddJob* jobs, int n, const Modulus* mods) {
    const AddJob* j = job_of(jobs, n);
    if (!j) return;
    const uint64_t q = mods[j->mod].q;
    uint64_t x[kWide], y[kWide];
#pragma unroll
    for (int r = 0; r < kWide; ++r) x[r] = j->x[wide_index(r)], y[r] = j->y[wide_index(r)];
    if (j->sub) {
#pragma unroll
        for (int r = 0; r < kWide; ++r) j->x[wide_index(r)] = sub_mod(x[r], y[r], q);
    } else {
#pragma unroll
        for (int r = 0; r < kWide; ++r) j->x[wide_index(r)] = add_mod(x[r], y[r], q);
    }
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
        WG_SPAN("free");
        // chunks go back to the context for later operation sets (see Context::give_chunk)
        for (const auto& ch : owned_) c_.give_chunk(ch.first, ch.second * 8, s_);
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
        const std::vector<uint64_t*> bufs = buffers(2 * count_, level + 1, true);
        for (size_t i = 0; i < count_; ++i) x.p[i] = {bufs[2 * i], bufs[2 * i + 1], nullptr};
        x.np = 2;
        x.level = level;
        x.cap = level + 1;
        x.scale = scale;
        return x;
    }

    // fresh copy of limbs [0, level] of every polynomial (one launch)
    CtBatch clone(const CtBatch& x) {
        const size_t N = c_.N;
        CtBatch y = x;
        y.cap = x.level + 1;
        std::vector<CopyJob> jobs;
        jobs.reserve(count_ * x.np * y.cap);
        const std::vector<uint64_t*> bufs = buffers(count_ * x.np, y.cap, false);
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k) {
                y.p[i][k] = bufs[i * x.np + k];
                for (size_t l = 0; l < y.cap; ++l) jobs.push_back({y.p[i][k] + l * N, x.p[i][k] + l * N});
            }
        JobTable t;
        const CopyJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 16.0 * N * jobs.size(), s_);
        kb_copy<<<grid_wide(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size());
        check_cuda(cudaGetLastError(), "batched copy");
        return y;
    }

    void pad(CtBatch& x, int np) {
        if (np < x.np) throw std::invalid_argument("ckks_evalchebyshev: cannot shrink ciphertext degree by padding");
        while (x.np < np) {
            const std::vector<uint64_t*> bufs = buffers(count_, x.cap, true);
            for (size_t i = 0; i < count_; ++i) x.p[i][x.np] = bufs[i];
            ++x.np;
        }
    }

    // (b, a) x (b', a') -> (b b', a b' + b a', a a'); y must not alias x.
    void tensor(CtBatch& x, const CtBatch& y) {
        const size_t N = c_.N;
        if (x.np != 2) throw std::invalid_argument("ckks_mul_inplace(ct,ct): expected 2-component inputs");
        const std::vector<uint64_t*> bufs = buffers(count_, x.cap, false);  // fully written below
        for (size_t i = 0; i < count_; ++i) x.p[i][2] = bufs[i];
        x.np = 3;
        std::vector<TensorJob> jobs;
        for (size_t i = 0; i < count_; ++i)
            for (size_t l = 0; l <= x.level; ++l)
                jobs.push_back({x.p[i][0] + l * N, x.p[i][1] + l * N, y.p[i][0] + l * N, y.p[i][1] + l * N,
                                x.p[i][2] + l * N, (int)l, 0});
        JobTable t;
        const TensorJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 8.0 * N * jobs.size() * 7.0, s_);
        kb_tensor<<<grid_wide(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
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
        uint64_t* r = scratch(count_ * x.np * lv);
        RescaleJobs rj;
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k) {
                rj.add(x.p[i][k], lv, r);
                r += lv * N;
            }
        JobTable t;
        rj.plan(c_, t);
        t.upload(c_, s_);
        rj.run(c_, t, s_);
        x.scale = x.scale / static_cast<long double>(c_.q[lv]);
        x.level = lv - 1;
    }

    // x +-= y on every polynomial and limb of the batch: one launch
    void add(CtBatch& x, const CtBatch& y, bool subtract) {
        const size_t N = c_.N;
        std::vector<AddJob> jobs;
        jobs.reserve(count_ * x.np * (x.level + 1));
        for (size_t i = 0; i < count_; ++i)
            for (int k = 0; k < x.np; ++k)
                for (size_t l = 0; l <= x.level; ++l)
                    jobs.push_back({x.p[i][k] + l * N, y.p[i][k] + l * N, (int)l, subtract ? 1 : 0});
        add_jobs(jobs);
    }

    void add_jobs(const std::vector<AddJob>& jobs) {
        if (jobs.empty()) return;
        JobTable t;
        const AddJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 8.0 * c_.N * jobs.size() * 3.0, s_);
        kb_add<<<grid_wide(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "batched add");
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
        kb_scalar<<<grid_wide(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "evalpoly scalar");
    }

    // One term of a linear combination: a batch and one constant per limb (canonical).
    struct LinTerm {
        CtBatch x;
        std::vector<uint64_t> c;
    };

    // A fresh batch (level, np) = cadd (on the b polynomial) + sum of c_t x_t per limb; a term
    // with fewer polynomials than np contributes zeros to the others.  Up to kMaxLincombTerms
    // terms per launch.
    CtBatch lincomb(size_t level, int np, long double scale, const std::vector<uint64_t>& cadd,
                    const std::vector<LinTerm>& terms) {
        const size_t N = c_.N;
        CtBatch out = alloc(level, np);
        out.scale = scale;
        const size_t chunks = std::max<size_t>(1, (terms.size() + kMaxLincombTerms - 1) / kMaxLincombTerms);
        for (size_t ch = 0; ch < chunks; ++ch) {
            std::vector<LincombJob> jobs;
            for (size_t i = 0; i < count_; ++i)
                for (int poly = 0; poly < np; ++poly)
                    for (size_t l = 0; l <= level; ++l) {
                        LincombJob jb{};
                        jb.out = out.p[i][poly] + l * N;
                        jb.mod = (int)l;
                        jb.accumulate = ch > 0;
                        jb.add = (ch == 0 && poly == 0) ? cadd[l] : 0;
                        const uint64_t q = c_.q[l];
                        for (size_t t = ch * kMaxLincombTerms; t < std::min(terms.size(), (ch + 1) * kMaxLincombTerms); ++t) {
                            const LinTerm& tm = terms[t];
                            if (poly >= tm.x.np || tm.c[l] == 0) continue;
                            jb.src[jb.n] = tm.x.p[i][poly] + l * N;
                            jb.c[jb.n] = tm.c[l];
                            jb.cs[jb.n] = host::shoup(tm.c[l], q);
                            ++jb.n;
                        }
                        jobs.push_back(jb);
                    }
            JobTable t;
            const LincombJob* j = t.add(jobs);
            t.upload(c_, s_);
            double words = 0;
            for (const auto& jb : jobs) words += jb.n + 1 + jb.accumulate;
            Probe probe(kClsElementwise, 8.0 * N * words, s_);
            kb_lincomb<<<grid_wide(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
            check_cuda(cudaGetLastError(), "linear combination");
        }
        return out;
    }

    // ckks_conjugate: automorphism X -> X^(2N-1) of (b, a), then key switch of the permuted a.
    CtBatch conjugate(const CtBatch& x) {
        const size_t N = c_.N, L = x.level + 1;
        const KeyEntry& k = c_.key(WG_KEY_CONJ, 0);
        CtBatch perm = alloc(x.level, 2);
        CtBatch out = alloc(x.level, 2);
        out.scale = x.scale;
        std::vector<KsItem> items(count_);
        // X -> X^(2N-1) of every limb of every ciphertext in one launch
        std::vector<GatherJob> gather;
        gather.reserve(count_ * L);
        for (size_t i = 0; i < count_; ++i)
            for (size_t l = 0; l < L; ++l)
                gather.push_back({x.p[i][0] + l * N, x.p[i][1] + l * N, perm.p[i][0] + l * N, perm.p[i][1] + l * N,
                                  2 * N - 1});
        {
            JobTable t;
            const GatherJob* j = t.add(gather);
            t.upload(c_, s_);
            Probe probe(kClsCombine, 8.0 * N * 4.0 * gather.size(), s_);
            kb_gather<<<grid_for(c_, gather.size()), kT, 0, s_>>>(t.at(j), (int)gather.size(), c_.logN);
            check_cuda(cudaGetLastError(), "conjugation automorphism");
        }
        for (size_t i = 0; i < count_; ++i) {
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
    // Evaluation-form plaintext of the slot constant re + i im at `scale` (the host encoder,
    // the same residues as the reference's ckks_encode; for a constant they are
    // round(scale re) + round(scale im) X^(N/2) up to the FFT's rounding), then NTT.  Cached per
    // (value, scale, limbs) for the lifetime of this object.
    // Constants are shared through the context (up to kConstCacheBytes), else kept for the life
    // of this operation set.
    uint64_t* constant_plaintext(size_t L, double re, double im, double scale) {
        const auto key = std::make_tuple(re, im, scale, L);
        auto it = const_cache_.find(key);
        if (it != const_cache_.end()) return it->second;
        uint64_t* pt = shared_constant(key);
        if (!pt) pt = constant_plaintext_new(L, re, im, scale);
        const_cache_.emplace(key, pt);
        return pt;
    }

    static constexpr size_t kConstCacheBytes = size_t{2} << 30;

    uint64_t* shared_constant(const std::tuple<double, double, double, size_t>& key) {
        const auto [re, im, scale, L] = key;
        std::lock_guard<std::mutex> g(c_.const_mutex);
        auto ct = c_.consts.find(key);
        if (ct != c_.consts.end()) {
            if (ct->second.stream != s_) check_cuda(cudaStreamWaitEvent(s_, ct->second.ready, 0), "constant wait");
            return ct->second.d;
        }
        const size_t bytes = L * c_.N * 8;
        if (c_.const_bytes + bytes > kConstCacheBytes) return nullptr;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (s_) cudaStreamIsCapturing(s_, &cs);
        if (cs != cudaStreamCaptureStatusNone) return nullptr;
        Context::ConstPlain cp{nullptr, nullptr, s_, bytes};
        check_cuda(cudaMalloc((void**)&cp.d, bytes), "constant plaintext");
        if (cudaEventCreateWithFlags(&cp.ready, cudaEventDisableTiming) != cudaSuccess) {
            cudaFree(cp.d);
            fail(kRuntime, "constant plaintext event");
        }
        try {
            const size_t N = c_.N;
            std::vector<double> vr(N / 2, re), vi(N / 2, im);
            std::vector<uint64_t> host(L * N);
            host::encode_slots(N, vr.data(), vi.data(), scale, c_.q.data(), L, host.data());
            upload_plain_into(host.data(), L, cp.d);
            check_cuda(cudaEventRecord(cp.ready, s_), "constant plaintext event");
        } catch (...) {
            cudaFree(cp.d);
            cudaEventDestroy(cp.ready);
            throw;
        }
        c_.consts.emplace(key, cp);
        c_.const_bytes += bytes;
        return cp.d;
    }

    uint64_t* constant_plaintext_new(size_t L, double re, double im, double scale) {
        const size_t N = c_.N;
        std::vector<double> vr(N / 2, re), vi(N / 2, im);
        std::vector<uint64_t> host(L * N);
        host::encode_slots(N, vr.data(), vi.data(), scale, c_.q.data(), L, host.data());
        return upload_plain(host.data(), L);
    }

    // Evaluation-form plaintext from coefficient-form residues (L limbs): upload, then NTT.
    uint64_t* upload_plain(const uint64_t* coeff, size_t L) {
        uint64_t* pt = buffer(L, false);
        upload_plain_into(coeff, L, pt);
        return pt;
    }

    void upload_plain_into(const uint64_t* coeff, size_t L, uint64_t* pt) {
        const size_t N = c_.N;
        // staged copy of the coefficients; the forward NTT reads it and writes the plaintext
        auto* staged = static_cast<uint64_t*>(c_.batch_buffers(s_).stage(c_, coeff, L * N * 8, s_));
        std::vector<NttJob> jobs;
        for (size_t l = 0; l < L; ++l) jobs.push_back({staged + l * N, pt + l * N, (int)l, 0});
        JobTable t;
        const NttJob* j = t.add(jobs);
        t.upload(c_, s_);
        ntt_jobs(c_, t.at(j), (int)jobs.size(), true, s_);
    }

    // Many plaintexts at once: coeff[k] holds L limbs of plaintext k (coefficient form); one
    // staged upload and one NTT launch for all of them.
    std::vector<uint64_t*> upload_plains(const std::vector<std::vector<uint64_t>>& coeff, size_t L) {
        const size_t words = L * c_.N;
        return upload_plains_filled(coeff.size(), L, [&](uint64_t* host) {
            for (size_t k = 0; k < coeff.size(); ++k) std::memcpy(host + k * words, coeff[k].data(), words * 8);
        });
    }

    // `count` coefficient-form plaintexts of L limbs written by fill(host) straight into the
    // pinned staging ring ([item][limb][N]), uploaded once and transformed in one NTT launch
    template <class Fill>
    std::vector<uint64_t*> upload_plains_filled(size_t count, size_t L, Fill&& fill) {
        const size_t N = c_.N, words = L * N;
        BatchBuffers& bb = c_.batch_buffers(s_);
        const size_t off = bb.reserve(c_, count * words * 8, s_);
        fill(reinterpret_cast<uint64_t*>(bb.h_ring + off));
        auto* staged = static_cast<uint64_t*>(bb.commit(off, count * words * 8, s_));
        std::vector<uint64_t*> out(count);
        std::vector<NttJob> jobs;
        for (size_t k = 0; k < count; ++k) {
            out[k] = buffer(L, false);
            for (size_t l = 0; l < L; ++l) jobs.push_back({staged + k * words + l * N, out[k] + l * N, (int)l, 0});
        }
        JobTable t;
        const NttJob* j = t.add(jobs);
        t.upload(c_, s_);
        ntt_jobs(c_, t.at(j), (int)jobs.size(), true, s_);
        return out;
    }

    // b += pt (evaluation form, x.level+1 limbs) on every ciphertext (ckks_add_inplace(ct, pt))
    void add_plain(CtBatch& x, const uint64_t* pt) {
        const size_t N = c_.N;
        std::vector<AddJob> jobs;
        for (size_t i = 0; i < count_; ++i)
            for (size_t l = 0; l <= x.level; ++l) jobs.push_back({x.p[i][0] + l * N, pt + l * N, (int)l, 0});
        add_jobs(jobs);
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
        kb_pmul<<<grid_wide(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
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
        kb_pmul<<<grid_wide(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "evalpoly plaintext multiply");
    }

    // b += the encoding of the slot constant re + i im at `scale` (closed form, as in
    // mul_complex_constant), on every ciphertext of the batch.
    void add_complex_constant(CtBatch& x, double re, double im, double scale) {
        add_plain(x, constant_plaintext(x.level + 1, re, im, scale));
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
        const std::vector<uint64_t*> bufs = buffers(count_ * np, level + 1, false);
        for (size_t i = 0; i < count_; ++i) {
            x.p[i] = {nullptr, nullptr, nullptr};
            for (int k = 0; k < np; ++k) x.p[i][k] = bufs[i * np + k];
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
    // Buffers are carved from chunks of stream-ordered memory and all released together when
    // the operation set ends (none is freed earlier), so one allocation serves many buffers.
    static constexpr size_t kFirstChunkWords = size_t{1} << 20;   // 8 MiB
    static constexpr size_t kMaxChunkWords = size_t{1} << 26;     // 512 MiB

    uint64_t* carve(size_t words) {
        words = (words + 31) & ~size_t{31};  // 256-byte alignment
        if (words > left_) {
            WG_SPAN("alloc");
            // power-of-two chunk sizes, so chunks handed back by earlier operation sets fit
            size_t chunk = kFirstChunkWords;
            while (chunk < std::max(words, next_chunk_)) chunk <<= 1;
            next_chunk_ = std::min(next_chunk_ * 2, kMaxChunkWords);
            size_t got = 0;
            uint64_t* p = static_cast<uint64_t*>(c_.take_chunk(chunk * 8, s_, &got));
            if (p) {
                chunk = got / 8;
            } else if (cudaMallocAsync((void**)&p, chunk * 8, s_) != cudaSuccess) {
                cudaGetLastError();
                fail(kNoMemory, "ckks_evalchebyshev: device allocation failed");
            }
            owned_.push_back({p, chunk});
            cur_ = p;
            left_ = chunk;
        }
        uint64_t* p = cur_;
        cur_ += words;
        left_ -= words;
        return p;
    }

    uint64_t* buffer(size_t limbs, bool zero) {
        const size_t words = std::max<size_t>(limbs, 1) * c_.N;
        uint64_t* p = carve(words);
        if (zero) check_cuda(cudaMemsetAsync(p, 0, words * 8, s_), "evalpoly zero");
        return p;
    }

    // n contiguous buffers of `limbs` limbs each, zeroed by one memset when asked
    std::vector<uint64_t*> buffers(size_t n, size_t limbs, bool zero) {
        const size_t words = std::max<size_t>(limbs, 1) * c_.N;
        uint64_t* base = carve(words * std::max<size_t>(n, 1));
        if (zero && n) check_cuda(cudaMemsetAsync(base, 0, words * n * 8, s_), "evalpoly zero");
        std::vector<uint64_t*> out(n);
        for (size_t i = 0; i < n; ++i) out[i] = base + i * words;
        return out;
    }
    uint64_t* scratch(size_t limbs) { return buffer(limbs, false); }

    Context& c_;
    size_t count_;
    cudaStream_t s_;
    std::vector<std::pair<uint64_t*, size_t>> owned_;  // chunks and their sizes in words
    uint64_t* cur_ = nullptr;
    size_t left_ = 0, next_chunk_ = kFirstChunkWords;
    std::map<std::tuple<double, double, double, size_t>, uint64_t*> const_cache_;
};

}  // namespace
}  // namespace wg
