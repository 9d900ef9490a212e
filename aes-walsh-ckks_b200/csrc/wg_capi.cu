// C ABI (include/walsh_gpu.h): argument checks, key registry, workspace routing and the
// operation sequences of rotation, conjugation, relinearization and the batched workload.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_encode.hpp"
#include "wg_evalmod_fit.hpp"
#include "wg_dftplan.hpp"
#include "wg_ctwire.hpp"
#include "wg_internal.hpp"
#include "wg_serve.hpp"

namespace wg {
Context* create_context(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np, size_t dnum,
                        int device);
}

struct wg_lt_stage {
    wg::LtStage* s;
};

namespace {

thread_local std::string g_err;

template <class F>
int guard(F&& f) {
    try {
        f();
        g_err.clear();
        return WG_OK;
    } catch (const wg::Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return WG_ERR_INVALID;
    } catch (const std::exception& e) {
        g_err = e.what();
        return WG_ERR_RUNTIME;
    } catch (...) {
        g_err = "unknown error";
        return WG_ERR_RUNTIME;
    }
}

wg::Context& C(wg_context* h) {
    if (!h || !h->c) wg::fail(wg::kInvalid, "null context");
    return *h->c;
}

cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int64_t normalize_rotation(const wg::Context& c, int64_t r) {
    const int64_t slots = (int64_t)(c.N / 2);
    r %= slots;
    if (r < 0) r += slots;
    return r;
}

uint64_t rotation_galois(const wg::Context& c, int64_t r) { return wg::host::powmod(5, (uint64_t)r, 2 * c.N); }

void check_level(const wg::Context& c, size_t level, const char* who) {
    if (level >= c.nq) wg::fail(wg::kInvalid, std::string(who) + ": invalid ciphertext level");
}
void check_ptr(const void* p, const char* who) {
    if (!p) wg::fail(wg::kInvalid, std::string(who) + ": null buffer");
}

bool stream_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (s) cudaStreamIsCapturing(s, &cs);
    return cs != cudaStreamCaptureStatusNone;
}

// One key switch of one ciphertext.  Outside stream capture it runs as a batch of one (each
// stage of the switch, all digits included, in a single launch); under capture, stage by stage
// on the stream's reserved workspace (the batched path stages a job table per call).
void switch_one(wg::Context& c, size_t level, const uint64_t* key_term, const wg::KeyEntry& k, const uint64_t* b_in,
                const uint64_t* a_in, uint64_t* b, uint64_t* a, bool a_add, uint64_t galois, cudaStream_t s) {
    if (stream_capturing(s)) {
        wg::keyswitch(c, level, key_term, k, b_in, a_in, b, a, true, a_add, galois, c.workspace(s), s);
        return;
    }
    wg::KsItem it;
    it.level = level;
    it.key_term = key_term;
    it.key = &k;
    it.b_in = b_in;
    it.a_in = a_in;
    it.b = b;
    it.a = a;
    it.b_add = 1;
    it.a_add = a_add ? 1 : 0;
    it.galois = galois;
    wg::batch_keyswitch(c, &it, 1, s);
}

void do_rotate(wg::Context& c, size_t level, uint64_t* b, uint64_t* a, int64_t rotation, cudaStream_t s) {
    const int64_t r = normalize_rotation(c, rotation);
    if (r == 0) return;
    const wg::KeyEntry& k = c.key(WG_KEY_ROTATION, r);
    switch_one(c, level, a, k, b, a, b, a, false, rotation_galois(c, r), s);
}

void do_relin(wg::Context& c, size_t level, uint64_t* c0, uint64_t* c1, const uint64_t* c2, cudaStream_t s) {
    const wg::KeyEntry& k = c.key(WG_KEY_RELIN, 0);
    switch_one(c, level, c2, k, c0, c1, c0, c1, true, 0, s);
}

uint64_t* scratch_after_switch(wg::Context& c, cudaStream_t s) {
    return c.workspace(s) + wg::keyswitch_workspace_words(c, c.nq - 1);
}

void do_rescale(wg::Context& c, size_t level, uint64_t* polys, size_t npolys, size_t stride, cudaStream_t s) {
    uint64_t* ws = scratch_after_switch(c, s);
    for (size_t k = 0; k < npolys; k += 2) {
        const int n = (int)std::min<size_t>(2, npolys - k);
        wg::rescale(c, level, polys + k * stride, n, stride, ws, s);
    }
}

}  // namespace

namespace wg {
void set_last_error(const std::string& m) { g_err = m; }
}  // namespace wg

extern "C" {

const char* wg_last_error(void) { return g_err.c_str(); }
int wg_version(void) { return 100; }

int wg_find_primes(const uint64_t* p_bits, size_t np, const uint64_t* q_bits, size_t nq, uint64_t N,
                   uint64_t* p_out, uint64_t* q_out) {
    return guard([&] {
        if (!N || (N & (N - 1))) wg::fail(wg::kInvalid, "N must be a power of two");
        std::vector<uint64_t> pb(p_bits, p_bits + np), qb(q_bits, q_bits + nq), p, q;
        wg::host::find_primes(pb, qb, N, p, q);
        std::memcpy(p_out, p.data(), np * 8);
        std::memcpy(q_out, q.data(), nq * 8);
    });
}

int wg_encode_slots(uint64_t N, const double* re, const double* im, double scale, const uint64_t* moduli,
                    size_t limbs, uint64_t* out) {
    return guard([&] {
        if (!re || !im || !moduli || !out) wg::fail(wg::kInvalid, "ckks_encode: null argument");
        wg::host::encode_slots(N, re, im, scale, moduli, limbs, out);
    });
}

int wg_ctx_create(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np, size_t dnum, int device,
                  wg_context** out) {
    return guard([&] {
        if (!out || !q || !p) wg::fail(wg::kInvalid, "wg_ctx_create: null argument");
        *out = nullptr;
        wg::Context* c = wg::create_context(N, q, nq, p, np, dnum, device);
        *out = new wg_context{c};
    });
}

void wg_ctx_destroy(wg_context* ctx) {
    if (!ctx) return;
    delete ctx->c;
    delete ctx;
}

int wg_ctx_set_key(wg_context* ctx, int kind, int64_t rotation, const uint64_t* host_key, size_t parts,
                   size_t key_level) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(host_key, "wg_ctx_set_key");
        if (kind < WG_KEY_RELIN || kind > WG_KEY_SPARSE_TO_DENSE) wg::fail(wg::kInvalid, "wg_ctx_set_key: unknown key kind");
        if (key_level >= c.nq) wg::fail(wg::kInvalid, "wg_ctx_set_key: key level out of range");
        const bool compact = kind == WG_KEY_DENSE_TO_SPARSE;
        if (compact && (parts != 1 || key_level != 0))
            wg::fail(wg::kInvalid, "wg_ctx_set_key: the dense-to-sparse key is one level-0 part");
        if (!compact && (parts < c.parts_at(key_level) || parts > 16))
            wg::fail(wg::kInvalid, "wg_ctx_set_key: invalid part count");
        const int64_t r = kind == WG_KEY_ROTATION ? normalize_rotation(c, rotation) : 0;
        if (kind == WG_KEY_ROTATION && r == 0) wg::fail(wg::kInvalid, "wg_ctx_set_key: zero rotation needs no key");
        const size_t words = compact ? 4 * c.N : parts * 2 * (key_level + 1 + c.np) * c.N;
        wg::KeyEntry e;
        e.parts = parts;
        e.key_level = key_level;
        wg::check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
        if (cudaMalloc(&e.d_data, words * 8) != cudaSuccess) {
            cudaGetLastError();
            wg::fail(wg::kNoMemory, "wg_ctx_set_key: device allocation failed");
        }
        if (cudaMemcpy(e.d_data, host_key, words * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(e.d_data);
            wg::fail(wg::kCuda, "wg_ctx_set_key: upload failed");
        }
        auto it = c.keys.find({kind, r});
        if (it != c.keys.end()) {
            cudaFree(it->second.d_data);
            it->second = e;
        } else {
            c.keys.emplace(std::make_pair(kind, r), e);
        }
    });
}

int wg_keygen_switch_key(wg_context* ctx, int kind, int64_t rotation, const int8_t* secret, const uint64_t* a,
                           const int64_t* e, uint64_t seed, double sigma, uint64_t* out, void* stream) {
    return guard([&] { wg::keygen_switch_key(C(ctx), kind, rotation, secret, a, e, seed, sigma, out, S(stream)); });
}

int wg_keygen_secret_switch(wg_context* ctx, int kind, const int8_t* source, const int8_t* target, const uint64_t* a,
                            const int64_t* e, uint64_t seed, double sigma, uint64_t* out, void* stream) {
    return guard([&] { wg::keygen_secret_switch(C(ctx), kind, source, target, a, e, seed, sigma, out, S(stream)); });
}

int wg_ctx_has_key(const wg_context* ctx, int kind, int64_t rotation) {
    if (!ctx || !ctx->c) return 0;
    const int64_t r = kind == WG_KEY_ROTATION ? normalize_rotation(*ctx->c, rotation) : 0;
    if (kind == WG_KEY_ROTATION && r == 0) return 1;
    return ctx->c->keys.count({kind, r}) ? 1 : 0;
}

int wg_ctx_reserve(wg_context* ctx, void* stream) {
    return guard([&] { C(ctx).workspace(S(stream)); });
}

size_t wg_ctx_workspace_words(const wg_context* ctx) { return ctx && ctx->c ? ctx->c->workspace_words() : 0; }

static int ntt_call(wg_context* ctx, uint64_t* poly, size_t limbs, size_t first, int basis, size_t polys,
                    size_t stride, void* stream, bool fwd) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(poly, "ntt");
        const size_t avail = basis ? c.np : c.nq;
        if (basis != 0 && basis != 1) wg::fail(wg::kInvalid, "ntt: basis must be 0 (Q) or 1 (P)");
        if (first + limbs > avail) wg::fail(wg::kInvalid, "ntt: limb range exceeds the modulus chain");
        if (polys > 1 && stride < limbs * c.N) wg::fail(wg::kInvalid, "ntt: polynomial stride too small");
        const wg::LimbMap map = basis ? wg::LimbMap{0, 0, (int)(c.nq + first)} : wg::LimbMap{(int)limbs, (int)first, 0};
        if (fwd)
            wg::ntt_forward(c, poly, (int)limbs, (int)polys, stride, map, S(stream));
        else
            wg::ntt_inverse(c, poly, (int)limbs, (int)polys, stride, map, S(stream));
    });
}

int wg_ntt_forward(wg_context* ctx, uint64_t* poly, size_t limbs, size_t first, int basis, size_t polys,
                   size_t poly_stride, void* stream) {
    return ntt_call(ctx, poly, limbs, first, basis, polys, poly_stride, stream, true);
}
int wg_ntt_inverse(wg_context* ctx, uint64_t* poly, size_t limbs, size_t first, int basis, size_t polys,
                   size_t poly_stride, void* stream) {
    return ntt_call(ctx, poly, limbs, first, basis, polys, poly_stride, stream, false);
}

size_t wg_ct_wire_bytes(uint64_t N, size_t level, size_t npolys) { return wg::ct_wire_bytes(N, level, npolys); }

int wg_ct_wire_encode(uint64_t N, const uint64_t* q, size_t level, size_t npolys, const uint64_t* polys, double scale,
                      int secret_owner, int encoding_state, uint8_t* out, size_t cap) {
    return guard([&] {
        if (!q || !polys || !out) wg::fail(wg::kInvalid, "ciphertext wire: null argument");
        if (npolys == 0 || npolys > 3 || (secret_owner & ~1) || (encoding_state & ~1))
            wg::fail(wg::kInvalid, "ciphertext wire: invalid polynomial count or labels");
        wg::CtRecord r;
        r.N = N;
        r.level = level;
        r.npolys = npolys;
        r.scale = scale;
        r.owner = (uint8_t)secret_owner;
        r.state = (uint8_t)encoding_state;
        r.q.assign(q, q + level + 1);
        r.polys.assign(polys, polys + npolys * (level + 1) * N);
        wg::ct_wire_encode(r, out, cap);
    });
}

int wg_ct_wire_decode(const uint8_t* in, size_t len, uint64_t N, const uint64_t* q, size_t nq, uint64_t* polys,
                      size_t cap_words, size_t* level, size_t* npolys, double* scale, int* secret_owner,
                      int* encoding_state) {
    return guard([&] {
        if (!in || !q || !polys) wg::fail(wg::kInvalid, "ciphertext wire: null argument");
        const wg::CtRecord r = wg::ct_wire_decode(in, len);
        if (r.N != N) wg::fail(wg::kInvalid, "ciphertext wire: ring degree differs from the context's");
        if (r.level >= nq || !std::equal(r.q.begin(), r.q.end(), q))
            wg::fail(wg::kInvalid, "ciphertext wire: moduli differ from the context's");
        if (r.polys.size() > cap_words) wg::fail(wg::kInvalid, "ciphertext wire: output buffer too small");
        std::copy(r.polys.begin(), r.polys.end(), polys);
        if (level) *level = r.level;
        if (npolys) *npolys = r.npolys;
        if (scale) *scale = r.scale;
        if (secret_owner) *secret_owner = r.owner;
        if (encoding_state) *encoding_state = r.state;
    });
}

int wg_evalmod_fit(double K, size_t degree, size_t double_angle, double interval_radius, size_t validation_points,
                   double prune_threshold, double* coeffs, size_t* ncoeffs, double* max_error, double* interval) {
    return guard([&] {
        if (!coeffs || !ncoeffs) wg::fail(wg::kInvalid, "evalmod fit: null output");
        const wg::fit::EvalModFit f =
            wg::fit::fit_evalmod(K, degree, double_angle, interval_radius, validation_points, prune_threshold);
        if (f.coeffs.size() > degree + 1) wg::fail(wg::kRuntime, "evalmod fit: more coefficients than degree + 1");
        std::copy(f.coeffs.begin(), f.coeffs.end(), coeffs);
        *ncoeffs = f.coeffs.size();
        if (max_error) *max_error = f.max_error;
        if (interval) {
            interval[0] = f.interval_min;
            interval[1] = f.interval_max;
        }
    });
}

int wg_evalmod_k_bound(size_t coefficients, size_t hamming_weight, double log2_failure, size_t* k) {
    return guard([&] {
        if (!k) wg::fail(wg::kInvalid, "evalmod K bound: null output");
        *k = wg::fit::evalmod_k_bound(coefficients, hamming_weight, std::exp2((long double)log2_failure));
    });
}

int wg_ntt_tuning(const wg_context* ctx, int* chosen, float* ms, int* limbs) {
    return guard([&] {
        if (!ctx || !ctx->c) wg::fail(wg::kInvalid, "null context");
        const wg::Context& c = *ctx->c;
        for (int d = 0; d < 2; ++d)
            for (int p = 0; p < 2; ++p) {
                if (chosen) chosen[d * 2 + p] = c.ntt_variant[d][p];
                for (int v = 0; v < wg::kNttGeometries && ms; ++v) ms[(d * 2 + p) * wg::kNttGeometries + v] = c.tuning.ms[d][p][v];
            }
        if (limbs) *limbs = c.tuning.limbs;
    });
}

int wg_ntt_set_geometry(wg_context* ctx, int direction, int phase, int geometry) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (direction < 0 || direction > 1 || phase < 0 || phase > 1) wg::fail(wg::kInvalid, "ntt: invalid direction or phase");
        if (geometry >= wg::kNttGeometries) wg::fail(wg::kInvalid, "ntt: unknown geometry");
        c.ntt_variant[direction][phase] = geometry < 0 ? c.tuning.chosen[direction][phase] : geometry;
    });
}

int wg_ctx_trim(wg_context* ctx, void* stream) {
    return guard([&] { C(ctx).trim(S(stream)); });
}

int wg_set_ntt_fusion(wg_context* ctx, int mode) {
    return guard([&] {
        if (mode < 0 || mode > 2) wg::fail(wg::kInvalid, "ntt fusion: mode must be 0, 1 or 2");
        C(ctx).ntt_fusion = mode;
    });
}

int wg_keyswitch(wg_context* ctx, size_t level, const uint64_t* key_term, int kind, int64_t rotation, uint64_t* b,
                 uint64_t* a, int b_add, int a_add, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_level(c, level, "ckks_hybrid_keyswitch");
        check_ptr(key_term, "ckks_hybrid_keyswitch");
        check_ptr(b, "ckks_hybrid_keyswitch");
        check_ptr(a, "ckks_hybrid_keyswitch");
        const int64_t r = kind == WG_KEY_ROTATION ? normalize_rotation(c, rotation) : 0;
        const wg::KeyEntry& k = c.key(kind, r);
        wg::keyswitch(c, level, key_term, k, b, a, b, a, b_add != 0, a_add != 0, 0, c.workspace(S(stream)),
                      S(stream));
    });
}

int wg_rotate(wg_context* ctx, size_t level, uint64_t* b, uint64_t* a, int64_t rotation, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_level(c, level, "ckks_rotate");
        check_ptr(b, "ckks_rotate");
        check_ptr(a, "ckks_rotate");
        do_rotate(c, level, b, a, rotation, S(stream));
    });
}

int wg_conjugate(wg_context* ctx, size_t level, uint64_t* b, uint64_t* a, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_level(c, level, "ckks_conjugate");
        check_ptr(b, "ckks_conjugate");
        check_ptr(a, "ckks_conjugate");
        const wg::KeyEntry& k = c.key(WG_KEY_CONJ, 0);
        const size_t n = (level + 1) * c.N;
        uint64_t* pb = scratch_after_switch(c, S(stream));
        uint64_t* pa = pb + n;
        const uint64_t g = 2 * c.N - 1;
        wg::automorphism(c, b, pb, (int)(level + 1), 1, 0, g, S(stream));
        wg::automorphism(c, a, pa, (int)(level + 1), 1, 0, g, S(stream));
        wg::keyswitch(c, level, pa, k, pb, pa, b, a, true, false, 0, c.workspace(S(stream)), S(stream));
    });
}

int wg_rotate_many(wg_context* ctx, size_t level, const uint64_t* b, const uint64_t* a, const int64_t* rotations,
                   size_t nrot, uint64_t* out, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_level(c, level, "ckks_rotate");
        check_ptr(b, "ckks_rotate");
        check_ptr(a, "ckks_rotate");
        check_ptr(out, "ckks_rotate");
        if (nrot && !rotations) wg::fail(wg::kInvalid, "ckks_rotate: null rotation list");
        wg::rotate_many(c, level, b, a, rotations, nrot, out, S(stream));
    });
}

int wg_mul(wg_context* ctx, size_t level, uint64_t* b1, uint64_t* a1, const uint64_t* b2, const uint64_t* a2,
           uint64_t* c2, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_level(c, level, "ckks_mul_inplace(ct,ct)");
        for (const void* p : {(const void*)b1, (const void*)a1, (const void*)b2, (const void*)a2, (const void*)c2})
            check_ptr(p, "ckks_mul_inplace(ct,ct)");
        wg::tensor(c, level, b1, a1, b2, a2, c2, S(stream));
    });
}

int wg_relin(wg_context* ctx, size_t level, uint64_t* c0, uint64_t* c1, const uint64_t* c2, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_level(c, level, "ckks_relin");
        check_ptr(c0, "ckks_relin");
        check_ptr(c1, "ckks_relin");
        check_ptr(c2, "ckks_relin");
        do_relin(c, level, c0, c1, c2, S(stream));
    });
}

int wg_rescale(wg_context* ctx, size_t level, uint64_t* polys, size_t npolys, size_t poly_stride, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (level == 0 || level >= c.nq) wg::fail(wg::kInvalid, "ckks_rescale: invalid level");
        check_ptr(polys, "ckks_rescale");
        if (npolys == 0) wg::fail(wg::kInvalid, "ckks_rescale: empty ciphertext");
        if (npolys > 1 && poly_stride < (level + 1) * c.N) wg::fail(wg::kInvalid, "ckks_rescale: stride too small");
        do_rescale(c, level, polys, npolys, poly_stride, S(stream));
    });
}

static int add_sub_call(wg_context* ctx, size_t level, uint64_t* x, const uint64_t* y, size_t npolys, size_t stride,
                        void* stream, bool sub) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_level(c, level, sub ? "ckks_sub_inplace" : "ckks_add_inplace");
        check_ptr(x, "ckks_add_inplace");
        check_ptr(y, "ckks_add_inplace");
        if (npolys > 1 && stride < (level + 1) * c.N) wg::fail(wg::kInvalid, "ckks_add_inplace: stride too small");
        wg::add_sub(c, level, x, y, (int)npolys, stride, sub, S(stream));
    });
}
int wg_add(wg_context* ctx, size_t level, uint64_t* x, const uint64_t* y, size_t npolys, size_t poly_stride,
           void* stream) {
    return add_sub_call(ctx, level, x, y, npolys, poly_stride, stream, false);
}
int wg_sub(wg_context* ctx, size_t level, uint64_t* x, const uint64_t* y, size_t npolys, size_t poly_stride,
           void* stream) {
    return add_sub_call(ctx, level, x, y, npolys, poly_stride, stream, true);
}

static void check_batch(wg::Context& c, size_t count, const size_t* levels, uint64_t* const* xb,
                        uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                        const int64_t* rots) {
    if (count && (!levels || !xb || !xa || !yb || !ya || !rots)) wg::fail(wg::kInvalid, "batch: null array");
    for (size_t i = 0; i < count; ++i) {
        if (levels[i] == 0 || levels[i] >= c.nq) wg::fail(wg::kInvalid, "batch: ciphertext level must be in [1, L)");
        for (const void* p : {(const void*)xb[i], (const void*)xa[i], (const void*)yb[i], (const void*)ya[i]})
            check_ptr(p, "batch");
        const int64_t r = normalize_rotation(c, rots[i]);
        if (r) c.key(WG_KEY_ROTATION, r);
    }
    c.key(WG_KEY_RELIN, 0);
}

int wg_batch_mul_relin_rescale_rotate(wg_context* ctx, size_t count, const size_t* levels, uint64_t* const* xb,
                                      uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                                      const int64_t* rots, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_batch(c, count, levels, xb, xa, yb, ya, rots);
        std::vector<uint64_t> galois(count);
        std::vector<const wg::KeyEntry*> keys(count, nullptr);
        for (size_t i = 0; i < count; ++i) {
            const int64_t r = normalize_rotation(c, rots[i]);
            galois[i] = r ? rotation_galois(c, r) : 0;
            if (r) keys[i] = &c.key(WG_KEY_ROTATION, r);
        }
        wg::batch_mul_relin_rescale_rotate(c, count, levels, xb, xa, yb, ya, rots, galois.data(),
                                           &c.key(WG_KEY_RELIN, 0), keys.data(), S(stream));
    });
}

static void check_cts(wg::Context& c, size_t count, uint64_t* const* b, uint64_t* const* a, const char* who) {
    if (count && (!b || !a)) wg::fail(wg::kInvalid, std::string(who) + ": null array");
    for (size_t i = 0; i < count; ++i) {
        check_ptr(b[i], who);
        check_ptr(a[i], who);
    }
}

static void check_key_bits(const uint64_t* const* key_b, const uint64_t* const* key_a, size_t count) {
    if (!key_b || !key_a) wg::fail(wg::kInvalid, "ckks_aes: null key bits");
    for (size_t k = 0; k < count; ++k) {
        check_ptr(key_b[k], "ckks_aes");
        check_ptr(key_a[k], "ckks_aes");
    }
}

int wg_modraise(wg_context* ctx, size_t count, size_t target_level, uint64_t* const* b, uint64_t* const* a,
                void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (target_level == 0 || target_level >= c.nq)
            wg::fail(wg::kInvalid, "ckks_modraise: target level must be in [1, max_level]");
        check_cts(c, count, b, a, "ckks_modraise");
        wg::modraise(c, count, target_level, b, a, S(stream));
    });
}

int wg_dense_to_sparse(wg_context* ctx, size_t count, uint64_t* const* b, uint64_t* const* a, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_cts(c, count, b, a, "ckks_key_switch");
        const wg::KeyEntry& k = c.key(WG_KEY_DENSE_TO_SPARSE, 0);
        wg::q0p0_switch(c, count, b, a, k, S(stream));
    });
}

int wg_sparse_to_dense(wg_context* ctx, size_t count, const size_t* levels, uint64_t* const* b,
                       uint64_t* const* a, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_cts(c, count, b, a, "ckks_key_switch");
        if (count && !levels) wg::fail(wg::kInvalid, "ckks_key_switch: null levels");
        const wg::KeyEntry& k = c.key(WG_KEY_SPARSE_TO_DENSE, 0);
        std::vector<wg::KsItem> items(count);
        for (size_t i = 0; i < count; ++i) {
            check_level(c, levels[i], "ckks_key_switch");
            wg::KsItem& it = items[i];
            it.level = levels[i];
            it.key_term = a[i];
            it.key = &k;
            it.b_in = b[i];
            it.a_in = a[i];
            it.b = b[i];
            it.a = a[i];
            it.b_add = 1;
            it.a_add = 0;
            it.galois = 0;
        }
        wg::batch_keyswitch(c, items.data(), count, S(stream));
    });
}

int wg_evalchebyshev(wg_context* ctx, size_t count, size_t level, double scale, const double* coeffs,
                     size_t ncoeffs, double target_scale, double default_scale, uint64_t* const* b,
                     uint64_t* const* a, uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level,
                     double* out_scale, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_cts(c, count, b, a, "ckks_evalchebyshev");
        check_cts(c, count, out_b, out_a, "ckks_evalchebyshev");
        check_ptr(coeffs, "ckks_evalchebyshev");
        check_ptr(out_level, "ckks_evalchebyshev");
        check_ptr(out_scale, "ckks_evalchebyshev");
        wg::evalchebyshev(c, count, level, scale, coeffs, ncoeffs, target_scale, default_scale, b, a, out_b, out_a,
                          out_level, out_scale, S(stream));
    });
}

static wg::BootstrapParams boot_args(const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                                     const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs,
                                     std::vector<const wg::LtStage*>& vs, std::vector<const wg::LtStage*>& vc) {
    check_ptr(params, "ckks EvalMod");
    check_ptr(coeffs, "ckks EvalMod");
    if ((ns2c && !s2c) || (nc2s && !c2s)) wg::fail(wg::kInvalid, "ckks EvalMod: null stage list");
    vs.resize(ns2c);
    vc.resize(nc2s);
    for (size_t k = 0; k < ns2c; ++k) {
        check_ptr(s2c[k], "ckks EvalMod");
        vs[k] = s2c[k]->s;
    }
    for (size_t k = 0; k < nc2s; ++k) {
        check_ptr(c2s[k], "ckks EvalMod");
        vc[k] = c2s[k]->s;
    }
    wg::BootstrapParams bp;
    bp.s2c_depth = params->s2c_depth;
    bp.depth = params->depth;
    bp.evalmod_log_scale = params->evalmod_log_scale;
    bp.double_angle = params->double_angle;
    bp.active_slots = params->active_slots;
    bp.slots = params->slots;
    bp.scale = params->scale;
    if (bp.active_slots == 0 || bp.slots == 0 || bp.active_slots > bp.slots)
        wg::fail(wg::kInvalid, "ckks EvalMod: invalid slot counts");
    return bp;
}

int wg_bootstrap_evalmod(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                         size_t ns2c, const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs,
                         size_t ncoeffs, size_t count, uint64_t* const* b, uint64_t* const* a,
                         uint64_t* const* out0_b, uint64_t* const* out0_a, uint64_t* const* out1_b,
                         uint64_t* const* out1_a, size_t* out_level, double* out_scale, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out_level, "ckks EvalMod");
        check_ptr(out_scale, "ckks EvalMod");
        check_cts(c, count, b, a, "ckks EvalMod");
        check_cts(c, count, out0_b, out0_a, "ckks EvalMod");
        check_cts(c, count, out1_b, out1_a, "ckks EvalMod");
        std::vector<const wg::LtStage*> vs, vc;
        const wg::BootstrapParams bp = boot_args(params, s2c, ns2c, c2s, nc2s, coeffs, vs, vc);
        const wg::S2cPlan plan{1, vs.data(), ns2c};
        wg::bootstrap_evalmod(c, bp, &plan, 1, vc.data(), nc2s, coeffs, ncoeffs, count, bp.scale, b, a, out0_b, out0_a,
                              out1_b, out1_a, out_level, out_scale, S(stream));
    });
}

int wg_walsh_sbox(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                  const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                  size_t block_count, size_t count, size_t level, double scale, uint64_t* const* in_b,
                  uint64_t* const* in_a, uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level,
                  double* out_scale, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out_level, "ckks_walsh_sbox");
        check_ptr(out_scale, "ckks_walsh_sbox");
        check_cts(c, 8 * count, in_b, in_a, "ckks_walsh_sbox");
        check_cts(c, 8 * count, out_b, out_a, "ckks_walsh_sbox");
        std::vector<const wg::LtStage*> vs, vc;
        const wg::BootstrapParams bp = boot_args(params, s2c, ns2c, c2s, nc2s, coeffs, vs, vc);
        const wg::S2cPlan plan{1, vs.data(), ns2c};
        wg::walsh_sbox(c, bp, &plan, 1, vc.data(), nc2s, coeffs, ncoeffs, block_count, count, level, scale, in_b, in_a,
                       out_b, out_a, out_level, out_scale, S(stream));
    });
}

static int aes_ctr_walsh_call(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                              size_t ns2c, const wg_lt_stage* const* s2c_x2, size_t ns2c_x2,
                              const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                              size_t packing_block_count, size_t packed_segment_count, const uint64_t* const* key_b,
                              const uint64_t* const* key_a, const double* key_scales, size_t key_level,
                              const uint8_t* counters, const uint8_t* ciphertexts, size_t active_blocks,
                              uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                              void* stream, bool per_instance) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out_level, "ckks_aes_walsh");
        check_ptr(out_scale, "ckks_aes_walsh");
        check_cts(c, 128, out_b, out_a, "ckks_aes_walsh");
        if (!key_b || !key_a) wg::fail(wg::kInvalid, "ckks_aes_walsh: null key bits");
        for (size_t k = 0; k < 1408; ++k) {
            check_ptr(key_b[k], "ckks_aes_walsh");
            check_ptr(key_a[k], "ckks_aes_walsh");
        }
        std::vector<const wg::LtStage*> vs, vc, vs2(ns2c_x2);
        const wg::BootstrapParams bp = boot_args(params, s2c, ns2c, c2s, nc2s, coeffs, vs, vc);
        if (ns2c_x2 && !s2c_x2) wg::fail(wg::kInvalid, "ckks_aes_walsh: null stage list");
        for (size_t k = 0; k < ns2c_x2; ++k) {
            check_ptr(s2c_x2[k], "ckks_aes_walsh");
            vs2[k] = s2c_x2[k]->s;
        }
        const wg::S2cPlan plans[2] = {{1, vs.data(), ns2c}, {2, vs2.data(), ns2c_x2}};
        wg::AesArgs a;
        a.key_b = key_b;
        a.key_a = key_a;
        a.key_scales = key_scales;
        a.key_level = key_level;
        a.counters = counters;
        a.ciphertexts = ciphertexts;
        a.active_blocks = active_blocks;
        a.packing_block_count = packing_block_count;
        a.packed_segment_count = packed_segment_count;
        a.per_instance = per_instance;
        wg::aes_ctr_walsh(c, bp, plans, ns2c_x2 ? 2 : 1, vc.data(), nc2s, coeffs, ncoeffs, a, out_b, out_a, out_level,
                          out_scale, S(stream));
    });
}

int wg_aes_ctr_walsh(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                     size_t ns2c, const wg_lt_stage* const* s2c_x2, size_t ns2c_x2,
                     const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                     size_t packing_block_count, size_t packed_segment_count, const uint64_t* const* key_b,
                     const uint64_t* const* key_a, const double* key_scales, size_t key_level,
                     const uint8_t* counters, const uint8_t* ciphertexts, size_t active_blocks,
                     uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                     void* stream) {
    return aes_ctr_walsh_call(ctx, params, s2c, ns2c, s2c_x2, ns2c_x2, c2s, nc2s, coeffs, ncoeffs, packing_block_count,
                              packed_segment_count, key_b, key_a, key_scales, key_level, counters, ciphertexts,
                              active_blocks, out_b, out_a, out_level, out_scale, stream, false);
}

int wg_aes_ctr_walsh_plain(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                           size_t ns2c, const wg_lt_stage* const* s2c_x2, size_t ns2c_x2,
                           const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                           size_t packing_block_count, size_t packed_segment_count, const uint64_t* const* key_b,
                           const uint64_t* const* key_a, const double* key_scales, size_t key_level,
                           const uint8_t* counters, const uint8_t* ciphertexts, size_t active_blocks,
                           uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                           void* stream) {
    return aes_ctr_walsh_call(ctx, params, s2c, ns2c, s2c_x2, ns2c_x2, c2s, nc2s, coeffs, ncoeffs, packing_block_count,
                              packed_segment_count, key_b, key_a, key_scales, key_level, counters, ciphertexts,
                              active_blocks, out_b, out_a, out_level, out_scale, stream, true);
}

int wg_xboot_sbox(wg_context* ctx, size_t count, size_t level, double scale, uint64_t* const* in_b,
                  uint64_t* const* in_a, uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level,
                  double* out_scale, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out_level, "ckks_aes");
        check_ptr(out_scale, "ckks_aes");
        if (level >= c.nq) wg::fail(wg::kInvalid, "ckks_aes: invalid XBOOT S-box input level");
        check_cts(c, 8 * count, in_b, in_a, "ckks_aes");
        check_cts(c, 8 * count, out_b, out_a, "ckks_aes");
        wg::xboot_sbox(c, count, level, scale, in_b, in_a, out_b, out_a, out_level, out_scale, S(stream));
    });
}

int wg_bootstrap_pair(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                      const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs, size_t count,
                      double scale, uint64_t* const* b0, uint64_t* const* a0, uint64_t* const* b1,
                      uint64_t* const* a1, size_t* out_level, double* out_scale, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out_level, "ckks_batch_bootstrap_evalmod");
        check_ptr(out_scale, "ckks_batch_bootstrap_evalmod");
        check_cts(c, count, b0, a0, "ckks_batch_bootstrap_evalmod");
        check_cts(c, count, b1, a1, "ckks_batch_bootstrap_evalmod");
        std::vector<const wg::LtStage*> vs, vc;
        const wg::BootstrapParams bp = boot_args(params, s2c, ns2c, c2s, nc2s, coeffs, vs, vc);
        const wg::S2cPlan plan{1, vs.data(), ns2c};
        wg::bootstrap_pair(c, bp, &plan, 1, vc.data(), nc2s, coeffs, ncoeffs, count, scale, b0, a0, b1, a1, out_level,
                           out_scale, S(stream));
    });
}

int wg_aes_ctr_xboot(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                     const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs,
                     const uint64_t* const* key_b, const uint64_t* const* key_a, const double* key_scales,
                     const size_t* key_levels, const uint8_t* counters, const uint8_t* ciphertexts, size_t blocks,
                     uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale,
                     void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out_level, "ckks_aes");
        check_ptr(out_scale, "ckks_aes");
        check_ptr(key_scales, "ckks_aes");
        check_ptr(key_levels, "ckks_aes");
        check_ptr(counters, "ckks_aes");
        check_ptr(ciphertexts, "ckks_aes");
        check_cts(c, 128, out_b, out_a, "ckks_aes");
        if (!key_b || !key_a) wg::fail(wg::kInvalid, "ckks_aes: null key bits");
        for (size_t k = 0; k < 1408; ++k) {
            check_ptr(key_b[k], "ckks_aes");
            check_ptr(key_a[k], "ckks_aes");
        }
        std::vector<const wg::LtStage*> vs, vc;
        const wg::BootstrapParams bp = boot_args(params, s2c, ns2c, c2s, nc2s, coeffs, vs, vc);
        const wg::S2cPlan plan{1, vs.data(), ns2c};
        wg::XbootAesArgs a;
        a.key_b = key_b;
        a.key_a = key_a;
        a.key_scales = key_scales;
        a.key_levels = key_levels;
        a.counters = counters;
        a.ciphertexts = ciphertexts;
        a.blocks = blocks;
        wg::aes_ctr_xboot(c, bp, &plan, 1, vc.data(), nc2s, coeffs, ncoeffs, a, out_b, out_a, out_level, out_scale,
                          S(stream));
    });
}

int wg_xboot_initial_state(wg_context* ctx, const wg_bootstrap_params* params, const uint64_t* const* key_b,
                           const uint64_t* const* key_a, const double* key_scales, const size_t* key_levels,
                           const uint8_t* counters, size_t blocks, uint64_t* const* out_b, uint64_t* const* out_a,
                           size_t* out_level, double* out_scale, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(params, "ckks_aes");
        check_ptr(key_scales, "ckks_aes");
        check_ptr(key_levels, "ckks_aes");
        check_ptr(counters, "ckks_aes");
        check_ptr(out_level, "ckks_aes");
        check_ptr(out_scale, "ckks_aes");
        check_cts(c, 128, out_b, out_a, "ckks_aes");
        check_key_bits(key_b, key_a, 128);
        wg::BootstrapParams bp;
        bp.active_slots = params->active_slots;
        bp.slots = params->slots;
        bp.scale = params->scale;
        if (bp.active_slots == 0 || bp.active_slots > c.N / 2) wg::fail(wg::kInvalid, "ckks_aes: invalid slot counts");
        wg::XbootAesArgs a;
        a.key_b = key_b;
        a.key_a = key_a;
        a.key_scales = key_scales;
        a.key_levels = key_levels;
        a.counters = counters;
        a.blocks = blocks;
        wg::xboot_initial_state(c, bp, a, out_b, out_a, out_level, out_scale, S(stream));
    });
}

int wg_xboot_linear_layer(wg_context* ctx, size_t level, const double* in_scale, uint64_t* const* in_b,
                          uint64_t* const* in_a, const uint64_t* const* key_b, const uint64_t* const* key_a,
                          const size_t* key_levels, int mix, uint64_t* const* out_b, uint64_t* const* out_a,
                          double* out_scale, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(in_scale, "ckks_aes");
        check_ptr(key_levels, "ckks_aes");
        check_ptr(out_scale, "ckks_aes");
        check_cts(c, 128, in_b, in_a, "ckks_aes");
        check_key_bits(key_b, key_a, 128);
        check_cts(c, 128, out_b, out_a, "ckks_aes");
        for (size_t k = 0; k < 128; ++k)
            if (in_b[k] == out_b[k] || in_a[k] == out_a[k] || in_b[k] == out_a[k] || in_a[k] == out_b[k])
                wg::fail(wg::kInvalid, "ckks_aes: linear layer outputs must not alias its inputs");
        wg::XbootAesArgs a;
        a.key_b = key_b;
        a.key_a = key_a;
        a.key_levels = key_levels;
        wg::xboot_linear_layer(c, level, in_scale, in_b, in_a, a, mix != 0, out_b, out_a, out_scale, S(stream));
    });
}

int wg_encrypt_symmetric(wg_context* ctx, size_t count, size_t level, const uint64_t* const* pts, const int8_t* secret,
                         const uint64_t* a, const int64_t* e, uint64_t seed, double sigma, uint64_t* const* out_b,
                         uint64_t* const* out_a, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_cts(c, count, out_b, out_a, "ckks_encrypt");
        if (count && !pts) wg::fail(wg::kInvalid, "ckks_encrypt: null plaintext array");
        for (size_t i = 0; i < count; ++i) check_ptr(pts[i], "ckks_encrypt");
        wg::encrypt_symmetric(c, count, level, pts, secret, a, e, seed, sigma, out_b, out_a, S(stream));
    });
}

int wg_aes_xboot_encrypt_round_key_bits(wg_context* ctx, const wg_bootstrap_params* params,
                                        const uint8_t* expanded_key, size_t first_round_key_level,
                                        const int8_t* secret, uint64_t seed, double sigma, uint64_t* const* out_b,
                                        uint64_t* const* out_a, double* out_scale, size_t* out_level, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(params, "ckks_aes");
        check_ptr(out_scale, "ckks_aes");
        check_ptr(out_level, "ckks_aes");
        check_cts(c, 1408, out_b, out_a, "ckks_aes");
        wg::BootstrapParams bp;
        bp.s2c_depth = params->s2c_depth;
        bp.scale = params->scale;
        if (!(bp.scale > 0.0)) wg::fail(wg::kInvalid, "ckks_aes: invalid scale");
        wg::xboot_encrypt_round_key_bits(c, bp, expanded_key, first_round_key_level, secret, seed, sigma, out_b, out_a,
                                         out_scale, out_level, S(stream));
    });
}

int wg_encode_slots_device(wg_context* ctx, size_t count, size_t limbs, double scale, const double* re, const double* im,
                    uint64_t* const* out, int eval, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (count && !out) wg::fail(wg::kInvalid, "ckks_encode: null output array");
        for (size_t i = 0; i < count; ++i) check_ptr(out[i], "ckks_encode");
        wg::encode_slots_device(c, count, limbs, scale, re, im, out, eval != 0, S(stream));
    });
}

int wg_bundle_save(wg_context* ctx, const char* path, const wg_lt_stage* const* stages, size_t nstages) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(path, "wg_bundle");
        if (nstages && !stages) wg::fail(wg::kInvalid, "wg_bundle: null stage list");
        wg::Bundle b;
        b.N = c.N;
        b.dnum = c.dnum;
        b.q.assign(c.q.begin(), c.q.end());
        b.p.assign(c.p.begin(), c.p.end());
        wg::check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
        wg::check_cuda(cudaDeviceSynchronize(), "wg_bundle");
        for (const auto& [id, e] : c.keys) {
            wg::BundleKey k;
            k.kind = id.first;
            k.rotation = id.second;
            k.parts = e.parts;
            k.key_level = e.key_level;
            const size_t words = id.first == WG_KEY_DENSE_TO_SPARSE ? 4 * c.N
                                                                    : e.parts * 2 * (e.key_level + 1 + c.np) * c.N;
            k.data.resize(words);
            wg::check_cuda(cudaMemcpy(k.data.data(), e.d_data, words * 8, cudaMemcpyDeviceToHost), "wg_bundle: key download");
            b.keys.push_back(std::move(k));
        }
        for (size_t i = 0; i < nstages; ++i) {
            check_ptr(stages[i], "wg_bundle");
            b.stages.emplace_back();
            wg::lt_stage_export(c, *stages[i]->s, b.stages.back());
        }
        const std::vector<uint8_t> bytes = wg::bundle_encode(b);
        FILE* f = std::fopen(path, "wb");
        if (!f) wg::fail(wg::kRuntime, std::string("wg_bundle: cannot open ") + path);
        const size_t written = std::fwrite(bytes.data(), 1, bytes.size(), f);
        const bool ok = written == bytes.size() && std::fclose(f) == 0;
        if (!ok) wg::fail(wg::kRuntime, std::string("wg_bundle: write failed: ") + path);
    });
}

int wg_bundle_load(wg_context* ctx, const char* path, wg_lt_stage** stages, size_t max_stages, size_t* nstages) {
    std::vector<wg_lt_stage*> made;
    const int rc = guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(path, "wg_bundle");
        check_ptr(nstages, "wg_bundle");
        FILE* f = std::fopen(path, "rb");
        if (!f) wg::fail(wg::kInvalid, std::string("wg_bundle: cannot open ") + path);
        std::vector<uint8_t> bytes;
        uint8_t buf[1 << 16];
        size_t got;
        while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + got);
        std::fclose(f);
        const wg::Bundle b = wg::bundle_decode(bytes.data(), bytes.size());
        if (b.N != c.N || b.dnum != c.dnum || b.q.size() != c.nq || b.p.size() != c.np ||
            !std::equal(b.q.begin(), b.q.end(), c.q.begin()) || !std::equal(b.p.begin(), b.p.end(), c.p.begin()))
            wg::fail(wg::kInvalid, "wg_bundle: the bundle's parameters differ from the context's");
        if (b.stages.size() > max_stages || (!b.stages.empty() && !stages))
            wg::fail(wg::kInvalid, "wg_bundle: more stages in the bundle than room for their handles");
        for (const auto& k : b.keys) {
            const size_t words = k.kind == WG_KEY_DENSE_TO_SPARSE ? 4 * c.N
                                                                  : k.parts * 2 * (k.key_level + 1 + c.np) * c.N;
            if (k.data.size() != words) wg::fail(wg::kInvalid, "wg_bundle: key size does not match its shape");
            const int r = wg_ctx_set_key(ctx, (int)k.kind, k.rotation, k.data.data(), k.parts, k.key_level);
            if (r != WG_OK) wg::fail(r, g_err);
        }
        for (const auto& st : b.stages) {
            const size_t per = (st.level + 1 + c.np) * c.N;
            if (st.indices.empty() || st.diagonals.size() != st.indices.size() * per)
                wg::fail(wg::kInvalid, "wg_bundle: stage size does not match its shape");
            wg_lt_stage* h = nullptr;
            const int r = wg_lt_stage_create(ctx, st.level, st.indices.size(), st.indices.data(), st.diagonals.data(),
                                             st.baby, st.slots, (int)st.rescale, &h);
            if (r != WG_OK) wg::fail(r, g_err);
            made.push_back(h);
        }
        for (size_t i = 0; i < made.size(); ++i) stages[i] = made[i];
        *nstages = made.size();
    });
    if (rc != WG_OK)
        for (auto* h : made) wg_lt_stage_destroy(h);
    return rc;
}

int wg_aes_walsh_encrypt_round_key_bits(wg_context* ctx, const wg_bootstrap_params* params,
                                        const uint8_t* expanded_key, size_t active_blocks, const int8_t* secret,
                                        uint64_t seed, double sigma, uint64_t* const* out_b, uint64_t* const* out_a,
                                        double* out_scale, size_t* out_level, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(params, "ckks_aes_walsh");
        check_ptr(out_scale, "ckks_aes_walsh");
        check_ptr(out_level, "ckks_aes_walsh");
        check_cts(c, 1408, out_b, out_a, "ckks_aes_walsh");
        wg::BootstrapParams bp;
        bp.s2c_depth = params->s2c_depth;
        bp.scale = params->scale;
        if (!(bp.scale > 0.0)) wg::fail(wg::kInvalid, "ckks_aes_walsh: invalid scale");
        wg::walsh_encrypt_round_key_bits(c, bp, expanded_key, active_blocks, secret, seed, sigma, out_b, out_a,
                                         out_scale, out_level, S(stream));
    });
}

int wg_decrypt_decode(wg_context* ctx, size_t count, size_t level, const double* scales, const uint64_t* const* b,
                      const uint64_t* const* a, const uint64_t* const* c2, const int8_t* secret, double* re, double* im,
                      void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (count && (!b || !a)) wg::fail(wg::kInvalid, "ckks_decrypt: null ciphertext array");
        for (size_t k = 0; k < count; ++k) {
            check_ptr(b[k], "ckks_decrypt");
            check_ptr(a[k], "ckks_decrypt");
        }
        wg::decrypt_decode_device(c, count, level, scales, b, a, c2, secret, re, im, S(stream));
    });
}

int wg_xboot_sbox_coefficients(int64_t* out) {
    return guard([&] {
        check_ptr(out, "ckks_aes");
        const auto cf = wg::xboot_sbox_coefficients();
        for (size_t b = 0; b < 8; ++b)
            for (size_t m = 0; m < 256; ++m) out[b * 256 + m] = cf[b][m];
    });
}

struct wg_server {
    wg::Server* s;
};

struct wg_serve_budget {
    wg::ServeBudget b;
};

int wg_serve_budget_create(size_t bytes, wg_serve_budget** out) {
    return guard([&] {
        if (!out) wg::fail(wg::kInvalid, "wg_serve: null output");
        if (bytes == 0) wg::fail(wg::kInvalid, "wg_serve: budget must be positive");
        *out = new wg_serve_budget;
        (*out)->b.capacity = bytes;
    });
}

void wg_serve_budget_destroy(wg_serve_budget* budget) { delete budget; }

int wg_serve_create(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c, size_t ns2c,
                    const wg_lt_stage* const* s2c_x2, size_t ns2c_x2, const wg_lt_stage* const* c2s, size_t nc2s,
                    const double* coeffs, size_t ncoeffs, size_t packing_block_count, size_t packed_segment_count,
                    const uint64_t* const* key_b, const uint64_t* const* key_a, const double* key_scales,
                    size_t key_level, const wg_serve_config* config, wg_server** out) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out, "wg_serve");
        check_ptr(config, "wg_serve");
        check_ptr(key_scales, "wg_serve");
        if (!key_b || !key_a) wg::fail(wg::kInvalid, "wg_serve: null key bits");
        wg::ServeSetup su;
        su.bp = boot_args(params, s2c, ns2c, c2s, nc2s, coeffs, su.s2c, su.c2s);
        if (ns2c_x2 && !s2c_x2) wg::fail(wg::kInvalid, "wg_serve: null stage list");
        for (size_t k = 0; k < ns2c_x2; ++k) {
            check_ptr(s2c_x2[k], "wg_serve");
            su.s2c_x2.push_back(s2c_x2[k]->s);
        }
        su.coeffs.assign(coeffs, coeffs + ncoeffs);
        for (size_t k = 0; k < 1408; ++k) {
            check_ptr(key_b[k], "wg_serve");
            check_ptr(key_a[k], "wg_serve");
            su.key_b.push_back(key_b[k]);
            su.key_a.push_back(key_a[k]);
            su.key_scales.push_back(key_scales[k]);
        }
        su.key_level = key_level;
        su.packing_block_count = packing_block_count;
        su.packed_segment_count = packed_segment_count;
        wg::ServeConfig cfg;
        cfg.workers = config->workers;
        cfg.hbm_budget = config->hbm_budget_bytes;
        cfg.eval_bytes = config->eval_bytes;
        cfg.max_blocks = config->max_blocks;
        cfg.batch_window_ms = config->batch_window_ms;
        cfg.priority = config->priority;
        cfg.budget = config->budget ? &config->budget->b : nullptr;
        auto* h = new wg_server{nullptr};
        try {
            h->s = new wg::Server(c, std::move(su), cfg);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int wg_serve_create_xboot(wg_context* ctx, const wg_bootstrap_params* params, const wg_lt_stage* const* s2c,
                          size_t ns2c, const wg_lt_stage* const* c2s, size_t nc2s, const double* coeffs,
                          size_t ncoeffs, const uint64_t* const* key_b, const uint64_t* const* key_a,
                          const double* key_scales, const size_t* key_levels, const wg_serve_config* config,
                          wg_server** out) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out, "wg_serve");
        check_ptr(config, "wg_serve");
        check_ptr(key_scales, "wg_serve");
        if (!key_b || !key_a) wg::fail(wg::kInvalid, "wg_serve: null key bits");
        wg::ServeSetup su;
        su.bp = boot_args(params, s2c, ns2c, c2s, nc2s, coeffs, su.s2c, su.c2s);
        check_ptr(key_levels, "wg_serve");
        su.xboot = true;
        su.coeffs.assign(coeffs, coeffs + ncoeffs);
        for (size_t k = 0; k < 1408; ++k) {
            check_ptr(key_b[k], "wg_serve");
            check_ptr(key_a[k], "wg_serve");
            su.key_b.push_back(key_b[k]);
            su.key_a.push_back(key_a[k]);
            su.key_scales.push_back(key_scales[k]);
            su.key_levels.push_back(key_levels[k]);
        }
        wg::ServeConfig cfg;
        cfg.workers = config->workers;
        cfg.hbm_budget = config->hbm_budget_bytes;
        cfg.eval_bytes = config->eval_bytes;
        cfg.max_blocks = config->max_blocks;
        cfg.batch_window_ms = config->batch_window_ms;
        cfg.priority = config->priority;
        cfg.budget = config->budget ? &config->budget->b : nullptr;
        auto* h = new wg_server{nullptr};
        try {
            h->s = new wg::Server(c, std::move(su), cfg);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int wg_serve_submit(wg_server* server, const uint8_t* counters, const uint8_t* ciphertexts, size_t blocks,
                    uint64_t* const* out_b, uint64_t* const* out_a, uint64_t* id) {
    return guard([&] {
        if (!server || !server->s) wg::fail(wg::kInvalid, "wg_serve: null server");
        check_ptr(id, "wg_serve");
        *id = server->s->submit(counters, ciphertexts, blocks, out_b, out_a);
    });
}

int wg_serve_wait(wg_server* server, uint64_t id, double timeout_s, wg_serve_result* result) {
    bool ready = false;
    std::string err;
    const int rc = guard([&] {
        if (!server || !server->s) wg::fail(wg::kInvalid, "wg_serve: null server");
        check_ptr(result, "wg_serve");
        wg::ServeResult r;
        ready = server->s->wait(id, timeout_s, &r);
        if (!ready) return;
        result->status = r.status;
        result->block_offset = r.block_offset;
        result->active_blocks = r.active_blocks;
        result->batch_requests = r.batch_requests;
        result->batch_blocks = r.batch_blocks;
        result->queue_ms = r.queue_ms;
        result->latency_ms = r.latency_ms;
        for (size_t k = 0; k < 128; ++k) {
            result->out_level[k] = r.out_level[k];
            result->out_scale[k] = r.out_scale[k];
        }
        err = r.error;
    });
    if (rc != WG_OK) return rc;
    if (!ready) return WG_NOT_READY;
    if (!err.empty()) wg::set_last_error(err);
    return WG_OK;
}

void wg_serve_destroy(wg_server* server) {
    if (!server) return;
    delete server->s;
    delete server;
}

struct wg_batch_plan {
    wg::Context* c;
    wg::BatchGraph* g;
};

int wg_batch_plan_create(wg_context* ctx, size_t count, const size_t* levels, uint64_t* const* xb,
                         uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                         const int64_t* rots, wg_batch_plan** out) {
    return guard([&] {
        wg::Context& c = C(ctx);
        check_ptr(out, "wg_batch_plan_create");
        *out = nullptr;
        check_batch(c, count, levels, xb, xa, yb, ya, rots);
        std::vector<uint64_t> galois(count);
        std::vector<const wg::KeyEntry*> keys(count, nullptr);
        for (size_t i = 0; i < count; ++i) {
            const int64_t r = normalize_rotation(c, rots[i]);
            galois[i] = r ? rotation_galois(c, r) : 0;
            if (r) keys[i] = &c.key(WG_KEY_ROTATION, r);
        }
        wg::BatchGraph* g = wg::batch_graph_create(c, count, levels, xb, xa, yb, ya, galois.data(),
                                                   &c.key(WG_KEY_RELIN, 0), keys.data());
        *out = new wg_batch_plan{&c, g};
    });
}

int wg_batch_plan_launch(wg_batch_plan* plan, void* stream) {
    return guard([&] {
        check_ptr(plan, "wg_batch_plan_launch");
        wg::check_cuda(cudaSetDevice(plan->c->device), "cudaSetDevice");
        wg::batch_graph_launch(*plan->g, S(stream));
    });
}

void wg_batch_plan_destroy(wg_batch_plan* plan) {
    if (!plan) return;
    cudaSetDevice(plan->c->device);
    delete plan->g;
    delete plan;
}

int wg_sequence_mul_relin_rescale_rotate(wg_context* ctx, size_t count, const size_t* levels, uint64_t* const* xb,
                                         uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                                         const int64_t* rots, void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        cudaStream_t s = S(stream);
        check_batch(c, count, levels, xb, xa, yb, ya, rots);
        uint64_t* c2 = scratch_after_switch(c, s) + 2 * c.nq * c.N;
        for (size_t i = 0; i < count; ++i) {
            const size_t lv = levels[i];
            wg::tensor(c, lv, xb[i], xa[i], yb[i], ya[i], c2, s);
            do_relin(c, lv, xb[i], xa[i], c2, s);
            do_rescale(c, lv, xb[i], 1, 0, s);
            do_rescale(c, lv, xa[i], 1, 0, s);
            do_rotate(c, lv - 1, xb[i], xa[i], rots[i], s);
        }
    });
}

int wg_lt_stage_create(wg_context* ctx, size_t level, size_t nterms, const uint64_t* indices,
                       const uint64_t* diagonals, size_t baby_step_count, size_t slot_count, int rescale_after,
                       wg_lt_stage** out) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (!out || !indices || !diagonals) wg::fail(wg::kInvalid, "ckks_linear_transform: null argument");
        *out = nullptr;
        wg::LtStage* st = wg::lt_stage_create(c, level, nterms, indices, diagonals, baby_step_count, slot_count,
                                              rescale_after != 0);
        *out = new wg_lt_stage{st};
    });
}

int wg_lt_stage_info(const wg_lt_stage* st, size_t* level, size_t* nterms, size_t* baby, size_t* slots,
                     int* rescale_after, double* plaintext_scale) {
    return guard([&] {
        if (!st || !st->s) wg::fail(wg::kInvalid, "ckks_linear_transform: null stage");
        size_t l, n, b, sl;
        bool r;
        double ps;
        wg::lt_stage_info(*st->s, l, n, b, sl, r, ps);
        if (level) *level = l;
        if (nterms) *nterms = n;
        if (baby) *baby = b;
        if (slots) *slots = sl;
        if (rescale_after) *rescale_after = r ? 1 : 0;
        if (plaintext_scale) *plaintext_scale = ps;
    });
}

int wg_lt_stage_download(wg_context* ctx, const wg_lt_stage* st, uint64_t* indices, uint64_t* diagonals) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (!st || !st->s) wg::fail(wg::kInvalid, "ckks_linear_transform: null stage");
        wg::BundleStage b;
        wg::lt_stage_export(c, *st->s, b);
        if (indices) std::copy(b.indices.begin(), b.indices.end(), indices);
        if (diagonals) std::copy(b.diagonals.begin(), b.diagonals.end(), diagonals);
    });
}

static wg::dft::Literal dft_literal(const wg_dft_literal* lit) {
    if (!lit) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: null literal");
    wg::dft::Literal L;
    L.coeffs_to_slots = lit->coeffs_to_slots != 0;
    L.level = lit->level;
    L.baby_step_count = lit->baby_step_count;
    L.log_bsgs_ratio = lit->log_bsgs_ratio;
    L.stage_count = lit->stage_count;
    size_t k = 0;
    for (size_t g = 0; g < lit->ngroups; ++g) {
        if (!lit->group_sizes || !lit->group_bits) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: null scale schedule");
        L.scale_groups.emplace_back(lit->group_bits + k, lit->group_bits + k + lit->group_sizes[g]);
        k += lit->group_sizes[g];
    }
    if (lit->nmerge) {
        if (!lit->merge_depths) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: null merge depths");
        L.merge_depths.assign(lit->merge_depths, lit->merge_depths + lit->nmerge);
    }
    L.active_slots = lit->active_slots;
    L.transform_scale = lit->transform_scale;
    L.input_selector_start = lit->input_selector_start;
    L.input_selector_size = lit->input_selector_size;
    return L;
}

int wg_dft_plan_describe(uint64_t N, const uint64_t* q, size_t nq, const wg_dft_literal* lit, size_t stage,
                         size_t* nstages, size_t* level, size_t* nterms, size_t* baby, int* rescale_after,
                         double* plaintext_scale, uint64_t* indices, double* diagonals) {
    return guard([&] {
        if (!q || nq == 0) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: empty modulus chain");
        if (N < 1024 || N > 65536 || (N & (N - 1))) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: invalid ring degree");
        const auto stages = wg::dft::generate_plan(dft_literal(lit), N, std::vector<uint64_t>(q, q + nq));
        if (nstages) *nstages = stages.size();
        if (stage >= stages.size()) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: stage index out of range");
        const auto& st = stages[stage];
        if (level) *level = st.level;
        if (nterms) *nterms = st.indices.size();
        if (baby) *baby = st.baby;
        if (rescale_after) *rescale_after = st.rescale_after ? 1 : 0;
        if (plaintext_scale) *plaintext_scale = st.plaintext_scale;
        if (indices) std::copy(st.indices.begin(), st.indices.end(), indices);
        if (diagonals)
            for (size_t t = 0; t < st.diagonals.size(); ++t)
                for (size_t i = 0; i < st.diagonals[t].size(); ++i) {
                    diagonals[2 * (t * st.slots + i)] = st.diagonals[t][i].real();
                    diagonals[2 * (t * st.slots + i) + 1] = st.diagonals[t][i].imag();
                }
    });
}

int wg_dft_plan_create(wg_context* ctx, const wg_dft_literal* lit, wg_lt_stage** stages, size_t max_stages,
                       size_t* nstages, void* stream) {
    std::vector<wg::LtStage*> made;
    const int rc = guard([&] {
        wg::Context& c = C(ctx);
        if (!lit || !stages || !nstages) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: null argument");
        const wg::dft::Literal L = dft_literal(lit);
        wg::check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
        made = wg::dft_plan_create(c, L, S(stream));
        *nstages = made.size();
        if (made.size() > max_stages) wg::fail(wg::kInvalid, "ckks_bootstrap_dft: more stages than max_stages");
        for (size_t i = 0; i < made.size(); ++i) stages[i] = new wg_lt_stage{made[i]};
        made.clear();
    });
    for (auto* m : made) wg::lt_stage_destroy(m);
    return rc;
}

void wg_lt_stage_destroy(wg_lt_stage* st) {
    if (!st) return;
    wg::lt_stage_destroy(st->s);
    delete st;
}

int wg_lt_stage_apply(wg_context* ctx, const wg_lt_stage* st, size_t count, uint64_t* const* b, uint64_t* const* a,
                      void* stream) {
    return guard([&] {
        wg::Context& c = C(ctx);
        if (!st || !st->s) wg::fail(wg::kInvalid, "ckks_linear_transform: null stage");
        if (count && (!b || !a)) wg::fail(wg::kInvalid, "ckks_linear_transform: null ciphertext array");
        for (size_t i = 0; i < count; ++i) {
            check_ptr(b[i], "ckks_linear_transform");
            check_ptr(a[i], "ckks_linear_transform");
        }
        wg::lt_stage_apply(c, *st->s, count, b, a, S(stream));
    });
}

int wg_malloc(void** ptr, size_t bytes) {
    return guard([&] {
        if (cudaMalloc(ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            wg::fail(wg::kNoMemory, "cudaMalloc failed");
        }
    });
}
int wg_free(void* ptr) {
    return guard([&] { wg::check_cuda(cudaFree(ptr), "cudaFree"); });
}
int wg_memcpy_htod(void* dst, const void* src, size_t bytes, void* stream) {
    return guard([&] { wg::check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S(stream)), "memcpy"); });
}
int wg_memcpy_dtoh(void* dst, const void* src, size_t bytes, void* stream) {
    return guard([&] { wg::check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S(stream)), "memcpy"); });
}
int wg_stream_synchronize(void* stream) {
    return guard([&] { wg::check_cuda(cudaStreamSynchronize(S(stream)), "cudaStreamSynchronize"); });
}

}  // extern "C"
