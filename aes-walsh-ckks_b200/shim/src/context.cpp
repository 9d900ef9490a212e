// CKKSContext of the reference API, built on the device (see ckks_context.hpp).
//
// What the reference's constructor derives (src/ckks/context/ckks_context.cpp:157-400, 603-705)
// is derived here by the same rules: the SlotToCoeff literal at level s2c_depth with transform
// scale (q0 / 2) / scale (and / (2 scale) for inputs at twice the scale), the CoeffToSlot literal
// at the top level with the binary transform scale 2^(evalmod bits - q0 bits) scale / q0 / K
// divided by the sparse trace factor, the EvalMod fit of the parameter set, and the rotation
// set: the configured rotations, every plan's baby and giant steps, the sparse trace rotations
// and the AES-Walsh segment rotations, normalised modulo N/2 and deduplicated in that order.
#include "context_engine.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <random>
#include <stdexcept>
#include <string>

#include "../../../include/walsh_gpu.h"
#include "ckks_context.hpp"

namespace {

void ok(int rc, const char* what) {
    if (rc == WG_OK) return;
    const std::string msg = std::string(what) + ": " + wg_last_error();
    if (rc == WG_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

int64_t normalize_rotation(size_t N, int64_t r) {
    const int64_t slots = (int64_t)(N / 2);
    r %= slots;
    if (r < 0) r += slots;
    return r;
}

// Ternary secret with exactly h nonzero coefficients (+-1 with equal probability) at uniformly
// drawn positions, or uniform ternary coefficients when h == 0.
std::vector<int8_t> sample_secret(size_t N, size_t h, std::random_device& rd) {
    std::vector<int8_t> s(N, 0);
    auto draw = [&](uint64_t bound) {  // uniform in [0, bound)
        const uint64_t lim = UINT64_MAX - UINT64_MAX % bound;
        for (;;) {
            const uint64_t x = ((uint64_t)rd() << 32) | rd();
            if (x < lim) return x % bound;
        }
    };
    if (h == 0) {
        for (size_t i = 0; i < N; ++i) s[i] = (int8_t)((int)draw(3) - 1);
        return s;
    }
    if (h > N) throw std::invalid_argument("ckks_context: Hamming weight exceeds the ring degree");
    std::vector<uint32_t> pos(N);
    for (size_t i = 0; i < N; ++i) pos[i] = (uint32_t)i;
    for (size_t i = 0; i < h; ++i) {
        const size_t j = i + (size_t)draw(N - i);
        std::swap(pos[i], pos[j]);
        s[pos[i]] = draw(2) ? 1 : -1;
    }
    return s;
}

}  // namespace

CKKSContext::Engine::~Engine() {
    for (auto* v : {&s2c, &s2c_x2, &c2s})
        for (wg_lt_stage* st : *v) wg_lt_stage_destroy(st);
    if (ctx) wg_ctx_destroy(ctx);
}

uint64_t CKKSContext::Engine::next_seed() { return ((uint64_t)rd() << 32) | rd(); }

std::vector<wg_lt_stage*> CKKSContext::Engine::make_plan(bool c2s_plan, double transform_scale) {
    const CKKSParams& p = params;
    const auto& sched = c2s_plan ? p.getBootstrapC2SLogPlaintextScales() : p.getBootstrapS2CLogPlaintextScales();
    const auto& merge = c2s_plan ? p.getBootstrapC2SMergeDepths() : p.getBootstrapS2CMergeDepths();
    std::vector<size_t> sizes, bits;
    for (const auto& g : sched) {
        sizes.push_back(g.size());
        bits.insert(bits.end(), g.begin(), g.end());
    }
    wg_dft_literal lit{};
    lit.coeffs_to_slots = c2s_plan ? 1 : 0;
    lit.level = c2s_plan ? p.getDepth() : p.getBootstrapS2CDepth();
    lit.baby_step_count = p.getBootstrapLinearTransformBsgsBabyStepCounts()[c2s_plan ? 1 : 0];
    lit.log_bsgs_ratio = c2s_plan ? p.getBootstrapC2SLogBsgsRatio() : p.getBootstrapS2CLogBsgsRatio();
    lit.stage_count = c2s_plan ? p.getBootstrapC2SDepth() : p.getBootstrapS2CDepth();
    lit.group_sizes = sizes.data();
    lit.group_bits = bits.data();
    lit.ngroups = sizes.size();
    lit.merge_depths = merge.data();
    lit.nmerge = merge.size();
    lit.active_slots = p.getBootstrapActiveSlotCount();
    lit.transform_scale = transform_scale;
    std::vector<wg_lt_stage*> st(64, nullptr);
    size_t n = 0;
    ok(wg_dft_plan_create(ctx, &lit, st.data(), st.size(), &n, nullptr), "ckks_bootstrap_dft");
    st.resize(n);
    return st;
}

CKKSContext::CKKSContext(CKKSParams ckks_params) : eng(new Engine(std::move(ckks_params))) {
    Engine& e = *eng;
    const CKKSParams& p = e.params;
    const size_t N = p.getN();
    if (p.bts_keys || p.s2c_ptxt || p.c2s_ptxt) (void)p.getBootstrapParams();
    // hybrid key switching needs P at least as wide as the widest Q digit
    {
        size_t pbits = 0;
        for (uint64_t m : p.getPModuli()) pbits += 64 - (size_t)__builtin_clzll(m);
        const auto& q = p.getModuli();
        const size_t alpha = (q.size() + p.getDnum() - 1) / p.getDnum();
        for (size_t s = 0; s < q.size(); s += alpha) {
            size_t dbits = 0;
            for (size_t i = s; i < std::min(q.size(), s + alpha); ++i) dbits += 64 - (size_t)__builtin_clzll(q[i]);
            if (pbits < dbits)
                throw std::invalid_argument(
                    "ckks_context: hybrid key-switch P basis is smaller than the widest Q digit");
        }
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) throw std::runtime_error("ckks_context: no CUDA device");
    const std::vector<uint64_t> q(p.getModuli().begin(), p.getModuli().end());
    const std::vector<uint64_t> pm(p.getPModuli().begin(), p.getPModuli().end());
    ok(wg_ctx_create(N, q.data(), q.size(), pm.data(), pm.size(), p.getDnum(), device, &e.ctx), "ckks_context");

    const bool s2c_plan = (p.bts_keys || p.s2c_ptxt) && p.getBootstrapS2CDepth() > 0;
    const bool c2s_plan = (p.bts_keys || p.c2s_ptxt) && p.getBootstrapC2SDepth() > 0;
    const double q0 = (double)q[0], scale = p.getScale();
    if (s2c_plan) {
        e.s2c = e.make_plan(false, (q0 * 0.5) / scale);
        if (p.usesAesWalsh()) e.s2c_x2 = e.make_plan(false, (q0 * 0.5) / (scale * 2.0));
    }
    if (c2s_plan) {
        const CKKSBootstrapParams& b = p.getBootstrapParams();
        const size_t evalmod_bits = b.evalmod_bit_size == 0 ? p.getDefaultQBit() : b.evalmod_bit_size;
        e.c2s_transform_scale =
            std::ldexp(scale, (int)evalmod_bits - (int)p.getQ0Bit()) / q0 / (double)p.getBootstrapEvalModK();
        const size_t trace = p.getSlots() / p.getBootstrapActiveSlotCount();
        e.c2s = e.make_plan(true, e.c2s_transform_scale / (double)trace);
    }
    if (p.bts_keys && p.getBootstrapEvalModDepth() > 0) {
        e.evalmod = binboot_han_ki_discrete_multi_interval_approximate(
            (double)p.getBootstrapEvalModK(), p.getBootstrapEvalModPolynomialDegree(), p.getBootstrapEvalModDoubleAngle(),
            p.getBootstrapEvalModDiscreteIntervalRadius(), p.getBootstrapEvalModDiscreteValidationPointsPerInterval(),
            p.getBootstrapEvalModCoefficientPruneThreshold());
        e.has_evalmod = true;
    }
    e.has_plans = s2c_plan || c2s_plan;

    // secrets
    e.secret = sample_secret(N, p.getSecretKeyHammingWeight(), e.rd);
    if (p.bts_keys) e.low_secret = sample_secret(N, p.getBootstrapSparseSecretHammingWeight(), e.rd);

    // rotation set
    auto add = [&](int64_t r) {
        const int64_t n = normalize_rotation(N, r);
        if (n == 0 || std::find(e.rotations.begin(), e.rotations.end(), n) != e.rotations.end()) return;
        e.rotations.push_back(n);
    };
    for (int64_t r : p.getRotateValues()) add(r);
    auto add_plan = [&](const std::vector<wg_lt_stage*>& plan) {
        for (wg_lt_stage* st : plan) {
            size_t level = 0, nterms = 0, baby = 0, slots = 0;
            int resc = 0;
            double ps = 0;
            ok(wg_lt_stage_info(st, &level, &nterms, &baby, &slots, &resc, &ps), "ckks_context");
            std::vector<uint64_t> idx(nterms);
            ok(wg_lt_stage_download(e.ctx, st, idx.data(), nullptr), "ckks_context");
            for (uint64_t d : idx) {
                const size_t br = d % baby, gr = d - br;
                if (br) add((int64_t)br);
                if (gr) add((int64_t)gr);
            }
        }
    };
    if (p.bts_keys || p.s2c_ptxt || p.c2s_ptxt) {
        if (s2c_plan) add_plan(e.s2c);
        if (c2s_plan) {
            add_plan(e.c2s);
            for (size_t r = p.getBootstrapActiveSlotCount(); r < p.getSlots(); r <<= 1) add((int64_t)r);
        }
    }
    if (p.usesAesWalsh()) {
        const size_t bc = p.getAesWalshBlockCount(), segs = p.getAesWalshPackedSegmentCount();
        if (bc == 0) throw std::invalid_argument("ckks_context: AES Walsh block count must be positive");
        if (segs < 30) throw std::invalid_argument("ckks_context: AES Walsh packed segment count must be at least 30");
        if (segs > p.getSlots() / bc) throw std::invalid_argument("ckks_context: AES Walsh block count exceeds packed slot capacity");
        for (size_t k = 1; k < segs; ++k) {
            add((int64_t)(k * bc));
            add(-(int64_t)(k * bc));
        }
    }

    // switching keys on the device, each from its own seed
    const double sigma = p.getSigma();
    for (int64_t r : e.rotations)
        ok(wg_keygen_switch_key(e.ctx, WG_KEY_ROTATION, r, e.secret.data(), nullptr, nullptr, e.next_seed(), sigma, nullptr,
                                nullptr),
           "ckks_context: rotation key");
    ok(wg_keygen_switch_key(e.ctx, WG_KEY_CONJ, 0, e.secret.data(), nullptr, nullptr, e.next_seed(), sigma, nullptr,
                            nullptr),
       "ckks_context: conjugation key");
    ok(wg_keygen_switch_key(e.ctx, WG_KEY_RELIN, 0, e.secret.data(), nullptr, nullptr, e.next_seed(), sigma, nullptr,
                            nullptr),
       "ckks_context: relinearisation key");
    if (p.bts_keys) {
        ok(wg_keygen_secret_switch(e.ctx, WG_KEY_DENSE_TO_SPARSE, e.secret.data(), e.low_secret.data(), nullptr, nullptr,
                                   e.next_seed(), sigma, nullptr, nullptr),
           "ckks_context: dense-to-sparse key");
        ok(wg_keygen_secret_switch(e.ctx, WG_KEY_SPARSE_TO_DENSE, e.low_secret.data(), e.secret.data(), nullptr,
                                   nullptr, e.next_seed(), sigma, nullptr, nullptr),
           "ckks_context: sparse-to-dense key");
        e.has_switch_keys = true;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("ckks_context: device error while building");
}

CKKSContext::~CKKSContext() = default;
CKKSContext::CKKSContext(CKKSContext&&) noexcept = default;
CKKSContext& CKKSContext::operator=(CKKSContext&&) noexcept = default;

const CKKSParams& CKKSContext::getParams() const { return eng->params; }
bool CKKSContext::hasSparseSecretEncapsulationKeys() const { return eng->has_switch_keys; }
bool CKKSContext::hasConjugationKey() const { return true; }
size_t CKKSContext::getRotationKeyCount() const { return eng->rotations.size(); }
bool CKKSContext::hasRotationKey(int64_t rotation) const {
    const int64_t n = normalize_rotation(eng->params.getN(), rotation);
    return n == 0 || std::find(eng->rotations.begin(), eng->rotations.end(), n) != eng->rotations.end();
}
bool CKKSContext::hasEvalModBootstrapDftPlans() const { return eng->has_plans; }
double CKKSContext::getEvalModScaledC2STransformScale() const { return eng->c2s_transform_scale; }
const PolynomialApproximation& CKKSContext::getEvalModPolynomial() const {
    if (!eng->has_evalmod) throw std::runtime_error("ckks_context: EvalMod polynomial is unavailable");
    return eng->evalmod;
}
CKKSContext::Engine& CKKSContext::engine() const { return *eng; }

wg_bootstrap_params CKKSContext::Engine::bootstrap_params() const {
    wg_bootstrap_params b{};
    b.s2c_depth = params.getBootstrapS2CDepth();
    b.depth = params.getDepth();
    const CKKSBootstrapParams& bp = params.getBootstrapParams();
    b.evalmod_log_scale = bp.evalmod_bit_size == 0 ? params.getDefaultQBit() : bp.evalmod_bit_size;
    b.double_angle = params.getBootstrapEvalModDoubleAngle();
    b.active_slots = params.getBootstrapActiveSlotCount();
    b.slots = params.getSlots();
    b.scale = params.getScale();
    return b;
}
