// The XBOOT AES S-box on lazy bits, batched over S-box instances.
//
// Reference: ckks_aes_xboot_sbox_impl and its helpers, src/ckks/operations/circuits/aes/
// ckks_aes_ctr.cpp:160-336.  Each output bit of the S-box is written as an integer combination
// of the 255 monomials prod_{i in mask} x_i of the input bits (coefficients from the Moebius
// transform of the bit's truth table, :258-278).  The monomials come from a layered product tree
// (:185-256): the bit pairs (0,1), (2,3), (4,5), (6,7); within each nibble, every monomial of
// its first pair times every monomial of its second; across the nibbles, every nibble monomial
// of the low half times every one of the high half.  Every product is multiply + relinearize +
// rescale with both operands dropped to their common level and relabelled to the input scale,
// and the result relabelled to it again (:160-183).  All monomials therefore share one scale,
// and the exact additions of the combination (:151-158) only drop levels; an output bit is the
// constant term plus sum c_m x_m at the lowest level involved.
//
// Device plan: the products of one layer are independent, so each layer runs as a few batched
// multiply + relinearize + rescale calls (grouped by output level, chunked to bound the memory
// of a call) over all products and instances at once; each output bit is then one linear
// combination over the monomials (DeviceOps::lincomb).  Multiplication by an integer and the
// additions are exact modular operations on canonical residues, so forming the sum at once gives
// the reference's residues.
//
// The XBOOT AES-128-CTR circuit (ckks_aes_ctr and its helpers, ckks_aes_ctr.cpp:337-779) is
// built from it: the initial public XOR of the counter bits, ten rounds of SubBytes (all 16
// byte positions as one batch of S-box instances), ShiftRows (a relabelling), MixColumns and
// AddRoundKey (one fused launch of integer combinations), the pair bootstraps that refresh the
// state after rounds 1..9 (all 64 pairs batched), then the public ciphertext XOR and a last
// refresh.
#include <algorithm>
#include <cmath>
#include <exception>
#include <memory>
#include <stdexcept>
#include <thread>

#include "wg_aes_linear.cuh"
#include "wg_ctops.cuh"

namespace wg {

std::array<std::array<int64_t, 256>, 8> xboot_sbox_coefficients() {
    const auto sb = aes_sbox_table();
    std::array<std::array<int64_t, 256>, 8> c{};
    for (size_t bit = 0; bit < 8; ++bit) {
        // truth table of the bit, then the subset differences variable by variable
        for (size_t x = 0; x < 256; ++x) c[bit][x] = (sb[x] >> bit) & 1;
        for (size_t v = 0; v < 8; ++v)
            for (size_t m = 0; m < 256; ++m)
                if (m >> v & 1) c[bit][m] -= c[bit][m ^ (size_t{1} << v)];
    }
    return c;
}

namespace {

constexpr size_t kBits = 8;
constexpr size_t kMaxProductCts = 512;  // ciphertexts per batched product call

// rounded_scaled_integer_mod_q: round(k * scale) mod q (ckks_add_integer_constant_inplace)
uint64_t scaled_integer_mod(int64_t k, long double scale, uint64_t q) {
    if (k == 0) return 0;
    const long double v = static_cast<long double>(k) * scale;
    if (!std::isfinite(v)) throw std::invalid_argument("ckks_add_integer_constant_inplace: non-finite scaled constant");
    long double r = std::fmod(std::round(v), static_cast<long double>(q));
    if (r < 0.0L) r += static_cast<long double>(q);
    uint64_t u = static_cast<uint64_t>(r);
    return u >= q ? u % q : u;
}

class XbootSbox {
public:
    XbootSbox(Context& c, size_t count, long double scale, cudaStream_t s) : c_(c), count_(count), scale_(scale), s_(s) {}

    struct Mono {
        size_t mask;
        CtBatch x;  // count ciphertexts, two polynomials, at the input scale
    };

    // the monomials of input bits [begin, end) (end - begin a power of two), as the tree builds them
    std::vector<Mono> layered(const std::vector<CtBatch>& in, size_t begin, size_t end) {
        const size_t n = end - begin;
        std::vector<Mono> out;
        if (n == 1) {
            CtBatch x = in[begin];
            x.scale = scale_;
            out.push_back({size_t{1} << begin, x});
            return out;
        }
        if (n == 2) {
            CtBatch l = in[begin], r = in[begin + 1];
            l.scale = r.scale = scale_;
            const CtBatch prod = products({{&l, &r}})[0];
            out.push_back({size_t{1} << begin, l});
            out.push_back({size_t{1} << (begin + 1), r});
            out.push_back({(size_t{1} << begin) | (size_t{1} << (begin + 1)), prod});
            return out;
        }
        const size_t mid = begin + n / 2;
        std::vector<Mono> left = layered(in, begin, mid), right = layered(in, mid, end);
        std::vector<std::pair<const CtBatch*, const CtBatch*>> pairs;
        for (const Mono& a : left)
            for (const Mono& b : right) pairs.push_back({&a.x, &b.x});
        const std::vector<CtBatch> prod = products(pairs);
        size_t k = 0;
        for (const Mono& a : left)
            for (const Mono& b : right) out.push_back({a.mask | b.mask, prod[k++]});
        for (const Mono& a : left) out.push_back(a);
        for (const Mono& b : right) out.push_back(b);
        return out;
    }

    // xboot_mul_relin_rescale for every pair: operands dropped to their common level and labelled
    // with the input scale, tensor, relinearisation, rescale, result labelled with the input scale
    std::vector<CtBatch> products(const std::vector<std::pair<const CtBatch*, const CtBatch*>>& pairs) {
        std::vector<CtBatch> out(pairs.size());
        std::map<size_t, std::vector<size_t>> by_level;
        for (size_t k = 0; k < pairs.size(); ++k) {
            const size_t level = std::min(pairs[k].first->level, pairs[k].second->level);
            if (level == 0) throw std::invalid_argument("ckks_aes: insufficient level for XBOOT S-box multiplication");
            by_level[level].push_back(k);
        }
        const size_t per_call = std::max<size_t>(1, kMaxProductCts / count_);
        for (const auto& [level, ks] : by_level)
            for (size_t k0 = 0; k0 < ks.size(); k0 += per_call) {
                const size_t np = std::min(per_call, ks.size() - k0);
                auto ops = std::make_unique<DeviceOps>(c_, np * count_, s_);
                CtBatch l, r;
                l.p.resize(np * count_);
                r.p.resize(np * count_);
                for (size_t j = 0; j < np; ++j)
                    for (size_t i = 0; i < count_; ++i) {
                        l.p[j * count_ + i] = pairs[ks[k0 + j]].first->p[i];
                        r.p[j * count_ + i] = pairs[ks[k0 + j]].second->p[i];
                    }
                l.np = r.np = 2;
                l.level = r.level = level;
                l.cap = r.cap = level + 1;
                l.scale = r.scale = scale_;
                CtBatch x = ops->clone(l);
                ops->tensor(x, r);
                ops->relin(x);
                ops->rescale(x);
                for (size_t j = 0; j < np; ++j) {
                    CtBatch& o = out[ks[k0 + j]];
                    o.p.assign(x.p.begin() + j * count_, x.p.begin() + (j + 1) * count_);
                    o.np = 2;
                    o.level = x.level;
                    o.cap = x.cap;
                    o.scale = scale_;
                }
                keep_.push_back(std::move(ops));  // the products live until the combination
            }
        return out;
    }

private:
    Context& c_;
    size_t count_;
    long double scale_;
    cudaStream_t s_;
    std::vector<std::unique_ptr<DeviceOps>> keep_;
};

}  // namespace

void xboot_sbox(Context& c, size_t count, size_t level, double scale, uint64_t* const* in_b, uint64_t* const* in_a,
                uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s) {
    if (count == 0) return;
    if (level >= c.nq) throw std::invalid_argument("ckks_aes: invalid XBOOT S-box input level");
    DeviceOps ops(c, count, s);
    std::vector<CtBatch> in(kBits);
    for (size_t k = 0; k < kBits; ++k) in[k] = ops.wrap(in_b + k * count, in_a + k * count, level, scale);
    const long double target = in[0].scale;
    XbootSbox sb(c, count, target, s);
    std::vector<XbootSbox::Mono> mono = sb.layered(in, 0, kBits);
    std::vector<const CtBatch*> by_mask(256, nullptr);
    for (const auto& m : mono) by_mask[m.mask] = &m.x;
    for (size_t m = 1; m < 256; ++m)
        if (!by_mask[m]) throw std::runtime_error("ckks_aes: missing XBOOT S-box monomial");
    const auto cf = xboot_sbox_coefficients();
    for (size_t bit = 0; bit < kBits; ++bit) {
        // the accumulator ends at the lowest level of the constant (input level) and the terms
        size_t lv = cf[bit][0] != 0 ? level : c.nq;
        for (size_t m = 1; m < 256; ++m)
            if (cf[bit][m] != 0) lv = std::min(lv, by_mask[m]->level);
        if (lv == c.nq) lv = level;  // an all-zero bit is a zero ciphertext at the input level
        std::vector<uint64_t> cadd(lv + 1, 0);
        for (size_t l = 0; l <= lv; ++l) cadd[l] = scaled_integer_mod(cf[bit][0], target, c.q[l]);
        std::vector<DeviceOps::LinTerm> terms;
        for (size_t m = 1; m < 256; ++m) {
            if (cf[bit][m] == 0) continue;
            DeviceOps::LinTerm t;
            t.x = *by_mask[m];
            t.x.level = lv;
            t.c.resize(lv + 1);
            for (size_t l = 0; l <= lv; ++l) {
                const int64_t qi = (int64_t)c.q[l];
                t.c[l] = (uint64_t)(((cf[bit][m] % qi) + qi) % qi);
            }
            terms.push_back(std::move(t));
        }
        CtBatch o = ops.lincomb(lv, 2, target, cadd, terms);
        ops.copy_out(o, out_b + bit * count, out_a + bit * count);
        out_level[bit] = lv;
        out_scale[bit] = static_cast<double>(target);
    }
}

void bootstrap_pair(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                    size_t nc2s, const double* coeffs, size_t ncoeffs, size_t count, double scale, uint64_t* const* b0,
                    uint64_t* const* a0, uint64_t* const* b1, uint64_t* const* a1, size_t* out_level, double* out_scale,
                    cudaStream_t s) {
    if (count == 0) return;
    const size_t lv = p.s2c_depth, N = c.N;
    if (lv == 0 || p.depth >= c.nq) throw std::invalid_argument("ckks_batch_bootstrap_evalmod: S2C depth must be positive");
    DeviceOps ops(c, count, s);
    // packed = ct0 + ct1 * (the slot constant i encoded at scale 1), labelled with ct0's scale,
    // in buffers with room for the bootstrap's depth + 1 limbs
    CtBatch pk = ops.alloc(p.depth, 2);
    pk.level = lv;
    pk.scale = scale;
    for (size_t i = 0; i < count; ++i) {
        check_cuda(cudaMemcpyAsync(pk.p[i][0], b1[i], (lv + 1) * N * 8, cudaMemcpyDeviceToDevice, s), "pair pack");
        check_cuda(cudaMemcpyAsync(pk.p[i][1], a1[i], (lv + 1) * N * 8, cudaMemcpyDeviceToDevice, s), "pair pack");
    }
    ops.mul_complex_constant(pk, 0.0, 1.0, 1.0);
    ops.add(pk, ops.wrap(b0, a0, lv, scale), false);
    std::vector<uint64_t*> pb(count), pa(count);
    for (size_t i = 0; i < count; ++i) {
        pb[i] = pk.p[i][0];
        pa[i] = pk.p[i][1];
    }
    // the inputs are consumed by the packing (stream order), so the results may overwrite them
    bootstrap_evalmod(c, p, s2c, nplans, c2s, nc2s, coeffs, ncoeffs, count, scale, pb.data(), pa.data(), b0, a0, b1, a1,
                      out_level, out_scale, s);
}

namespace {

constexpr size_t kStateBits = 128;
constexpr size_t kAesRounds = 10;

// One launch of `kernel` over a job table.  wide: the kernel takes kWide words per thread
// (kb_scalar, kb_pmul, kb_add: grid_wide); otherwise one word per thread (grid_for).
template <bool wide = false, class Job, class Kernel>
void launch_jobs(Context& c, const std::vector<Job>& jobs, Kernel kernel, double bytes_per_job, const char* what,
                 cudaStream_t s) {
    if (jobs.empty()) return;
    JobTable t;
    const Job* j = t.add(jobs);
    t.upload(c, s);
    Probe probe(kClsElementwise, bytes_per_job * (double)jobs.size(), s);
    const dim3 grid = wide ? grid_wide(c, jobs.size()) : grid_for(c, jobs.size());
    kernel<<<grid, kT, 0, s>>>(t.at(j), (int)jobs.size(), c.d_mod);
    check_cuda(cudaGetLastError(), what);
}

// One state bit: a ciphertext in buffers with room for every level the circuit uses.
struct Bit {
    uint64_t* b = nullptr;
    uint64_t* a = nullptr;
    size_t level = 0;
    long double scale = 0.0L;
};

class XbootAes {
public:
    // own_state: the state buffers (room for depth + 1 limbs) come from the operation set;
    // otherwise the caller binds its own before use
    XbootAes(Context& c, const BootstrapParams& p, const S2cPlan* plans, size_t nplans, const LtStage* const* c2s,
             size_t nc2s, const double* coeffs, size_t ncoeffs, const XbootAesArgs& a, cudaStream_t s,
             bool own_state = true)
        : c_(c), p_(p), plans_(plans), nplans_(nplans), c2s_(c2s), nc2s_(nc2s), coeffs_(coeffs), ncoeffs_(ncoeffs),
          a_(a), s_(s), ops_(c, 1, s) {
        const size_t full = p.depth + 1;
        if (own_state)
            for (auto* set : {&st_, &tmp_})
                for (Bit& x : *set) {
                    x.b = ops_.raw(full);
                    x.a = ops_.raw(full);
                }
    }

    Bit& state(size_t bit) { return st_[bit]; }
    Bit& staged(size_t bit) { return tmp_[bit]; }

    // make_batched_initial_counter_state (ckks_aes_ctr.cpp:576-683): per state bit, the
    // round-0 key bit XOR the counter bit plane, one level down.  An all-zero plane only drops
    // the level, an all-one plane negates and adds 1, a varying plane b multiplies by the
    // encoded signs 1 - 2b at scale q_level, rescales, and adds the encoded plane b.
    void initial_state() {
        WG_SPAN("xboot.initial");
        const size_t N = c_.N, slots = N / 2, logical = p_.active_slots, L = a_.key_levels[0];
        if (L == 0) throw std::invalid_argument("ckks_aes: exact public XOR requires one level");
        for (size_t bit = 0; bit < kStateBits; ++bit)
            if (a_.key_levels[bit] != L) throw std::invalid_argument("ckks_aes: round-0 key bits must share one level");
        enum { kZero, kOne, kVarying };
        std::vector<int> kind(kStateBits);
        std::vector<size_t> varying;
        for (size_t bit = 0; bit < kStateBits; ++bit) {
            bool saw_zero = a_.blocks < logical, saw_one = false;
            for (size_t k = 0; k < a_.blocks; ++k) {
                const bool v = (a_.counters[16 * k + bit / 8] >> (bit % 8)) & 1;
                saw_zero = saw_zero || !v;
                saw_one = saw_one || v;
            }
            kind[bit] = !saw_one ? kZero : (!saw_zero ? kOne : kVarying);
            if (kind[bit] == kVarying) varying.push_back(bit);
        }
        // the bit planes of the counters, slot s carrying logical slot s mod logical
        auto plane = [&](const uint8_t* blocks, size_t bit, std::vector<double>& re) {
            for (size_t s = 0; s < slots; ++s) {
                const size_t ls = s % logical;
                re[s] = ls < a_.blocks ? (double)((blocks[16 * ls + bit / 8] >> (bit % 8)) & 1) : 0.0;
            }
        };
        // copies (negated for all-one planes) of the key bits: all limbs for varying planes,
        // which the rescale drops, limbs [0, L) otherwise
        std::vector<LinearJob> copy;
        std::vector<ScalarJob> one;
        for (size_t bit = 0; bit < kStateBits; ++bit) {
            Bit& x = st_[bit];
            const size_t limbs = kind[bit] == kVarying ? L + 1 : L;
            const long double ks = a_.key_scales[bit];
            for (int poly = 0; poly < 2; ++poly)
                for (size_t l = 0; l < limbs; ++l) {
                    LinearJob jb{};
                    jb.out = (poly ? x.a : x.b) + l * N;
                    jb.key = (poly ? a_.key_a[bit] : a_.key_b[bit]) + l * N;
                    jb.kfac = kind[bit] == kOne ? c_.q[l] - 1 : 1;
                    jb.mod = (int)l;
                    copy.push_back(jb);
                }
            x.level = L - 1;
            x.scale = ks;
            if (kind[bit] == kOne)
                for (size_t l = 0; l < L; ++l)
                    one.push_back({x.b + l * N, nullptr, scaled_integer_mod(1, ks, c_.q[l]), 0, (int)l, kScalarAdd});
        }
        launch_jobs(c_, copy, kb_linear, 16.0 * N, "ckks_aes initial copy", s_);
        launch_jobs<true>(c_, one, kb_scalar, 16.0 * N, "ckks_aes initial constant", s_);
        if (varying.empty()) return;
        const size_t nv = varying.size();
        // sign selectors at scale q_L (level L) and the bit planes at the parameter scale (level L - 1)
        const double q_top = static_cast<double>(c_.q[L]);
        std::vector<uint64_t*> signs = ops_.upload_plains_filled(nv, L + 1, [&](uint64_t* host) {
            parallel_encode(nv, [&](size_t k, std::vector<double>& re, std::vector<double>& im) {
                plane(a_.counters, varying[k], re);
                for (double& v : re) v = v == 0.0 ? 1.0 : -1.0;
                host::encode_slots(N, re.data(), im.data(), q_top, c_.q.data(), L + 1, host + k * (L + 1) * N);
            });
        });
        std::vector<uint64_t*> bits = ops_.upload_plains_filled(nv, L, [&](uint64_t* host) {
            parallel_encode(nv, [&](size_t k, std::vector<double>& re, std::vector<double>& im) {
                plane(a_.counters, varying[k], re);
                host::encode_slots(N, re.data(), im.data(), p_.scale, c_.q.data(), L, host + k * L * N);
            });
        });
        std::vector<PmulJob> mul;
        DeviceOps vops(c_, nv, s_);
        CtBatch v;
        v.p.resize(nv);
        for (size_t k = 0; k < nv; ++k) {
            Bit& x = st_[varying[k]];
            v.p[k] = {x.b, x.a, nullptr};
            for (int poly = 0; poly < 2; ++poly)
                for (size_t l = 0; l <= L; ++l) mul.push_back({(poly ? x.a : x.b) + l * N, signs[k] + l * N, (int)l, 0});
        }
        launch_jobs<true>(c_, mul, kb_pmul, 24.0 * N, "ckks_aes sign selector", s_);
        v.np = 2;
        v.level = L;
        v.cap = L + 1;
        vops.rescale(v);
        std::vector<AddJob> add;
        for (size_t k = 0; k < nv; ++k) {
            Bit& x = st_[varying[k]];
            // ckks_mul_inplace(ct, pt) multiplies the scales, ckks_rescale divides by q_L
            x.scale = (static_cast<long double>(a_.key_scales[varying[k]]) * static_cast<long double>(q_top)) /
                      static_cast<long double>(c_.q[L]);
            for (size_t l = 0; l < L; ++l) add.push_back({x.b + l * N, bits[k] + l * N, (int)l, 0});
        }
        launch_jobs<true>(c_, add, kb_add, 24.0 * N, "ckks_aes public bits", s_);
    }

    // sub_bytes_inplace (ckks_aes_ctr.cpp:474-509): the 16 byte positions as S-box instances
    // of one batch per distinct scale of their bit 0 (the S-box relabels to it); st_ -> tmp_
    void sub_bytes() {
        WG_SPAN("xboot.sub_bytes");
        const size_t level = st_[0].level;
        for (const Bit& x : st_)
            if (x.level != level) throw std::invalid_argument("ckks_aes: SubBytes state bits at different levels");
        std::vector<bool> done(16, false);
        for (size_t first = 0; first < 16; ++first) {
            if (done[first]) continue;
            const long double sc = st_[first * 8].scale;
            std::vector<size_t> bytes;
            for (size_t byte = first; byte < 16; ++byte)
                if (!done[byte] && st_[byte * 8].scale == sc) {
                    bytes.push_back(byte);
                    done[byte] = true;
                }
            const size_t n = bytes.size();
            std::vector<uint64_t*> ib(8 * n), ia(8 * n), ob(8 * n), oa(8 * n);
            for (size_t i = 0; i < n; ++i)
                for (size_t k = 0; k < 8; ++k) {
                    ib[k * n + i] = st_[bytes[i] * 8 + k].b;
                    ia[k * n + i] = st_[bytes[i] * 8 + k].a;
                    ob[k * n + i] = tmp_[bytes[i] * 8 + k].b;
                    oa[k * n + i] = tmp_[bytes[i] * 8 + k].a;
                }
            size_t lv[8];
            double osc[8];
            xboot_sbox(c_, n, level, static_cast<double>(sc), ib.data(), ia.data(), ob.data(), oa.data(), lv, osc, s_);
            for (size_t i = 0; i < n; ++i)
                for (size_t k = 0; k < 8; ++k) {
                    tmp_[bytes[i] * 8 + k].level = lv[k];
                    tmp_[bytes[i] * 8 + k].scale = sc;  // the S-box labels every output with its input scale
                }
        }
    }

    // shift_rows_inplace (ckks_aes_ctr.cpp:511-526) on tmp_, then fmix_columns_inplace (:528-554,
    // when `mix`) and add_round_key_lazy_inplace (:460-472, key bits key_base + 0..127) as one
    // fused launch into st_.  Every
    // output is an integer combination of state bits plus the key bit; its scale label is the
    // one the reference's chain of in-place additions keeps (that of its first operand).
    void linear(size_t key_base, bool mix) {
        WG_SPAN("xboot.linear");
        std::array<Bit, kStateBits> sh;
        size_t w = 0;
        for (size_t col = 0; col < 4; ++col)
            for (size_t row = 0; row < 4; ++row) {
                const size_t src = 4 * ((col + row) % 4) + row;
                for (size_t bit = 0; bit < 8; ++bit) sh[w++] = tmp_[src * 8 + bit];
            }
        const size_t level = sh[0].level, N = c_.N;
        for (const Bit& x : sh)
            if (x.level != level) throw std::invalid_argument("ckks_aes: MixColumns state bits at different levels");
        std::vector<SymBit> sym;
        if (mix) {
            sym = mix_symbolic();
        } else {
            sym.assign(kStateBits, SymBit{});
            for (size_t j = 0; j < kStateBits; ++j) sym[j][j] = 1;
        }
        // xtime_byte_lazy's output k starts from input bit kXtimeFirst[k] of the byte's first operand
        static constexpr size_t kXtimeFirst[8] = {7, 0, 1, 2, 3, 4, 5, 6};
        std::vector<LinearJob> jobs;
        for (size_t o = 0; o < kStateBits; ++o) {
            const size_t key = key_base + o;
            if (a_.key_levels[key] < level) throw std::invalid_argument("ckks_aes: round key bit below the state level");
            Bit& x = st_[o];
            x.level = level;
            x.scale = mix ? sh[(o / 8) * 8 + kXtimeFirst[o % 8]].scale : sh[o].scale;
            for (int poly = 0; poly < 2; ++poly)
                for (size_t l = 0; l <= level; ++l) {
                    LinearJob jb{};
                    jb.out = (poly ? x.a : x.b) + l * N;
                    for (size_t j = 0; j < kStateBits; ++j)
                        if (sym[o][j]) {
                            if (jb.n == kMaxLinTerms) throw std::runtime_error("ckks_aes: linear layer too wide");
                            jb.src[jb.n] = (poly ? sh[j].a : sh[j].b) + l * N;
                            jb.cnt[jb.n++] = sym[o][j];
                        }
                    jb.key = (poly ? a_.key_a[key] : a_.key_b[key]) + l * N;
                    jb.kfac = 1;
                    jb.mod = (int)l;
                    jobs.push_back(jb);
                }
        }
        size_t words = 0;
        for (const auto& jb : jobs) words += jb.n + 2;
        launch_jobs(c_, jobs, kb_linear, 8.0 * N * (double)words / (double)jobs.size(), "ckks_aes linear layer", s_);
    }

    // xboot_state_inplace (ckks_aes_ctr.cpp:556-574): the pair bootstrap of bits (2p, 2p + 1),
    // all 64 pairs batched (pairs grouped by the scale of their first bit, which labels the
    // packed ciphertext), in place in st_
    void refresh() {
        WG_SPAN("xboot.refresh");
        for (const Bit& x : st_)
            if (x.level != p_.s2c_depth)
                throw std::invalid_argument("ckks_batch_bootstrap_evalmod: expected ciphertext level to equal S2C depth");
        const size_t batch = std::max<size_t>(1, a_.pair_batch);
        std::vector<bool> done(kStateBits / 2, false);
        for (size_t first = 0; first < kStateBits / 2; ++first) {
            if (done[first]) continue;
            const long double sc = st_[2 * first].scale;
            std::vector<size_t> pairs;
            for (size_t pr = first; pr < kStateBits / 2; ++pr)
                if (!done[pr] && st_[2 * pr].scale == sc) {
                    pairs.push_back(pr);
                    done[pr] = true;
                }
            for (size_t k0 = 0; k0 < pairs.size(); k0 += batch) {
                const size_t n = std::min(batch, pairs.size() - k0);
                std::vector<uint64_t*> b0(n), a0(n), b1(n), a1(n);
                for (size_t i = 0; i < n; ++i) {
                    const size_t pr = pairs[k0 + i];
                    b0[i] = st_[2 * pr].b;
                    a0[i] = st_[2 * pr].a;
                    b1[i] = st_[2 * pr + 1].b;
                    a1[i] = st_[2 * pr + 1].a;
                }
                size_t lv = 0;
                double osc = 0.0;
                bootstrap_pair(c_, p_, plans_, nplans_, c2s_, nc2s_, coeffs_, ncoeffs_, n, static_cast<double>(sc),
                               b0.data(), a0.data(), b1.data(), a1.data(), &lv, &osc, s_);
                for (size_t i = 0; i < n; ++i)
                    for (size_t k = 0; k < 2; ++k) {
                        st_[2 * pairs[k0 + i] + k].level = lv;
                        st_[2 * pairs[k0 + i] + k].scale = osc;
                    }
            }
        }
    }

    // encode_message_block (ckks_aes_ctr.cpp:337-363) of every bit at the parameter scale, added
    // to the state bits (ckks_add_inplace(ct, pt))
    void add_message() {
        WG_SPAN("xboot.add_message");
        const size_t N = c_.N, slots = N / 2, logical = p_.active_slots, level = st_[0].level, L = level + 1;
        for (const Bit& x : st_)
            if (x.level != level) throw std::invalid_argument("ckks_aes: state bits at different levels");
        std::vector<uint64_t*> pts = ops_.upload_plains_filled(kStateBits, L, [&](uint64_t* host) {
            parallel_encode(kStateBits, [&](size_t bit, std::vector<double>& re, std::vector<double>& im) {
                for (size_t s = 0; s < slots; ++s) {
                    const size_t ls = s % logical;
                    re[s] = ls < a_.blocks ? (double)((a_.ciphertexts[16 * ls + bit / 8] >> (bit % 8)) & 1) : 0.0;
                }
                host::encode_slots(N, re.data(), im.data(), p_.scale, c_.q.data(), L, host + bit * L * N);
            });
        });
        std::vector<AddJob> add;
        for (size_t bit = 0; bit < kStateBits; ++bit)
            for (size_t l = 0; l < L; ++l) add.push_back({st_[bit].b + l * N, pts[bit] + l * N, (int)l, 0});
        launch_jobs<true>(c_, add, kb_add, 24.0 * N, "ckks_aes message bits", s_);
    }

    void copy_out(uint64_t* const* out_b, uint64_t* const* out_a, size_t* out_level, double* out_scale) {
        for (size_t bit = 0; bit < kStateBits; ++bit) {
            const Bit& x = st_[bit];
            const size_t bytes = (x.level + 1) * c_.N * 8;
            check_cuda(cudaMemcpyAsync(out_b[bit], x.b, bytes, cudaMemcpyDeviceToDevice, s_), "ckks_aes output");
            check_cuda(cudaMemcpyAsync(out_a[bit], x.a, bytes, cudaMemcpyDeviceToDevice, s_), "ckks_aes output");
            out_level[bit] = x.level;
            out_scale[bit] = static_cast<double>(x.scale);
        }
    }

private:
    // fill(k, re, im) for k < n on host threads; re / im are zeroed slot vectors per call
    template <class F>
    void parallel_encode(size_t n, F&& fill) {
        const size_t slots = c_.N / 2;
        const size_t nthreads = std::max<size_t>(1, std::min<size_t>({16, n, std::thread::hardware_concurrency()}));
        std::vector<std::thread> pool;
        std::vector<std::exception_ptr> errs(nthreads);
        for (size_t w = 0; w < nthreads; ++w)
            pool.emplace_back([&, w] {
                try {
                    std::vector<double> re(slots), im(slots);
                    for (size_t k = w; k < n; k += nthreads) {
                        std::fill(re.begin(), re.end(), 0.0);
                        std::fill(im.begin(), im.end(), 0.0);
                        fill(k, re, im);
                    }
                } catch (...) {
                    errs[w] = std::current_exception();
                }
            });
        for (auto& th : pool) th.join();
        for (auto& e : errs)
            if (e) std::rethrow_exception(e);
    }

    Context& c_;
    const BootstrapParams& p_;
    const S2cPlan* plans_;
    size_t nplans_;
    const LtStage* const* c2s_;
    size_t nc2s_;
    const double* coeffs_;
    size_t ncoeffs_;
    const XbootAesArgs& a_;
    cudaStream_t s_;
    DeviceOps ops_;  // owns the state buffers and the public plaintexts
    std::array<Bit, kStateBits> st_, tmp_;
};

}  // namespace

void aes_ctr_xboot(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                   size_t nc2s, const double* coeffs, size_t ncoeffs, const XbootAesArgs& a, uint64_t* const* out_b,
                   uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s) {
    const size_t logical = p.active_slots;
    if (a.blocks == 0 || a.blocks > logical)
        throw std::invalid_argument("ckks_aes: public counter count exceeds logical slot count");
    if (!a.key_b || !a.key_a || !a.key_scales || !a.key_levels || !a.counters || !a.ciphertexts)
        throw std::invalid_argument("ckks_aes: null argument");
    for (size_t k = 0; k < 1408; ++k)
        if (a.key_levels[k] >= c.nq) throw std::invalid_argument("ckks_aes: invalid round key bit level");
    XbootAes aes(c, p, s2c, nplans, c2s, nc2s, coeffs, ncoeffs, a, s);
    aes.initial_state();
    for (size_t round = 1; round <= kAesRounds; ++round) {
        aes.sub_bytes();
        aes.linear(round * kStateBits, round < kAesRounds);
        if (round < kAesRounds) aes.refresh();
    }
    aes.add_message();
    aes.refresh();
    aes.copy_out(out_b, out_a, out_level, out_scale);
}

void xboot_initial_state(Context& c, const BootstrapParams& p, const XbootAesArgs& a, uint64_t* const* out_b,
                         uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s) {
    if (a.blocks == 0 || a.blocks > p.active_slots)
        throw std::invalid_argument("ckks_aes: public counter count exceeds logical slot count");
    if (!a.key_b || !a.key_a || !a.key_scales || !a.key_levels || !a.counters)
        throw std::invalid_argument("ckks_aes: null argument");
    if (a.key_levels[0] >= c.nq) throw std::invalid_argument("ckks_aes: invalid round key bit level");
    XbootAes aes(c, p, nullptr, 0, nullptr, 0, nullptr, 0, a, s, false);
    for (size_t bit = 0; bit < kStateBits; ++bit) {
        aes.state(bit).b = out_b[bit];
        aes.state(bit).a = out_a[bit];
    }
    aes.initial_state();
    *out_level = aes.state(0).level;
    for (size_t bit = 0; bit < kStateBits; ++bit) out_scale[bit] = static_cast<double>(aes.state(bit).scale);
}

void xboot_linear_layer(Context& c, size_t level, const double* in_scale, uint64_t* const* in_b,
                        uint64_t* const* in_a, const XbootAesArgs& a, bool mix, uint64_t* const* out_b,
                        uint64_t* const* out_a, double* out_scale, cudaStream_t s) {
    if (level >= c.nq) throw std::invalid_argument("ckks_aes: invalid state level");
    if (!a.key_b || !a.key_a || !a.key_levels) throw std::invalid_argument("ckks_aes: null argument");
    BootstrapParams none;
    XbootAes aes(c, none, nullptr, 0, nullptr, 0, nullptr, 0, a, s, false);
    for (size_t bit = 0; bit < kStateBits; ++bit) {
        Bit& x = aes.staged(bit);
        x.b = in_b[bit];
        x.a = in_a[bit];
        x.level = level;
        x.scale = in_scale[bit];
        aes.state(bit).b = out_b[bit];
        aes.state(bit).a = out_a[bit];
    }
    aes.linear(0, mix);
    for (size_t bit = 0; bit < kStateBits; ++bit) out_scale[bit] = static_cast<double>(aes.state(bit).scale);
}

void xboot_encrypt_round_key_bits(Context& c, const BootstrapParams& p, const uint8_t* expanded_key,
                                  size_t first_round_key_level, const int8_t* secret, uint64_t seed, double sigma,
                                  uint64_t* const* out_b, uint64_t* const* out_a, double* out_scale,
                                  size_t* out_level, cudaStream_t s) {
    if (!expanded_key) throw std::invalid_argument("ckks_aes: null expanded key");
    const size_t base = p.s2c_depth;
    if (base + first_round_key_level > c.nq - 1)
        throw std::invalid_argument("ckks_aes: invalid encryption level for first round key bits");
    constexpr size_t kKeyBits = 11 * kStateBits;
    DeviceOps ops(c, 1, s);
    // round 0 at base + first_round_key_level, the other rounds at base; plaintext of the bit's
    // value in every slot at the parameter scale (closed-form constant encodings)
    for (int round0 = 1; round0 >= 0; --round0) {
        const size_t level = round0 ? base + first_round_key_level : base;
        const size_t k0 = round0 ? 0 : kStateBits, k1 = round0 ? kStateBits : kKeyBits;
        const uint64_t* pt[2] = {ops.constant_plaintext(level + 1, 0.0, 0.0, p.scale),
                                 ops.constant_plaintext(level + 1, 1.0, 0.0, p.scale)};
        std::vector<const uint64_t*> pts;
        std::vector<uint64_t*> ob, oa;
        for (size_t k = k0; k < k1; ++k) {
            const int bit = (expanded_key[k / 8] >> (k % 8)) & 1;
            pts.push_back(pt[bit]);
            ob.push_back(out_b[k]);
            oa.push_back(out_a[k]);
            out_scale[k] = p.scale;
            out_level[k] = level;
        }
        encrypt_symmetric(c, pts.size(), level, pts.data(), secret, nullptr, nullptr, seed + (uint64_t)round0, sigma,
                          ob.data(), oa.data(), s);
    }
}

}  // namespace wg
