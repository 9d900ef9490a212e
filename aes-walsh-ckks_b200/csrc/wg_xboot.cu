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
#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>

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

}  // namespace wg
