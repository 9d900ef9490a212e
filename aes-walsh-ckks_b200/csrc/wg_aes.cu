// AES-128 in CTR mode on lazy bits, evaluated homomorphically: 128 bit ciphertexts, each slot
// carrying two AES blocks (real and imaginary lane), SubBytes by the mask-packed Walsh S-box
// (all 16 byte positions in one batch), ShiftRows as a relabelling, MixColumns and AddRoundKey
// as lazy additions, and a final binary refresh by packed bootstraps.
//
// Reference: ckks_aes_ctr_walsh_sbox_complex_blocks and its helpers,
// src/ckks/operations/circuits/aes/ckks_aes_ctr_walsh_sbox.cpp:42-1051.  Residues depend on the
// order of every addition and on every plaintext and scale factor, so the host side follows
// the reference's steps in the same order with the same long-double scale bookkeeping, and the
// public plaintexts (counter and ciphertext bit patterns, active-slot masks) come from the host
// encoder whose FP64 rounding matches the reference's (wg_encode.cpp).
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <exception>
#include <thread>
#include <vector>

#include "wg_aes_linear.cuh"
#include "wg_ctops.cuh"
#include "wg_encode.hpp"

namespace wg {
namespace {

constexpr size_t kBlockBits = 128;
constexpr size_t kRounds = 10;
constexpr size_t kKeyBits = 1408;
constexpr size_t kMinSegments = 30;

bool aes_close(long double l, long double r, long double tol = 0x1p-45L) {
    if (!std::isfinite(l) || !std::isfinite(r)) return false;
    const long double m = std::max<long double>({1.0L, std::abs(l), std::abs(r)});
    return std::abs(l - r) <= tol * m;
}

using Bits = std::vector<CtBatch>;  // one ciphertext per entry (batch count 1)

class Aes {
public:
    Aes(Context& c, DeviceOps& ops, const BootstrapParams& p, const S2cPlan* plans, size_t nplans,
        const LtStage* const* c2s, size_t nc2s, const double* coeffs, size_t ncoeffs, cudaStream_t s)
        : c_(c), ops_(ops), p_(p), plans_(plans), nplans_(nplans), c2s_(c2s), nc2s_(nc2s), coeffs_(coeffs),
          ncoeffs_(ncoeffs), s_(s) {}

    // ---- public plaintexts (evaluation form, level+1 limbs)
    uint64_t* encode(const std::vector<double>& re, const std::vector<double>& im, long double scale, size_t level) {
        std::vector<uint64_t> coeff((level + 1) * c_.N);
        host::encode_slots(c_.N, re.data(), im.data(), static_cast<double>(scale), c_.q.data(), level + 1, coeff.data());
        return ops_.upload_plain(coeff.data(), level + 1);
    }

    // encode_active_complex_block_public_bit: slot s = (bit of block s, bit of block acb + s)
    uint64_t* public_bit(const uint8_t* blocks, size_t bit, size_t acb, size_t level, long double scale) {
        std::vector<double> re(c_.N / 2, 0.0), im(c_.N / 2, 0.0);
        for (size_t s = 0; s < acb; ++s) {
            re[s] = (double)((blocks[16 * s + bit / 8] >> (bit % 8)) & 1);
            im[s] = (double)((blocks[16 * (acb + s) + bit / 8] >> (bit % 8)) & 1);
        }
        return encode(re, im, scale, level);
    }

    // encode_active_slot_mask: 1 in the first `count` slots
    uint64_t* slot_mask(size_t count, size_t level, long double scale) {
        std::vector<double> re(c_.N / 2, 0.0), im(c_.N / 2, 0.0);
        for (size_t s = 0; s < count; ++s) re[s] = 1.0;
        return encode(re, im, scale, level);
    }

    // ---- scale alignment with the AES path's tolerances
    void mul_integer(CtBatch& x, long double scalar, long double out_scale) {
        if (!std::isfinite(scalar) || scalar < 0.0L) throw std::invalid_argument("ckks_aes_walsh: invalid scalar scale-up");
        const long double r = std::round(scalar);
        if (r < 1.0L || std::abs(scalar - r) > std::max<long double>(1.0L, std::abs(scalar)) * 1e-3L)
            throw std::invalid_argument("ckks_aes_walsh: non-integral scalar scale-up");
        if (r > static_cast<long double>(std::numeric_limits<int64_t>::max()))
            throw std::invalid_argument("ckks_aes_walsh: scalar scale-up is too large");
        const int64_t k = static_cast<int64_t>(r);
        if (k != 1) ops_.mul_int(x, k);
        x.scale = out_scale;
    }

    void align_exact(CtBatch& x, size_t level, long double scale, int np) {
        if (level > x.level) throw std::invalid_argument("ckks_drop_to_level_inplace: cannot raise ciphertext level");
        x.level = level;
        ops_.pad(x, np);
        if (aes_close(x.scale, scale)) {
            x.scale = scale;
            return;
        }
        // (an all-zero ciphertext is also accepted by the reference; zero times an integer is
        // zero, so the residues agree)
        if (x.scale > scale) throw std::invalid_argument("ckks_aes_walsh: cannot scale down ciphertext for addition");
        mul_integer(x, scale / x.scale, scale);
    }

    void add_term(CtBatch& acc, CtBatch term) {
        const size_t level = std::min(acc.level, term.level);
        const long double scale = std::max(acc.scale, term.scale);
        const int np = std::max(acc.np, term.np);
        align_exact(acc, level, scale, np);
        align_exact(term, level, scale, np);
        ops_.add(acc, term, false);
    }

    CtBatch add_bits(const CtBatch& l, const CtBatch& r) {
        CtBatch out = ops_.clone(l);
        add_term(out, ops_.clone(r));
        return out;
    }

    // ---- the round layers
    Bits initial_state(const AesArgs& a) {
        Bits st(kBlockBits);
        for (size_t bit = 0; bit < kBlockBits; ++bit) {
            CtBatch k = key_bit(a, bit);
            st[bit] = ops_.clone(k);
            ops_.add_plain(st[bit], public_bit(a.counters, bit, a.active_blocks, st[bit].level, st[bit].scale));
        }
        return st;
    }

    CtBatch key_bit(const AesArgs& a, size_t k) {
        uint64_t* b = const_cast<uint64_t*>(a.key_b[k]);
        uint64_t* pa = const_cast<uint64_t*>(a.key_a[k]);
        return ops_.wrap(&b, &pa, a.key_level, static_cast<long double>(a.key_scales[k]));
    }

    // mask_inactive_slots_inplace: x <- rescale(x * mask), mask = 1 on the packing slots at
    // scale q_level; the scale is then reset to the state's
    void mask_inactive(Bits& st, size_t pack_count) {
        WG_SPAN("aes.mask");
        const size_t level = st[0].level;
        if (level <= p_.s2c_depth)
            throw std::invalid_argument("ckks_aes_walsh: active slot mask requires a selection limb above S2C input level");
        const long double target = st[0].scale;
        const uint64_t* mask = slot_mask(pack_count, level, static_cast<long double>(c_.q[level]));
        mul_plain_rescale(st, mask, level, true, target, true);
    }

    void mul_plain_rescale(Bits& st, const uint64_t* mask, size_t level, bool rescale, long double target,
                           bool check_scale) {
        DeviceOps all(c_, st.size(), s_);
        CtBatch x;
        x.p.resize(st.size());
        for (size_t i = 0; i < st.size(); ++i) {
            if (st[i].level != level) throw std::invalid_argument("ckks_aes_walsh: active slot mask level mismatch");
            if (check_scale && !aes_close(st[i].scale, target))
                throw std::invalid_argument("ckks_aes_walsh: active slot mask scale mismatch");
            x.p[i] = st[i].p[0];
        }
        x.np = 2;
        x.level = level;
        x.cap = level + 1;
        all.mul_plain(x, mask);
        if (rescale) all.rescale(x);
        for (auto& b : st) {
            b.level = x.level;
            if (rescale) b.scale = target;
        }
    }

    // SubBytes: the 16 byte positions as one batch of 16 Walsh S-box instances
    Bits sub_bytes(const Bits& st, size_t pack_count) {
        WG_SPAN("aes.sub_bytes");
        const size_t level = st[0].level;
        const size_t full = p_.depth + 1;
        std::vector<uint64_t*> ib(kBlockBits), ia(kBlockBits), ob(kBlockBits), oa(kBlockBits);
        for (size_t byte = 0; byte < 16; ++byte)
            for (size_t k = 0; k < 8; ++k) {
                ib[k * 16 + byte] = st[byte * 8 + k].p[0][0];
                ia[k * 16 + byte] = st[byte * 8 + k].p[0][1];
                ob[k * 16 + byte] = ops_.raw(full);
                oa[k * 16 + byte] = ops_.raw(full);
            }
        size_t lv[8];
        double sc[8];
        if (!per_instance_) {
            walsh_sbox(c_, p_, plans_, nplans_, c2s_, nc2s_, coeffs_, ncoeffs_, pack_count, 16, level,
                       static_cast<double>(st[0].scale), ib.data(), ia.data(), ob.data(), oa.data(), lv, sc, s_);
        } else {
            // one S-box instance per call: its 8 bit pointers, bit-major with count 1
            for (size_t byte = 0; byte < 16; ++byte) {
                uint64_t* i1b[8];
                uint64_t* i1a[8];
                uint64_t* o1b[8];
                uint64_t* o1a[8];
                for (size_t k = 0; k < 8; ++k) {
                    i1b[k] = ib[k * 16 + byte];
                    i1a[k] = ia[k * 16 + byte];
                    o1b[k] = ob[k * 16 + byte];
                    o1a[k] = oa[k * 16 + byte];
                }
                walsh_sbox(c_, p_, plans_, nplans_, c2s_, nc2s_, coeffs_, ncoeffs_, pack_count, 1, level,
                           static_cast<double>(st[0].scale), i1b, i1a, o1b, o1a, lv, sc, s_);
            }
        }
        Bits out(kBlockBits);
        for (size_t byte = 0; byte < 16; ++byte)
            for (size_t k = 0; k < 8; ++k) {
                CtBatch& x = out[byte * 8 + k];
                x.p = {{ob[k * 16 + byte], oa[k * 16 + byte], nullptr}};
                x.np = 2;
                x.level = lv[k];
                x.cap = full;
                x.scale = sc[k];
            }
        return out;
    }

    static void shift_rows(Bits& st) {
        Bits old = st;
        size_t w = 0;
        for (size_t col = 0; col < 4; ++col)
            for (size_t row = 0; row < 4; ++row) {
                const size_t src = 4 * ((col + row) % 4) + row;
                for (size_t bit = 0; bit < 8; ++bit) st[w++] = old[src * 8 + bit];
            }
    }

    using Byte = std::vector<CtBatch>;

    Byte byte_of(const Bits& st, size_t byte) {
        Byte b(8);
        for (size_t k = 0; k < 8; ++k) b[k] = ops_.clone(st[byte * 8 + k]);
        return b;
    }

    Byte add_bytes(const Byte& l, const Byte& r) {
        Byte o(8);
        for (size_t k = 0; k < 8; ++k) o[k] = add_bits(l[k], r[k]);
        return o;
    }

    void add_byte(Byte& acc, const Byte& t) {
        for (size_t k = 0; k < 8; ++k) add_term(acc[k], ops_.clone(t[k]));
    }

    // xtime on lazy bits: multiplication by x in GF(2^8) as additions
    Byte xtime(const Byte& b) {
        Byte o;
        o.push_back(ops_.clone(b[7]));
        o.push_back(add_bits(b[0], b[7]));
        o.push_back(ops_.clone(b[1]));
        o.push_back(add_bits(b[2], b[7]));
        o.push_back(add_bits(b[3], b[7]));
        o.push_back(ops_.clone(b[4]));
        o.push_back(ops_.clone(b[5]));
        o.push_back(ops_.clone(b[6]));
        return o;
    }

    Byte mix_byte(const Byte& b0, const Byte& b1, const Byte& b2, const Byte& b3) {
        Byte d = xtime(add_bytes(b0, b1));
        add_byte(d, b1);
        add_byte(d, b2);
        add_byte(d, b3);
        return d;
    }

    void mix_columns(Bits& st) {
        std::vector<Byte> out(16);
        for (size_t col = 0; col < 4; ++col) {
            const Byte b0 = byte_of(st, 4 * col), b1 = byte_of(st, 4 * col + 1), b2 = byte_of(st, 4 * col + 2),
                       b3 = byte_of(st, 4 * col + 3);
            out[4 * col + 0] = mix_byte(b0, b1, b2, b3);
            out[4 * col + 1] = mix_byte(b1, b2, b3, b0);
            out[4 * col + 2] = mix_byte(b2, b3, b0, b1);
            out[4 * col + 3] = mix_byte(b3, b0, b1, b2);
        }
        for (size_t byte = 0; byte < 16; ++byte)
            for (size_t k = 0; k < 8; ++k) st[byte * 8 + k] = out[byte][k];
    }

    void add_round_key(Bits& st, const AesArgs& a, size_t round) {
        for (size_t bit = 0; bit < kBlockBits; ++bit) add_term(st[bit], ops_.clone(key_bit(a, round * kBlockBits + bit)));
    }

    void add_public(Bits& st, const uint8_t* blocks, size_t acb) {
        for (size_t bit = 0; bit < kBlockBits; ++bit)
            ops_.add_plain(st[bit], public_bit(blocks, bit, acb, st[bit].level, st[bit].scale));
    }

    // MixColumns (when `mix`) and AddRoundKey as one launch: every output bit is a sum of state
    // bits with small multiplicities plus the round-key bit scaled up to the state scale.
    // Taken when the state bits share level and scale and the round-key bits are not above the
    // state scale (the reference then adds without re-aligning the state); otherwise the
    // operation-by-operation path.
    void linear_layer(Bits& st, const AesArgs& a, size_t round, bool mix) {
        WG_SPAN("aes.linear");
        const size_t level = st[0].level, L = level + 1, N = c_.N;
        const long double S = st[0].scale;
        bool uniform = a.key_level >= level;
        for (const auto& b : st) uniform = uniform && b.level == level && b.scale == S && b.np == 2;
        for (size_t bit = 0; bit < kBlockBits; ++bit) {
            const long double ks = a.key_scales[round * kBlockBits + bit];
            uniform = uniform && std::isfinite(ks) && !(ks > S && !aes_close(ks, S));
        }
        if (!uniform) {
            if (mix) mix_columns(st);
            add_round_key(st, a, round);
            return;
        }
        std::vector<SymBit> sym;
        if (mix) {
            sym = mix_symbolic();
        } else {
            sym.assign(128, SymBit{});
            for (size_t j = 0; j < 128; ++j) sym[j][j] = 1;
        }
        Bits out(kBlockBits);
        std::vector<LinearJob> jobs;
        for (size_t o = 0; o < kBlockBits; ++o) {
            // the key bit's scale-up factor (multiply_by_integer_scalar_inplace on the key clone);
            // a key bit within tolerance of the state scale only relabels the sum's scale
            const long double ks = a.key_scales[round * kBlockBits + o];
            uint64_t k = 1;
            out[o] = ops_.alloc(level, 2);
            out[o].scale = S;
            if (aes_close(ks, S)) {
                out[o].scale = std::max(S, ks);
            } else {
                const long double ratio = S / ks, r = std::round(ratio);
                if (r < 1.0L || std::abs(ratio - r) > std::max<long double>(1.0L, std::abs(ratio)) * 1e-3L)
                    throw std::invalid_argument("ckks_aes_walsh: non-integral scalar scale-up");
                if (r > static_cast<long double>(std::numeric_limits<int64_t>::max()))
                    throw std::invalid_argument("ckks_aes_walsh: scalar scale-up is too large");
                k = (uint64_t)r;
            }
            CtBatch key = key_bit(a, round * kBlockBits + o);
            for (int poly = 0; poly < 2; ++poly)
                for (size_t l = 0; l < L; ++l) {
                    LinearJob jb{};
                    jb.out = out[o].p[0][poly] + l * N;
                    for (size_t j = 0; j < 128; ++j)
                        if (sym[o][j]) {
                            if (jb.n == kMaxLinTerms) throw std::runtime_error("ckks_aes_walsh: linear layer too wide");
                            jb.src[jb.n] = st[j].p[0][poly] + l * N;
                            jb.cnt[jb.n++] = sym[o][j];
                        }
                    jb.key = key.p[0][poly] + l * N;
                    jb.kfac = k % c_.q[l];
                    jb.mod = (int)l;
                    jobs.push_back(jb);
                }
        }
        launch_linear(jobs);
        st = out;
    }

    void launch_linear(const std::vector<LinearJob>& jobs) {
        size_t words = 0;
        for (const auto& jb : jobs) words += jb.n + 1 + (jb.key ? 1 : 0);
        JobTable t;
        const LinearJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsElementwise, 8.0 * c_.N * words, s_);
        kb_linear<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "aes linear layer");
    }

    // public bit patterns of all 128 state bits at the bits' level and scale, added in one
    // launch (encodings on host threads, one staged upload)
    void add_public_all(Bits& st, const uint8_t* blocks, size_t acb) {
        WG_SPAN("aes.add_public");
        const size_t level = st[0].level, L = level + 1, N = c_.N;
        bool uniform = true;
        for (const auto& b : st) uniform = uniform && b.level == level;
        if (!uniform) {
            add_public(st, blocks, acb);
            return;
        }
        std::vector<double> scale(kBlockBits);
        for (size_t bit = 0; bit < kBlockBits; ++bit) scale[bit] = static_cast<double>(st[bit].scale);
        std::vector<uint64_t*> pts = ops_.upload_plains_filled(
            kBlockBits, L, [&](uint64_t* host) { encode_bits_parallel(blocks, acb, scale, L, host); });
        DeviceOps all(c_, kBlockBits, s_);
        std::vector<AddJob> jobs;
        for (size_t bit = 0; bit < kBlockBits; ++bit)
            for (size_t l = 0; l < L; ++l) jobs.push_back({st[bit].p[0][0] + l * N, pts[bit] + l * N, (int)l, 0});
        all.add_jobs(jobs);
    }

    // the 128 bit patterns of `blocks`, encoded on host threads into out[bit][L][N]
    void encode_bits_parallel(const uint8_t* blocks, size_t acb, const std::vector<double>& scale, size_t L,
                              uint64_t* out) {
        const size_t nthreads = std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        std::vector<std::exception_ptr> errs(nthreads);
        for (size_t w = 0; w < nthreads; ++w)
            pool.emplace_back([&, w] {
                try {
                    std::vector<double> re(c_.N / 2), im(c_.N / 2);
                    for (size_t bit = w; bit < kBlockBits; bit += nthreads) {
                        std::fill(re.begin(), re.end(), 0.0);
                        std::fill(im.begin(), im.end(), 0.0);
                        for (size_t s = 0; s < acb; ++s) {
                            re[s] = (double)((blocks[16 * s + bit / 8] >> (bit % 8)) & 1);
                            im[s] = (double)((blocks[16 * (acb + s) + bit / 8] >> (bit % 8)) & 1);
                        }
                        host::encode_slots(c_.N, re.data(), im.data(), scale[bit], c_.q.data(), L,
                                           out + bit * L * c_.N);
                    }
                } catch (...) {
                    errs[w] = std::current_exception();
                }
            });
        for (auto& th : pool) th.join();
        for (auto& e : errs)
            if (e) std::rethrow_exception(e);
    }

    // initial state: key bit + counter bit pattern, all 128 bits at once
    Bits initial_state_fast(const AesArgs& a) {
        WG_SPAN("aes.initial");
        const size_t level = a.key_level, L = level + 1, N = c_.N;
        std::vector<double> scale(kBlockBits);
        for (size_t bit = 0; bit < kBlockBits; ++bit) scale[bit] = a.key_scales[bit];
        std::vector<uint64_t*> pts = ops_.upload_plains_filled(
            kBlockBits, L, [&](uint64_t* host) { encode_bits_parallel(a.counters, a.active_blocks, scale, L, host); });
        Bits st(kBlockBits);
        std::vector<LinearJob> jobs;
        for (size_t bit = 0; bit < kBlockBits; ++bit) {
            st[bit] = ops_.alloc(level, 2);
            st[bit].scale = a.key_scales[bit];
            const CtBatch key = key_bit(a, bit);
            for (int poly = 0; poly < 2; ++poly)
                for (size_t l = 0; l < L; ++l) {
                    LinearJob jb{};
                    jb.out = st[bit].p[0][poly] + l * N;
                    jb.src[0] = key.p[0][poly] + l * N;
                    jb.cnt[0] = 1;
                    jb.n = 1;
                    jb.key = poly == 0 ? pts[bit] + l * N : nullptr;
                    jb.kfac = 1;
                    jb.mod = (int)l;
                    jobs.push_back(jb);
                }
        }
        launch_linear(jobs);
        return st;
    }

    // mask_final_refresh_slots_inplace
    void refresh_mask(Bits& st, size_t active, size_t min_keep) {
        const size_t level = st[0].level;
        const bool consume = level > min_keep;
        const long double target = st[0].scale;
        const long double mask_scale = consume ? static_cast<long double>(c_.q[level]) : 1.0L;
        const uint64_t* mask = slot_mask(active, level, mask_scale);
        mul_plain_rescale(st, mask, level, consume, target, false);
    }

    // final_binary_refresh_complex_block_output_bits_inplace; bops (one ciphertext per packed
    // lane) owns the refreshed bits, so it must outlive `st`
    static size_t refresh_batches(size_t slots, size_t acb) {
        const size_t per = acb ? slots / acb : 0;
        if (acb == 0 || per == 0 || acb * per > slots)
            throw std::invalid_argument("ckks_aes_walsh: invalid final refresh packing layout");
        return (kBlockBits + per - 1) / per;
    }

    void final_refresh(Bits& st, size_t acb, DeviceOps& bops) {
        WG_SPAN("aes.final_refresh");
        const size_t slots = c_.N / 2;
        const size_t stride = acb, per = slots / stride;
        const size_t batches = refresh_batches(slots, acb);
        if (bops.count() != batches) throw std::invalid_argument("ckks_aes_walsh: refresh batch count mismatch");
        refresh_mask(st, stride, p_.s2c_depth);
        const size_t N = c_.N, full = p_.depth + 1;
        // pack: segment s of batch b holds bit b * per + s, rotated by s * stride
        CtBatch packed = bops.zeros(st[0].level, st[0].scale);
        for (size_t seg = 0; seg < per; ++seg) {
            CtBatch term;
            term.p.resize(batches);
            term.np = 2;
            term.level = st[0].level;
            term.scale = st[0].scale;
            bool any = false;
            std::vector<size_t> idx;
            for (size_t b = 0; b < batches; ++b) {
                const size_t bit = b * per + seg;
                idx.push_back(bit);
                any |= bit < kBlockBits;
            }
            if (!any) break;
            // a batch without this segment adds zeros (its packing loop stops there)
            for (size_t b = 0; b < batches; ++b) {
                if (idx[b] < kBlockBits) {
                    term.p[b] = st[idx[b]].p[0];
                } else {
                    uint64_t* zb = bops.raw(st[0].level + 1);
                    uint64_t* za = bops.raw(st[0].level + 1);
                    check_cuda(cudaMemsetAsync(zb, 0, (st[0].level + 1) * N * 8, s_), "zero");
                    check_cuda(cudaMemsetAsync(za, 0, (st[0].level + 1) * N * 8, s_), "zero");
                    term.p[b] = {zb, za, nullptr};
                }
            }
            term.cap = st[0].level + 1;
            CtBatch t = bops.clone(term);
            if (seg) bops.rotate(t, (int64_t)(seg * stride));
            bops.add(packed, t, false);
        }
        // bootstrap all packed lanes at once; the packed buffers need room for depth+1 limbs
        std::vector<uint64_t*> pb(batches), pa(batches), o0b(batches), o0a(batches), o1b(batches), o1a(batches);
        for (size_t b = 0; b < batches; ++b) {
            pb[b] = bops.raw(full);
            pa[b] = bops.raw(full);
            for (auto* v : {&o0b, &o0a, &o1b, &o1a}) (*v)[b] = bops.raw(full);
            check_cuda(cudaMemcpyAsync(pb[b], packed.p[b][0], (packed.level + 1) * N * 8, cudaMemcpyDeviceToDevice, s_),
                       "refresh pack");
            check_cuda(cudaMemcpyAsync(pa[b], packed.p[b][1], (packed.level + 1) * N * 8, cudaMemcpyDeviceToDevice, s_),
                       "refresh pack");
        }
        size_t blv = 0;
        double bsc = 0.0;
        if (!per_instance_) {
            bootstrap_evalmod(c_, p_, plans_, nplans_, c2s_, nc2s_, coeffs_, ncoeffs_, batches,
                              static_cast<double>(packed.scale), pb.data(), pa.data(), o0b.data(), o0a.data(),
                              o1b.data(), o1a.data(), &blv, &bsc, s_);
        } else {
            for (size_t b = 0; b < batches; ++b)
                bootstrap_evalmod(c_, p_, plans_, nplans_, c2s_, nc2s_, coeffs_, ncoeffs_, 1,
                                  static_cast<double>(packed.scale), &pb[b], &pa[b], &o0b[b], &o0a[b], &o1b[b],
                                  &o1a[b], &blv, &bsc, s_);
        }
        CtBatch real = bops.wrap(o0b.data(), o0a.data(), blv, bsc);
        CtBatch imag = bops.wrap(o1b.data(), o1a.data(), blv, bsc);
        real.cap = imag.cap = full;
        bops.mul_complex_constant(imag, 0.0, 1.0, 1.0);
        bops.add(real, imag, false);
        // unpack: bit b * per + s = combined rotated back by s * stride
        Bits out(kBlockBits);
        for (size_t seg = 0; seg < per; ++seg) {
            CtBatch t = bops.clone(real);
            if (seg) bops.rotate(t, -(int64_t)(seg * stride));
            for (size_t b = 0; b < batches; ++b) {
                const size_t bit = b * per + seg;
                if (bit >= kBlockBits) continue;
                CtBatch& x = out[bit];
                x.p = {t.p[b]};
                x.np = 2;
                x.level = t.level;
                x.cap = t.cap;
                x.scale = real.scale;
            }
        }
        st = out;
        refresh_mask(st, stride, 0);
    }

    void set_per_instance(bool v) { per_instance_ = v; }

private:
    bool per_instance_ = false;
    Context& c_;
    DeviceOps& ops_;
    const BootstrapParams& p_;
    const S2cPlan* plans_;
    size_t nplans_;
    const LtStage* const* c2s_;
    size_t nc2s_;
    const double* coeffs_;
    size_t ncoeffs_;
    cudaStream_t s_;
};

}  // namespace

void aes_ctr_walsh(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                   size_t nc2s, const double* coeffs, size_t ncoeffs, const AesArgs& a, uint64_t* const* out_b,
                   uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s) {
    const size_t slots = c.N / 2;
    if (a.active_blocks == 0) throw std::invalid_argument("ckks_aes_walsh: complex-block counter/ciphertext spans must be non-empty, equal, and even");
    // walsh_packing_block_count
    const size_t pack = a.packing_block_count, segs = a.packed_segment_count;
    if (pack == 0 || segs < kMinSegments || a.active_blocks > pack || segs > slots / pack)
        throw std::invalid_argument("ckks_aes_walsh: active blocks exceed padded Walsh packing capacity");
    if (a.key_level != p.s2c_depth + 1)
        throw std::invalid_argument("ckks_aes_walsh: complex-block path received a round key bit at the wrong level");
    if (!a.key_b || !a.key_a || !a.key_scales || !a.counters || !a.ciphertexts)
        throw std::invalid_argument("ckks_aes_walsh: null argument");
    DeviceOps ops(c, 1, s);
    Aes aes(c, ops, p, s2c, nplans, c2s, nc2s, coeffs, ncoeffs, s);
    aes.set_per_instance(a.per_instance);
    Bits st = aes.initial_state_fast(a);
    for (size_t round = 1; round <= kRounds; ++round) {
        aes.mask_inactive(st, pack);
        st = aes.sub_bytes(st, pack);
        Aes::shift_rows(st);
        aes.linear_layer(st, a, round, round < kRounds);
    }
    aes.add_public_all(st, a.ciphertexts, a.active_blocks);
    DeviceOps bops(c, Aes::refresh_batches(slots, a.active_blocks), s);
    aes.final_refresh(st, a.active_blocks, bops);
    for (size_t bit = 0; bit < kBlockBits; ++bit) {
        ops.copy_out(st[bit], &out_b[bit], &out_a[bit]);
        out_level[bit] = st[bit].level;
        out_scale[bit] = static_cast<double>(st[bit].scale);
    }
}

void walsh_encrypt_round_key_bits(Context& c, const BootstrapParams& p, const uint8_t* expanded_key,
                                  size_t active_blocks, const int8_t* secret, uint64_t seed, double sigma,
                                  uint64_t* const* out_b, uint64_t* const* out_a, double* out_scale,
                                  size_t* out_level, cudaStream_t s) {
    if (!expanded_key) throw std::invalid_argument("ckks_aes_walsh: null expanded key");
    const size_t slots = c.N / 2;
    if (active_blocks == 0 || active_blocks > slots)
        throw std::invalid_argument("ckks_aes_walsh: invalid active complex block count");
    // aes_walsh_state_entry_level: one selection limb above the S2C input level
    const size_t level = p.s2c_depth + 1;
    if (level >= c.nq) throw std::invalid_argument("ckks_aes_walsh: selection key level exceeds parameter chain");
    DeviceOps ops(c, 1, s);
    // the bit's value in the real and imaginary part of the first active_blocks slots, zero
    // elsewhere; rounds 1..9 at a quarter of the parameter scale, rounds 0 and 10 at it
    const double full = p.scale, quarter = p.scale / 4.0;
    auto encode = [&](double v, double scale) {
        std::vector<double> re(slots, 0.0), im(slots, 0.0);
        for (size_t i = 0; i < active_blocks; ++i) re[i] = im[i] = v;
        std::vector<uint64_t> coeff((level + 1) * c.N);
        host::encode_slots(c.N, re.data(), im.data(), scale, c.q.data(), level + 1, coeff.data());
        return ops.upload_plain(coeff.data(), level + 1);
    };
    const uint64_t* pt[2][2] = {{encode(0.0, full), encode(1.0, full)}, {encode(0.0, quarter), encode(1.0, quarter)}};
    std::vector<const uint64_t*> pts(kKeyBits);
    for (size_t k = 0; k < kKeyBits; ++k) {
        const bool edge = k < kBlockBits || k >= kRounds * kBlockBits;
        const int bit = (expanded_key[k / 8] >> (k % 8)) & 1;
        pts[k] = pt[edge ? 0 : 1][bit];
        out_scale[k] = edge ? full : quarter;
        out_level[k] = level;
    }
    encrypt_symmetric(c, kKeyBits, level, pts.data(), secret, nullptr, nullptr, seed, sigma, out_b, out_a, s);
}

}  // namespace wg
