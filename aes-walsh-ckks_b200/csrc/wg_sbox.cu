// The AES S-box on lazy bits through its Walsh expansion, mask-packed, batched over S-box
// instances (each instance: 8 bit ciphertexts of one byte position).
//
// Reference: ckks_walsh_sbox_complex_blocks_mask_packed and its helpers,
// src/ckks/operations/circuits/ckks_walsh_sbox.cpp:130-1323.  Per instance:
//   1. the 30 nibble parities (sum of the bits a mask selects, low and high nibble) are packed
//      into one ciphertext, segment k rotated by k * block_count;
//   2. one EvalMod bootstrap of the packed ciphertext gives two lanes (real and imaginary
//      blocks), each turned from parities into signs (1 - 2 x);
//   3. each lane is unpacked into 15 + 15 sign ciphertexts by hoisted rotations, plus the
//      constant 1 for the empty mask;
//   4. per output-bit pair, the Walsh sum sum_{l,h} D[l][h] s_l s_h (D = Walsh coefficients
//      / 4, small integers) is formed as 15 products of a low-nibble linear combination with a
//      high-nibble sign, summed raw, relinearised once, rescaled, normalised to
//      (1/2 + i/2) - D/128, then split into real and imaginary bits by conjugation.
// Residues depend on the order of every addition and product and on each rounded constant, so
// the host side takes the reference's steps in the same order with the same long-double scale
// bookkeeping; the device side is the batched operation set of wg_ctops.cuh plus the hoisted
// rotations and the bootstrap of this library.
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <optional>
#include <stdexcept>
#include <vector>

#include "wg_ctops.cuh"
#include "wg_walsh.cuh"

namespace wg {
namespace {

constexpr size_t kBits = 8;
constexpr size_t kNibble = 16;
constexpr size_t kSegments = 2 * (kNibble - 1);
constexpr size_t kMaxAbsCoeff = 8;

// ---- AES S-box (FIPS-197 5.1.1): inverse in GF(2^8) mod x^8 + x^4 + x^3 + x + 1, then the
// affine map b ^ rotl(b,1) ^ rotl(b,2) ^ rotl(b,3) ^ rotl(b,4) ^ 0x63.
uint8_t gf_mul(uint8_t a, uint8_t b) {
    uint8_t r = 0;
    while (b) {
        if (b & 1) r ^= a;
        const bool hi = a & 0x80;
        a = (uint8_t)(a << 1);
        if (hi) a ^= 0x1b;
        b >>= 1;
    }
    return r;
}

std::array<uint8_t, 256> aes_sbox() {
    std::array<uint8_t, 256> s{};
    for (int x = 0; x < 256; ++x) {
        uint8_t inv = 0;
        if (x) {  // x^254
            uint8_t p = (uint8_t)x, r = 1;
            for (int e = 254; e; e >>= 1) {
                if (e & 1) r = gf_mul(r, p);
                p = gf_mul(p, p);
            }
            inv = r;
        }
        auto rotl = [](uint8_t v, int k) { return (uint8_t)((v << k) | (v >> (8 - k))); };
        s[x] = (uint8_t)(inv ^ rotl(inv, 1) ^ rotl(inv, 2) ^ rotl(inv, 3) ^ rotl(inv, 4) ^ 0x63);
    }
    return s;
}

using WalshTable = std::array<std::array<std::array<int16_t, kNibble>, kNibble>, kBits>;

// D[out][low][high] = (sum_x (-1)^(S(x)_out xor parity(mask & x))) / 4, mask = low | high << 4
const WalshTable& walsh_table() {
    static const WalshTable t = [] {
        const auto sb = aes_sbox();
        WalshTable w{};
        for (size_t ob = 0; ob < kBits; ++ob)
            for (size_t lm = 0; lm < kNibble; ++lm)
                for (size_t hm = 0; hm < kNibble; ++hm) {
                    const unsigned mask = (unsigned)(lm | (hm << 4));
                    int acc = 0;
                    for (unsigned x = 0; x < 256; ++x) {
                        const unsigned bit = (sb[x] >> ob) & 1u;
                        const unsigned dot = __builtin_parity(mask & x);
                        acc += (bit ^ dot) == 0 ? 1 : -1;
                    }
                    if (acc % 4) throw std::runtime_error("ckks_walsh_sbox: AES Walsh coefficient is not divisible by four");
                    w[ob][lm][hm] = (int16_t)(acc / 4);
                }
        return w;
    }();
    return t;
}

bool close_ld(long double l, long double r, long double tol = 0x1p-45L) {
    if (!std::isfinite(l) || !std::isfinite(r)) return false;
    const long double m = std::max<long double>({1.0L, std::abs(l), std::abs(r)});
    return std::abs(l - r) <= tol * m;
}

constexpr int kMaxLinLimbs = 16;

struct SumJob {
    uint64_t* out;
    const uint64_t* src[kSegments];
    int n, mod;
};

// out = sum of n residues (mod q): exact, so independent of the order the reference adds in
__global__ void __launch_bounds__(kT) kb_sum(const SumJob* jobs, int njobs, const Modulus* mods) {
    const SumJob* j = job_of(jobs, njobs);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q = mods[j->mod].q;
    uint64_t acc = j->src[0][k];
    for (int t = 1; t < j->n; ++t) acc = add_mod(acc, j->src[t][k], q);
    j->out[k] = acc;
}

// Coefficients of one paired linear combination real + i imag over the 15 nonzero nibble masks.
struct LinCoefs {
    int8_t cr[kNibble], ci[kNibble];
    uint64_t c0r[kMaxLinLimbs], c0i[kMaxLinLimbs];  // integer constants (b polynomial), per limb
};

// One limb of one instance for the fused Walsh products (masks 1..15 at their own index).
struct WalshJob {
    const uint64_t* low[2][kNibble];    // [b|a][mask]
    const uint64_t* high[2][kNibble];
    const uint64_t* pt_i;
    uint64_t* out[5];                   // acc b, acc a, raw b, raw a, raw c2
    int limb, pad;
};

__global__ void __launch_bounds__(kT, 2) kb_walsh_products(const WalshJob* jobs, int n, const WalshCoefs* cf,
                                                           const Modulus* mods) {
    const WalshJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const Modulus m = mods[j->limb];
    const uint64_t pt_i = j->pt_i[k];
    uint64_t lb[kNibble], la[kNibble];
    lb[0] = la[0] = 0;
#pragma unroll
    for (int t = 1; t < (int)kNibble; ++t) {
        lb[t] = j->low[0][t][k];
        la[t] = j->low[1][t][k];
    }
    WalshLow w;
    walsh_load_low(lb, la, w);
    uint64_t acc_b, acc_a;
    walsh_constant_pair(w, *cf, j->limb, pt_i, m, &acc_b, &acc_a);
    j->out[0][k] = acc_b;
    j->out[1][k] = acc_a;
    uint64_t rb = 0, ra = 0, rc = 0;
#pragma unroll 1
    for (int hm = 1; hm < (int)kNibble; ++hm)
        walsh_product(w, *cf, hm, j->limb, pt_i, m, j->high[0][hm][k], j->high[1][hm][k], &rb, &ra, &rc);
    j->out[2][k] = rb;
    j->out[3][k] = ra;
    j->out[4][k] = rc;
}

struct LinJob {
    uint64_t* out;
    const uint64_t* terms[kNibble - 1];  // sign ciphertext of mask m at terms[m - 1]
    const uint64_t* pt_i;                // evaluation form of the slot constant i, this limb
    int limb, poly;
};

// out = (c0r + sum_m cr[m] s_m) + pt_i * (c0i + sum_m ci[m] s_m) (mod q), one limb of one
// polynomial.  Exact modular sums, so equal to the reference's sequence of additions of
// precomputed multiples; pt_i times x by a Barrett product of canonical residues.
__global__ void __launch_bounds__(kT) kb_lin_pair(const LinJob* jobs, int n, LinCoefs cf, const Modulus* mods) {
    const LinJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const Modulus m = mods[j->limb];
    const uint64_t q = m.q;
    uint64_t r = j->poly == 0 ? cf.c0r[j->limb] : 0, im = j->poly == 0 ? cf.c0i[j->limb] : 0;
#pragma unroll
    for (int t = 1; t < (int)kNibble; ++t) {
        const int a = cf.cr[t], b = cf.ci[t];
        if (a == 0 && b == 0) continue;
        const uint64_t x = j->terms[t - 1][k];
        if (a) r = add_mod(r, barrett_mul(x, a > 0 ? (uint64_t)a : q - (uint64_t)(-a), m), q);
        if (b) im = add_mod(im, barrett_mul(x, b > 0 ? (uint64_t)b : q - (uint64_t)(-b), m), q);
    }
    j->out[k] = add_mod(r, barrett_mul(im, j->pt_i[k], m), q);
}

class Sbox {
public:
    Sbox(Context& c, DeviceOps& ops, cudaStream_t s) : c_(c), ops_(ops), s_(s), table_(walsh_table()) {}

    // rounded_scaled_integer_mod_q on every limb, added to b (ckks_add_integer_constant_inplace)
    void add_int(CtBatch& x, int64_t k) {
        if (k == 0) return;
        std::vector<uint64_t> v(x.level + 1);
        for (size_t l = 0; l <= x.level; ++l) {
            const long double scaled = static_cast<long double>(k) * x.scale;
            if (!std::isfinite(scaled)) throw std::invalid_argument("ckks_add_integer_constant_inplace: non-finite scaled constant");
            long double r = std::fmod(std::round(scaled), static_cast<long double>(c_.q[l]));
            if (r < 0.0L) r += static_cast<long double>(c_.q[l]);
            uint64_t u = static_cast<uint64_t>(r);
            if (u >= c_.q[l]) u %= c_.q[l];
            v[l] = u;
        }
        ops_.scalar(x, nullptr, v, kScalarAdd);
    }

    // ckks_rotate_inplace by r on every ciphertext of the batch
    void rotate(CtBatch& x, int64_t r) {
        const int64_t slots = (int64_t)(c_.N / 2);
        int64_t n = r % slots;
        if (n < 0) n += slots;
        if (n == 0) return;
        const KeyEntry& k = c_.key(WG_KEY_ROTATION, n);
        std::vector<KsItem> items(ops_.count());
        for (size_t i = 0; i < ops_.count(); ++i) {
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
        batch_keyswitch(c_, items.data(), items.size(), s_);
    }

    // 1. build_mask_packed_parity_input: the 30 nibble parities (one launch), their segment
    // rotations (one batched key switch), and their sum (one launch)
    CtBatch pack(const std::vector<CtBatch>& in, size_t bc) {
        WG_SPAN("sbox.pack");
        const size_t N = c_.N, level = in[0].level, L = level + 1, cnt = ops_.count();
        std::vector<CtBatch> terms(kSegments);
        std::vector<SumJob> par;
        for (size_t mask = 1; mask < kNibble; ++mask)
            for (int high = 0; high < 2; ++high) {
                const size_t seg = (high ? kNibble - 1 : 0) + (mask - 1);
                CtBatch t = ops_.alloc(level, 2);
                t.scale = in[0].scale;
                for (size_t i = 0; i < cnt; ++i)
                    for (int poly = 0; poly < 2; ++poly)
                        for (size_t l = 0; l < L; ++l) {
                            SumJob jb{};
                            jb.out = t.p[i][poly] + l * N;
                            for (size_t bit = 0; bit < 4; ++bit)
                                if ((mask >> bit) & 1) jb.src[jb.n++] = in[(high ? 4 : 0) + bit].p[i][poly] + l * N;
                            jb.mod = (int)l;
                            par.push_back(jb);
                        }
                terms[seg] = t;
            }
        run_sums(par);
        std::vector<KsItem> items;
        for (size_t seg = 1; seg < kSegments; ++seg) {
            const int64_t slots = (int64_t)(N / 2);
            int64_t r = (int64_t)(seg * bc) % slots;
            if (r == 0) continue;
            const KeyEntry& k = c_.key(WG_KEY_ROTATION, r);
            for (size_t i = 0; i < cnt; ++i) {
                KsItem it;
                it.level = level;
                it.key_term = terms[seg].p[i][1];
                it.key = &k;
                it.b_in = terms[seg].p[i][0];
                it.a_in = terms[seg].p[i][1];
                it.b = terms[seg].p[i][0];
                it.a = terms[seg].p[i][1];
                it.b_add = 1;
                it.a_add = 0;
                it.galois = host::powmod(5, (uint64_t)r, 2 * N);
                items.push_back(it);
            }
        }
        batch_keyswitch(c_, items.data(), items.size(), s_);
        CtBatch packed = ops_.alloc(level, 2);
        packed.scale = in[0].scale;
        std::vector<SumJob> tot;
        for (size_t i = 0; i < cnt; ++i)
            for (int poly = 0; poly < 2; ++poly)
                for (size_t l = 0; l < L; ++l) {
                    SumJob jb{};
                    jb.out = packed.p[i][poly] + l * N;
                    for (size_t seg = 0; seg < kSegments; ++seg) jb.src[jb.n++] = terms[seg].p[i][poly] + l * N;
                    jb.mod = (int)l;
                    tot.push_back(jb);
                }
        run_sums(tot);
        return packed;
    }

    void run_sums(const std::vector<SumJob>& jobs) {
        if (jobs.empty()) return;
        JobTable t;
        const SumJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsWalsh, 8.0 * c_.N * jobs.size() * 5.0, s_);
        kb_sum<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), c_.d_mod);
        check_cuda(cudaGetLastError(), "walsh parity sums");
    }

    // 2. parities -> signs: x <- -2 x + 1
    void to_sign(CtBatch& x) {
        WG_SPAN("sbox.to_sign");
        ops_.mul_int(x, -2);
        add_int(x, 1);
    }

    // 3. unpack_mask_packed_signs: low[0] = high[0] = constant 1, low[m] / high[m] rotated back
    void unpack(const CtBatch& lane, size_t bc, std::vector<CtBatch>& low, std::vector<CtBatch>& high) {
        WG_SPAN("sbox.unpack");
        const size_t N = c_.N, L = lane.level + 1;
        low.assign(kNibble, CtBatch{});
        high.assign(kNibble, CtBatch{});
        for (auto* v : {&low, &high}) {
            CtBatch one = ops_.zeros(lane.level, lane.scale);
            add_int(one, 1);
            (*v)[0] = one;
        }
        std::vector<int64_t> rots;
        for (size_t mask = 1; mask < kNibble; ++mask) {
            rots.push_back(-(int64_t)((mask - 1) * bc));
            rots.push_back(-(int64_t)((kNibble - 1 + mask - 1) * bc));
        }
        for (size_t mask = 1; mask < kNibble; ++mask) {
            low[mask] = lane;
            high[mask] = lane;
        }
        std::vector<const uint64_t*> lb(ops_.count()), la(ops_.count());
        std::vector<uint64_t*> outs(ops_.count());
        for (size_t i = 0; i < ops_.count(); ++i) {
            lb[i] = lane.p[i][0];
            la[i] = lane.p[i][1];
            outs[i] = ops_.raw(rots.size() * 2 * L);
        }
        rotate_many_batch(c_, lane.level, ops_.count(), lb.data(), la.data(), rots.data(), rots.size(), outs.data(), s_);
        for (size_t i = 0; i < ops_.count(); ++i) {
            uint64_t* out = outs[i];
            for (size_t mask = 1; mask < kNibble; ++mask) {
                const size_t kl = 2 * (mask - 1), kh = kl + 1;
                low[mask].p[i] = {out + (2 * kl) * L * N, out + (2 * kl + 1) * L * N, nullptr};
                high[mask].p[i] = {out + (2 * kh) * L * N, out + (2 * kh + 1) * L * N, nullptr};
            }
        }
        for (size_t mask = 1; mask < kNibble; ++mask) {
            low[mask].cap = high[mask].cap = L;
            low[mask].np = high[mask].np = 2;
        }
    }

    // 4. recombine_mask_packed_signs_to_paired_outputs
    std::vector<CtBatch> recombine(const std::vector<CtBatch>& low, const std::vector<CtBatch>& high) {
        WG_SPAN("sbox.recombine");
        if (low[1].level == 0) throw std::runtime_error("ckks_walsh_sbox: sign output level is too low for 4+4 products");
        for (size_t m = 1; m < kNibble; ++m)
            if (low[m].level != low[0].level || !close_ld(low[m].scale, low[0].scale))
                throw std::invalid_argument("ckks_walsh_sbox: same-metadata addition mismatch");
        std::vector<CtBatch> out;
        for (size_t pair = 0; pair < kBits / 2; ++pair) {
            CtBatch ws = walsh_sum(low, high, pair, pair + kBits / 2);
            out.push_back(to_bit_pair(ws));
        }
        return out;
    }

    // 5. combine_paired_lane_outputs_as_complex_bits
    std::vector<CtBatch> combine_lanes(const std::vector<CtBatch>& lane0, const std::vector<CtBatch>& lane1) {
        WG_SPAN("sbox.combine_lanes");
        std::vector<CtBatch> bits(kBits);
        for (size_t pair = 0; pair < kBits / 2; ++pair) {
            auto [rl, rh] = split(lane0[pair]);
            auto [il, ih] = split(lane1[pair]);
            bits[pair] = combine_ri(rl, il);
            bits[pair + kBits / 2] = combine_ri(rh, ih);
        }
        return bits;
    }

private:
    CtBatch parity(const std::vector<CtBatch>& in, size_t offset, size_t mask) {
        std::optional<CtBatch> out;
        for (size_t bit = 0; bit < 4; ++bit) {
            if (!((mask >> bit) & 1)) continue;
            if (!out)
                out = ops_.clone(in[offset + bit]);
            else
                ops_.add(*out, in[offset + bit], false);
        }
        return *out;
    }

    // linear_combination_pair_with_constant: (c0 + sum_m c_m s_m) for the real and imaginary
    // coefficient sets, combined as real + i imag (combine_real_imag), in one launch.  The
    // reference adds precomputed multiples |c| s_m one by one; the modular sum is the same.
    CtBatch lin_pair(const std::vector<CtBatch>& signs, const std::array<int16_t, kNibble>& rc,
                     const std::array<int16_t, kNibble>& ic) {
        const size_t N = c_.N, level = signs[0].level, L = level + 1;
        if (L > (size_t)kMaxLinLimbs) throw std::invalid_argument("ckks_walsh_sbox: too many limbs");
        LinCoefs cf{};
        for (size_t m = 0; m < kNibble; ++m) {
            if (rc[m] < -(int)kMaxAbsCoeff || rc[m] > (int)kMaxAbsCoeff || ic[m] < -(int)kMaxAbsCoeff ||
                ic[m] > (int)kMaxAbsCoeff)
                throw std::runtime_error("ckks_walsh_sbox: missing low-sign multiple");
            cf.cr[m] = (int8_t)rc[m];
            cf.ci[m] = (int8_t)ic[m];
        }
        const long double scale = signs[0].scale;
        for (size_t l = 0; l < L; ++l) {
            cf.c0r[l] = int_const(rc[0], scale, c_.q[l]);
            cf.c0i[l] = int_const(ic[0], scale, c_.q[l]);
        }
        const uint64_t* pti = ops_.constant_plaintext(L, 0.0, 1.0, 1.0);
        CtBatch out = ops_.alloc(level, 2);
        out.scale = scale;
        std::vector<LinJob> jobs;
        for (size_t i = 0; i < ops_.count(); ++i)
            for (int poly = 0; poly < 2; ++poly)
                for (size_t l = 0; l < L; ++l) {
                    LinJob jb{};
                    jb.out = out.p[i][poly] + l * N;
                    for (size_t m = 1; m < kNibble; ++m) jb.terms[m - 1] = signs[m].p[i][poly] + l * N;
                    jb.pt_i = pti + l * N;
                    jb.limb = (int)l;
                    jb.poly = poly;
                    jobs.push_back(jb);
                }
        JobTable t;
        const LinJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsWalsh, 8.0 * N * jobs.size() * 17.0, s_);
        kb_lin_pair<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), cf, c_.d_mod);
        check_cuda(cudaGetLastError(), "walsh linear combination");
        return out;
    }

    // rounded_scaled_integer_mod_q
    static uint64_t int_const(int64_t k, long double scale, uint64_t q) {
        if (k == 0) return 0;
        const long double scaled = static_cast<long double>(k) * scale;
        if (!std::isfinite(scaled)) throw std::invalid_argument("ckks_add_integer_constant_inplace: non-finite scaled constant");
        long double r = std::fmod(std::round(scaled), static_cast<long double>(q));
        if (r < 0.0L) r += static_cast<long double>(q);
        uint64_t u = static_cast<uint64_t>(r);
        if (u >= q) u %= q;
        return u;
    }

    bool same_storage(const CtBatch& x, const CtBatch& y) const {
        return x.level == y.level && x.np == y.np && close_ld(x.scale, y.scale);
    }

    // combine_real_imag: real + i imag (imag multiplied by the encoded i, scale kept)
    CtBatch combine_ri(CtBatch real, CtBatch imag) {
        ops_.mul_complex_constant(imag, 0.0, 1.0, 1.0);
        if (same_storage(real, imag)) {
            ops_.add(real, imag, false);
        } else {
            add_term(real, imag);
        }
        return real;
    }

    // multiply_by_integer_scalar_inplace (the S-box's own: int64 multiply, then scale)
    void mul_integer(CtBatch& x, long double scalar, long double out_scale) {
        if (!std::isfinite(scalar) || scalar < 0.0L) throw std::invalid_argument("ckks_walsh_sbox: invalid scalar scale-up");
        const long double r = std::round(scalar);
        if (r < 1.0L || std::abs(scalar - r) > std::max<long double>(1.0L, std::abs(scalar)) * 0x1p-20L)
            throw std::invalid_argument("ckks_walsh_sbox: non-integral scalar scale-up");
        if (r > static_cast<long double>(std::numeric_limits<int64_t>::max()))
            throw std::invalid_argument("ckks_walsh_sbox: scalar scale-up is too large");
        const int64_t k = static_cast<int64_t>(r);
        if (k != 1) ops_.mul_int(x, k);
        x.scale = out_scale;
    }

    void align_exact(CtBatch& x, size_t level, long double scale, int np) {
        if (level > x.level) throw std::invalid_argument("ckks_drop_to_level_inplace: cannot raise ciphertext level");
        x.level = level;
        ops_.pad(x, np);
        if (close_ld(x.scale, scale)) {
            x.scale = scale;
            return;
        }
        // (the reference also accepts an all-zero ciphertext here; zero times any integer is
        // zero, so the residues agree either way)
        if (x.scale > scale) throw std::invalid_argument("ckks_walsh_sbox: cannot scale down ciphertext for addition");
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

    CtBatch mul_raw(CtBatch lhs, const CtBatch& rhs, long double target) {
        if (lhs.level == 0 || rhs.level == 0) throw std::invalid_argument("ckks_walsh_sbox: insufficient level for 4+4 Walsh product");
        const size_t level = std::min(lhs.level, rhs.level);
        lhs.level = level;
        lhs.scale = target;
        if (rhs.level == level && close_ld(rhs.scale, target)) {
            const long double prod = lhs.scale * rhs.scale;
            ops_.tensor(lhs, rhs);
            lhs.scale = prod;
            return lhs;
        }
        CtBatch r = ops_.clone(rhs);
        r.level = level;
        r.scale = target;
        const long double prod = lhs.scale * r.scale;
        ops_.tensor(lhs, r);
        lhs.scale = prod;
        return lhs;
    }

    // The constant-term combination and the 15 unrelinearised products of one output pair in
    // one launch (the high signs share level and scale with the low ones, so the reference's
    // mul_raw multiplies without re-aligning and every step is an exact modular operation).
    std::pair<CtBatch, CtBatch> walsh_fused(const std::vector<CtBatch>& low, const std::vector<CtBatch>& high, size_t rb,
                                            size_t ib, long double target) {
        const size_t N = c_.N, level = low[0].level, L = level + 1, cnt = ops_.count();
        if (L > (size_t)kWalshLimbs) throw std::invalid_argument("ckks_walsh_sbox: too many limbs");
        std::vector<WalshCoefs> cf(1);
        std::memset(cf.data(), 0, sizeof(WalshCoefs));
        const long double scale = low[0].scale;
        for (size_t hm = 0; hm < kNibble; ++hm) {
            for (size_t lm = 0; lm < kNibble; ++lm) {
                const int rcm = table_[rb][lm][hm], icm = table_[ib][lm][hm];
                if (lm > 0 && (rcm < -(int)kMaxAbsCoeff || rcm > (int)kMaxAbsCoeff || icm < -(int)kMaxAbsCoeff ||
                               icm > (int)kMaxAbsCoeff))
                    throw std::runtime_error("ckks_walsh_sbox: missing low-sign multiple");
                reinterpret_cast<uint8_t*>(cf[0].cw[0][hm])[lm] = (uint8_t)((lm ? rcm : 0) + kWalshBias);
                reinterpret_cast<uint8_t*>(cf[0].cw[1][hm])[lm] = (uint8_t)((lm ? icm : 0) + kWalshBias);
            }
            for (size_t l = 0; l < L; ++l) {
                cf[0].c0[0][hm][l] = int_const(table_[rb][0][hm], scale, c_.q[l]);
                cf[0].c0[1][hm][l] = int_const(table_[ib][0][hm], scale, c_.q[l]);
            }
        }
        const uint64_t* pti = ops_.constant_plaintext(L, 0.0, 1.0, 1.0);
        CtBatch acc = ops_.alloc(level, 2);
        acc.scale = scale;
        CtBatch raw = ops_.alloc(level, 3);
        raw.scale = target * high[1].scale;
        std::vector<WalshJob> jobs;
        for (size_t i = 0; i < cnt; ++i)
            for (size_t l = 0; l < L; ++l) {
                WalshJob jb{};
                for (size_t m = 1; m < kNibble; ++m)
                    for (int poly = 0; poly < 2; ++poly) {
                        jb.low[poly][m] = low[m].p[i][poly] + l * N;
                        jb.high[poly][m] = high[m].p[i][poly] + l * N;
                    }
                jb.pt_i = pti + l * N;
                jb.out[0] = acc.p[i][0] + l * N;
                jb.out[1] = acc.p[i][1] + l * N;
                for (int poly = 0; poly < 3; ++poly) jb.out[2 + poly] = raw.p[i][poly] + l * N;
                jb.limb = (int)l;
                jobs.push_back(jb);
            }
        JobTable t;
        const WalshCoefs* cfd = t.add(cf);
        const WalshJob* j = t.add(jobs);
        t.upload(c_, s_);
        Probe probe(kClsWalsh, 8.0 * N * jobs.size() * 66.0, s_);
        kb_walsh_products<<<grid_for(c_, jobs.size()), kT, 0, s_>>>(t.at(j), (int)jobs.size(), t.at(cfd), c_.d_mod);
        check_cuda(cudaGetLastError(), "walsh products");
        return {acc, raw};
    }

    // walsh_sum_for_output_pair
    CtBatch walsh_sum(const std::vector<CtBatch>& low, const std::vector<CtBatch>& high, size_t rb, size_t ib) {
        WG_SPAN("sbox.walsh_sum");
        const long double target = low[0].scale;
        std::array<int16_t, kNibble> rc{}, ic{};
        for (size_t lm = 0; lm < kNibble; ++lm) {
            rc[lm] = table_[rb][lm][0];
            ic[lm] = table_[ib][lm][0];
        }
        // the constant term and the 15 raw products in one pass when the signs share level and
        // scale (the reference's mul_raw then multiplies without re-aligning)
        bool uniform = true;
        for (size_t m = 1; m < kNibble; ++m)
            uniform = uniform && high[m].level == low[0].level && close_ld(high[m].scale, target) &&
                      high[m].level > 0 && low[0].level > 0 && low[m].level == low[0].level &&
                      close_ld(low[m].scale, target) && low[m].np == 2 && high[m].np == 2;
        if (uniform) {
            auto [acc, raw] = walsh_fused(low, high, rb, ib, target);
            ops_.relin(raw);
            add_term(acc, raw);
            return acc;
        }
        CtBatch acc = lin_pair(low, rc, ic);
        std::optional<CtBatch> raw;
        for (size_t hm = 1; hm < kNibble; ++hm) {
            for (size_t lm = 0; lm < kNibble; ++lm) {
                rc[lm] = table_[rb][lm][hm];
                ic[lm] = table_[ib][lm][hm];
            }
            CtBatch ls = lin_pair(low, rc, ic);
            CtBatch prod = mul_raw(ls, high[hm], target);
            if (!raw)
                raw = prod;
            else
                add_term(*raw, prod);
        }
        if (raw) {
            if (raw->np != 3) throw std::invalid_argument("ckks_walsh_sbox: expected raw product before relin");
            ops_.relin(*raw);
            add_term(acc, *raw);
        }
        return acc;
    }

    // walsh_sum_to_bit_pair: (1/2 + i/2) - D/128 after one rescale
    CtBatch to_bit_pair(CtBatch ws) {
        if (ws.level == 0) throw std::invalid_argument("ckks_walsh_sbox: Walsh sum must have one level for final normalization");
        ops_.rescale(ws);
        const long double out_scale = ws.scale * 128.0L;
        ws.scale = out_scale;
        ops_.mul_int(ws, -1);
        ops_.add_complex_constant(ws, 0.5, 0.5, static_cast<double>(out_scale));
        return ws;
    }

    // split_real_imag_pair: (pair + conj, -i (pair - conj)), both at twice the scale
    std::pair<CtBatch, CtBatch> split(const CtBatch& pair) {
        CtBatch conj = ops_.conjugate(pair);
        CtBatch real = ops_.clone(pair);
        ops_.add(real, conj, false);
        real.scale = pair.scale * 2.0L;
        CtBatch imag = ops_.clone(pair);
        ops_.add(imag, conj, true);
        ops_.mul_complex_constant(imag, 0.0, -1.0, 1.0);
        imag.scale = pair.scale * 2.0L;
        return {real, imag};
    }

    Context& c_;
    DeviceOps& ops_;
    cudaStream_t s_;
    const WalshTable& table_;
};

}  // namespace

std::array<uint8_t, 256> aes_sbox_table() { return aes_sbox(); }

void walsh_sbox(Context& c, const BootstrapParams& p, const S2cPlan* s2c, size_t nplans, const LtStage* const* c2s,
                size_t nc2s, const double* coeffs, size_t ncoeffs, size_t block_count, size_t count, size_t level,
                double scale, uint64_t* const* in_b, uint64_t* const* in_a, uint64_t* const* out_b,
                uint64_t* const* out_a, size_t* out_level, double* out_scale, cudaStream_t s) {
    if (count == 0) return;
    if (block_count == 0 || block_count * kSegments > c.N / 2)
        throw std::invalid_argument("ckks_walsh_sbox: mask-packed block count exceeds slot capacity");
    if (level != p.s2c_depth) throw std::invalid_argument("ckks_walsh_sbox: input level must equal bootstrap S2C entry depth");
    for (size_t seg = 1; seg < kSegments; ++seg)
        for (int sign : {1, -1}) {
            int64_t r = sign * (int64_t)(seg * block_count) % (int64_t)(c.N / 2);
            if (r < 0) r += (int64_t)(c.N / 2);
            if (r && !c.keys.count({WG_KEY_ROTATION, r}))
                throw std::invalid_argument("ckks_walsh_sbox: missing mask-packed segment rotation key");
        }
    DeviceOps ops(c, count, s);
    Sbox sb(c, ops, s);
    std::vector<CtBatch> in(kBits);
    for (size_t k = 0; k < kBits; ++k) in[k] = ops.wrap(in_b + k * count, in_a + k * count, level, scale);
    CtBatch packed = sb.pack(in, block_count);
    // bootstrap: the packed ciphertexts in buffers with room for depth+1 limbs
    const size_t full = p.depth + 1;
    std::vector<uint64_t*> pb(count), pa(count), o0b(count), o0a(count), o1b(count), o1a(count);
    for (size_t i = 0; i < count; ++i) {
        pb[i] = ops.raw(full);
        pa[i] = ops.raw(full);
        for (auto* v : {&o0b, &o0a, &o1b, &o1a}) (*v)[i] = ops.raw(full);
        check_cuda(cudaMemcpyAsync(pb[i], packed.p[i][0], (level + 1) * c.N * 8, cudaMemcpyDeviceToDevice, s), "pack");
        check_cuda(cudaMemcpyAsync(pa[i], packed.p[i][1], (level + 1) * c.N * 8, cudaMemcpyDeviceToDevice, s), "pack");
    }
    size_t blv = 0;
    double bsc = 0.0;
    bootstrap_evalmod(c, p, s2c, nplans, c2s, nc2s, coeffs, ncoeffs, count, static_cast<double>(packed.scale),
                      pb.data(), pa.data(), o0b.data(), o0a.data(), o1b.data(), o1a.data(), &blv, &bsc, s);
    CtBatch lane0 = ops.wrap(o0b.data(), o0a.data(), blv, bsc);
    CtBatch lane1 = ops.wrap(o1b.data(), o1a.data(), blv, bsc);
    lane0.cap = lane1.cap = full;
    sb.to_sign(lane0);
    sb.to_sign(lane1);
    std::vector<CtBatch> l0low, l0high, l1low, l1high;
    sb.unpack(lane0, block_count, l0low, l0high);
    sb.unpack(lane1, block_count, l1low, l1high);
    std::vector<CtBatch> pairs0 = sb.recombine(l0low, l0high);
    std::vector<CtBatch> pairs1 = sb.recombine(l1low, l1high);
    std::vector<CtBatch> bits = sb.combine_lanes(pairs0, pairs1);
    for (size_t k = 0; k < kBits; ++k) {
        ops.copy_out(bits[k], out_b + k * count, out_a + k * count);
        out_level[k] = bits[k].level;
        out_scale[k] = static_cast<double>(bits[k].scale);
    }
}

}  // namespace wg
