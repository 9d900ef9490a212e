// The AES linear layers on lazy bits as one fused launch: every output bit ciphertext is an
// integer combination of input bit ciphertexts (small multiplicities) plus an optional scaled
// key-bit ciphertext.  Shared by the Walsh (wg_aes.cu) and XBOOT (wg_xboot.cu) AES circuits;
// included by several translation units, so everything here has internal linkage.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "wg_ctops.cuh"

namespace wg {
namespace {

constexpr int kMaxLinTerms = 8;

// One output limb of the fused linear layer: sum_t cnt[t] * src[t] + kfac * key (mod q).
struct LinearJob {
    uint64_t* out;
    const uint64_t* src[kMaxLinTerms];
    const uint64_t* key;
    uint64_t kfac;
    uint8_t cnt[kMaxLinTerms];
    int n, mod;
};

__global__ void __launch_bounds__(kT) kb_linear(const LinearJob* jobs, int njobs, const Modulus* mods) {
    const LinearJob* j = job_of(jobs, njobs);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const Modulus m = mods[j->mod];
    const uint64_t q = m.q;
    uint64_t acc = 0;
    for (int t = 0; t < j->n; ++t) {
        const uint64_t x = j->src[t][k];
        for (int r = 0; r < j->cnt[t]; ++r) acc = add_mod(acc, x, q);
    }
    if (j->key) acc = add_mod(acc, barrett_mul(j->key[k], j->kfac, m), q);
    j->out[k] = acc;
}

// The reference's MixColumns on lazy bits (clone, add_bits, xtime, fmix_column_byte) replayed on
// symbolic bits: out[o][j] = how many times state bit j enters output bit o.
using SymBit = std::array<uint8_t, 128>;

std::vector<SymBit> mix_symbolic() {
    using SymByte = std::array<SymBit, 8>;
    auto unit = [](size_t j) {
        SymBit b{};
        b[j] = 1;
        return b;
    };
    auto add = [](const SymBit& x, const SymBit& y) {
        SymBit r{};
        for (size_t j = 0; j < 128; ++j) r[j] = (uint8_t)(x[j] + y[j]);
        return r;
    };
    auto byte_of = [&](size_t b) {
        SymByte o;
        for (size_t k = 0; k < 8; ++k) o[k] = unit(b * 8 + k);
        return o;
    };
    auto add_bytes = [&](const SymByte& l, const SymByte& r) {
        SymByte o;
        for (size_t k = 0; k < 8; ++k) o[k] = add(l[k], r[k]);
        return o;
    };
    auto xtime = [&](const SymByte& b) {
        return SymByte{b[7], add(b[0], b[7]), b[1], add(b[2], b[7]), add(b[3], b[7]), b[4], b[5], b[6]};
    };
    auto mix = [&](const SymByte& b0, const SymByte& b1, const SymByte& b2, const SymByte& b3) {
        SymByte d = xtime(add_bytes(b0, b1));
        d = add_bytes(d, b1);
        d = add_bytes(d, b2);
        return add_bytes(d, b3);
    };
    std::vector<SymBit> out(128);
    for (size_t col = 0; col < 4; ++col) {
        const SymByte b0 = byte_of(4 * col), b1 = byte_of(4 * col + 1), b2 = byte_of(4 * col + 2), b3 = byte_of(4 * col + 3);
        const SymByte o[4] = {mix(b0, b1, b2, b3), mix(b1, b2, b3, b0), mix(b2, b3, b0, b1), mix(b3, b0, b1, b2)};
        for (size_t r = 0; r < 4; ++r)
            for (size_t k = 0; k < 8; ++k) out[(4 * col + r) * 8 + k] = o[r][k];
    }
    return out;
}

}  // namespace
}  // namespace wg
