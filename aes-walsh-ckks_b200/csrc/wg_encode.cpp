// CKKS slot encoding on the host (FP64), for the public plaintexts the AES circuit forms on the
// server side: counter and ciphertext bit patterns and active-slot masks.
//
// Reference: encode_slots_custom_basis, src/ckks/encoding/ckks_encoding.cpp:368-414, with the
// Hermitian embedding (:29-43), the FFT twiddles and DIF transform of src/math/fft/fft.cpp:36-97
// and the slot permutation of src/ckks/context/ckks_context.cpp:56-68.  The coefficients are
// llrint(Re(FFT) * scale / N), so the FFT's rounding errors decide the rare coefficients next to
// a rounding boundary.  Every complex product is therefore written out with the rounding the
// reference build (g++ -O3 -mfma) gives it, established against that build value for value:
// the scalar product (re = fma(a, c, -(b d)), im = fma(a, d, b c)) for the twiddle recurrences
// and the butterflies, the vectorised one (re = fma(a, c, -(b d)), im = fma(b, c, a d)) for the
// twist loop.  The file is compiled with -ffp-contract=off so nothing else is fused.
#include <atomic>
#include <bit>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <numbers>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "wg_encode.hpp"

namespace wg {
namespace host {
namespace {

using Cplx = std::complex<double>;

size_t rev_bits(size_t v, size_t width) {
    size_t r = 0;
    for (size_t i = 0; i < width; ++i) {
        r = (r << 1) | (v & 1);
        v >>= 1;
    }
    return r;
}

Cplx unit(double angle) { return {std::cos(angle), std::sin(angle)}; }

// product as the reference's scalar code rounds it
Cplx mul_s(Cplx x, Cplx y) {
    const double a = x.real(), b = x.imag(), c = y.real(), d = y.imag();
    return Cplx(std::fma(a, c, -(b * d)), std::fma(a, d, b * c));
}

// product as the reference's vectorised twist loop rounds it
Cplx mul_v(Cplx x, Cplx y) {
    const double a = x.real(), b = x.imag(), c = y.real(), d = y.imag();
    return Cplx(std::fma(a, c, -(b * d)), std::fma(b, c, a * d));
}

struct FftTables {
    std::vector<Cplx> fwd;      // conjugated inverse twiddles with the psi twist folded in
    std::vector<size_t> perm;   // slot i -> evaluation index
};

FftTables make_tables(size_t N) {
    FftTables t;
    std::vector<Cplx> tw(N);
    tw[0] = {0, 0};
    const Cplx w = unit(2.0 * std::numbers::pi / static_cast<double>(N));
    std::vector<Cplx> pw(N >> 1);
    pw[0] = {1.0, 0.0};
    for (size_t i = 1; i < (N >> 1); ++i) pw[i] = mul_s(pw[i - 1], w);
    for (size_t m = 1; m < N; m <<= 1) {
        const size_t step = N / (m << 1);
        const size_t bits = (size_t)std::countr_zero(m);
        for (size_t i = 0; i < m; ++i) tw[m + i] = pw[rev_bits(i, bits) * step];
    }
    const Cplx psi = unit(std::numbers::pi / static_cast<double>(N));
    std::vector<Cplx> psi_pw(N);
    psi_pw[0] = Cplx(1.0, 0.0);
    for (size_t j = 1; j < N; ++j) psi_pw[j] = mul_s(psi_pw[j - 1], psi);
    for (size_t m = N >> 1, k = 1; m > 0; m >>= 1, k <<= 1) {
        const Cplx pk = psi_pw[k];
        for (size_t i = 0; i < m; ++i) tw[m + i] = mul_v(tw[m + i], pk);
    }
    t.fwd.resize(N);
    for (size_t i = 0; i < N; ++i) t.fwd[i] = std::conj(tw[i]);
    const size_t width = (size_t)std::countr_zero(N);
    t.perm.resize(N >> 1);
    uint64_t cur = 1;
    for (size_t i = 0; i < (N >> 1); ++i) {
        t.perm[i] = rev_bits((cur - 1) >> 1, width);
        cur = (cur * 5) % (2 * N);
    }
    return t;
}

const FftTables& tables(size_t N) {
    static std::mutex mu;
    static std::unordered_map<size_t, FftTables> cache;
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(N);
    if (it == cache.end()) it = cache.emplace(N, make_tables(N)).first;
    return it->second;
}

void fft_dif(std::vector<Cplx>& x, const std::vector<Cplx>& tw, size_t N) {
    const Cplx* __restrict twp = tw.data();
    Cplx* __restrict xp = x.data();
    for (size_t m = N >> 1, k = 1; m > 0; m >>= 1, k <<= 1) {
        for (size_t i = 0; i < m; ++i) {
            const Cplx w = twp[m + i];
            Cplx* __restrict x0 = xp + ((i << 1) * k);
            Cplx* __restrict x1 = x0 + k;
            for (size_t j = 0; j < k; ++j) {
                const Cplx u = x0[j];
                const Cplx v = x1[j];
                x0[j] = Cplx(u.real() + v.real(), u.imag() + v.imag());
                x1[j] = mul_s(Cplx(u.real() - v.real(), u.imag() - v.imag()), w);
            }
        }
    }
}

std::atomic<uint64_t> g_encode_calls{0}, g_encode_ns{0};

}  // namespace

void encode_tables(size_t N, std::vector<double>& twiddles, std::vector<uint32_t>& perm) {
    if (N < 2 || (N & (N - 1))) throw std::invalid_argument("ckks_encode: ring degree must be a power of two");
    const FftTables& t = tables(N);
    twiddles.resize(2 * N);
    for (size_t i = 0; i < N; ++i) {
        twiddles[2 * i] = t.fwd[i].real();
        twiddles[2 * i + 1] = t.fwd[i].imag();
    }
    perm.assign(t.perm.begin(), t.perm.end());
}

void encode_stats(uint64_t* calls, uint64_t* ns) {
    *calls = g_encode_calls.load();
    *ns = g_encode_ns.load();
}

void encode_slots(size_t N, const double* re, const double* im, double scale, const uint64_t* moduli, size_t limbs,
                  uint64_t* out) {
    if (!(scale > 0.0)) throw std::invalid_argument("ckks_encode: scale must be positive");
    if (N < 2 || (N & (N - 1))) throw std::invalid_argument("ckks_encode: ring degree must be a power of two");
    const auto t0 = std::chrono::steady_clock::now();
    const FftTables& t = tables(N);
    const size_t half = N >> 1;
    std::vector<Cplx> ev(N);
    for (size_t i = 0; i < half; ++i) {
        const Cplx v(re[i], im[i]);
        const size_t d = t.perm[i];
        ev[d] = v;
        ev[N - 1 - d] = std::conj(v);
    }
    fft_dif(ev, t.fwd, N);
    const double s = scale / static_cast<double>(N);
    for (size_t l = 0; l < limbs; ++l) {
        const int64_t q = static_cast<int64_t>(moduli[l]);
        uint64_t* o = out + l * N;
        for (size_t i = 0; i < N; ++i) {
            const int64_t v = std::llrint(ev[i].real() * s);
            const int64_t r = v % q;
            o[i] = static_cast<uint64_t>(r + (q & (r >> 63)));
        }
    }
    g_encode_calls.fetch_add(1, std::memory_order_relaxed);
    g_encode_ns.fetch_add((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count(),
                          std::memory_order_relaxed);
}

}  // namespace host
}  // namespace wg
