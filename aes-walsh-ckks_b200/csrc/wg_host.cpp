// Host-side parameter and table generation for the device library.
//
// These routines restate the reference's context-build arithmetic so the device tables are
// identical to the ones the reference computes:
//   prime chain          src/util/random.cpp:74-131
//   NTT twiddles         src/math/ntt/ntt.cpp:28-148
//   Barrett / Shoup      src/math/modarith/modarith.cpp:3-13
#include <algorithm>

#include "wg_internal.hpp"

namespace wg::host {

using u128 = unsigned __int128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)(((u128)a * b) % m); }

uint64_t powmod(uint64_t a, uint64_t e, uint64_t m) {
    a %= m;
    uint64_t r = 1;
    for (; e; e >>= 1) {
        if (e & 1) r = mulmod(r, a, m);
        a = mulmod(a, a, m);
    }
    return r;
}

// Extended Euclid with the same sign handling as the reference's mod_inverse.
uint64_t inverse(uint64_t a, uint64_t m) {
    if (m == 1) return 0;
    int64_t x_prev = 0, x = 1;
    uint64_t mm = m;
    const int64_t m0 = (int64_t)m;
    while (a > 1) {
        const int64_t quot = (int64_t)(a / mm);
        const uint64_t rem = a % mm;
        a = mm;
        mm = rem;
        const int64_t nx = x - quot * x_prev;
        x = x_prev;
        x_prev = nx;
    }
    if (x < 0) x += m0;
    return (uint64_t)x;
}

uint64_t shoup(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

void barrett_const(uint64_t q, uint64_t& lo, uint64_t& hi) {
    const u128 r = (~(u128)0) / q;
    lo = (uint64_t)r;
    hi = (uint64_t)(r >> 64);
}

// Same estimate-and-one-correction Barrett product the reference uses (the precomputed
// base-change tables inherit its representation).
uint64_t barrett_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t lo, uint64_t hi) {
    const u128 z = (u128)a * b;
    const uint64_t zl = (uint64_t)z, zh = (uint64_t)(z >> 64);
    const u128 t = (u128)zh * lo + (((u128)zl * lo) >> 64);
    const uint64_t carry = (uint64_t)(t >> 64);
    const uint64_t qh = (uint64_t)((u128)zh * hi + (((u128)zl * hi) >> 64) + carry);
    uint64_t r = zl - qh * q;
    return r >= q ? r - q : r;
}

uint64_t mont_neg_inv(uint64_t q) {
    uint64_t inv = 1;
    for (int i = 0; i < 6; ++i) inv *= 2 - q * inv;
    return 0 - inv;
}

namespace {
bool probably_composite(uint64_t n, uint64_t base, uint64_t d, int s) {
    uint64_t v = powmod(base, d, n);
    if (v == 1 || v == n - 1) return false;
    for (int r = 1; r < s; ++r) {
        v = mulmod(v, v, n);
        if (v == n - 1) return false;
    }
    return true;
}
bool is_prime(uint64_t n) {
    if (n < 2) return false;
    uint64_t d = n - 1;
    int s = 0;
    while (!(d & 1)) d >>= 1, ++s;
    for (uint64_t base : {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37}) {
        if (n == base) return true;
        if (probably_composite(n, base, d, s)) return false;
    }
    return true;
}
uint64_t bitrev(uint64_t x, int bits) {
    uint64_t r = 0;
    for (int i = 0; i < bits; ++i) r = (r << 1) | ((x >> i) & 1);
    return r;
}
}  // namespace

// Primes k*2N+1 searched downwards from 2^bits per requested size, P sizes first.
void find_primes(const std::vector<uint64_t>& p_bits, const std::vector<uint64_t>& q_bits,
                 uint64_t N, std::vector<uint64_t>& p, std::vector<uint64_t>& q) {
    std::map<uint64_t, uint64_t> cursor;
    auto next = [&](uint64_t bits) {
        if (bits < 2 || bits > 62) fail(kInvalid, "prime bit size must be in [2, 62]");
        const uint64_t lo = (uint64_t{1} << (bits - 1)) / (2 * N);
        uint64_t& k = cursor[bits];
        if (k == 0) k = (uint64_t{1} << bits) / (2 * N);
        while (k-- > lo) {
            const uint64_t cand = k * 2 * N + 1;
            if (is_prime(cand)) return cand;
        }
        fail(kInvalid, "no unused prime found in the requested range");
    };
    p.clear();
    q.clear();
    for (uint64_t b : p_bits) p.push_back(next(b));
    for (uint64_t b : q_bits) q.push_back(next(b));
}

void ntt_tables(uint64_t N, uint64_t q, uint64_t* fwd, uint64_t* fwd_s, uint64_t* inv,
                uint64_t* inv_s, uint64_t& n_inv) {
    if ((q - 1) % (2 * N) != 0) fail(kInvalid, "modulus is not 1 mod 2N");
    // Smallest generator candidate whose (q-1)/2N power is a primitive 2N-th root.
    const uint64_t e = (q - 1) / (2 * N);
    uint64_t psi = 0;
    for (uint64_t a = 2; a + 2 <= q; ++a) {
        const uint64_t c = powmod(a, e, q);
        if (powmod(c, N, q) == q - 1) {
            psi = c;
            break;
        }
    }
    if (!psi) fail(kInvalid, "no primitive 2N-th root of unity");
    const uint64_t psi_inv = powmod(psi, q - 2, q);
    // fwd[m+i] = psi^((2*rev_m(i)+1) * N/(2m)); inv[m+i] = psi^-((2*rev_m(i)+1) * N/(2m)).
    // Exponents stay below N, so two power tables of N entries cover them.
    std::vector<uint64_t> pw(N), pwi(N);
    pw[0] = pwi[0] = 1;
    for (uint64_t j = 1; j < N; ++j) {
        pw[j] = mulmod(pw[j - 1], psi, q);
        pwi[j] = mulmod(pwi[j - 1], psi_inv, q);
    }
    fwd[0] = inv[0] = 1;
    for (uint64_t m = 1; m < N; m <<= 1) {
        const int mb = __builtin_ctzll(m);
        const uint64_t k = N / (2 * m);
        for (uint64_t i = 0; i < m; ++i) {
            const uint64_t ex = (2 * bitrev(i, mb) + 1) * k;
            fwd[m + i] = pw[ex];
            inv[m + i] = pwi[ex];
        }
    }
    for (uint64_t i = 0; i < N; ++i) {
        fwd_s[i] = shoup(fwd[i], q);
        inv_s[i] = shoup(inv[i], q);
    }
    n_inv = powmod(N, q - 2, q);
}

}  // namespace wg::host
