/* CPU oracle: plain-C restatement of the reference CKKS residue path.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker for the device library, never part of it.
 * Citations are file:line inside the reference project (TrustworthyComputing/aes-walsh-ckks).
 */
#define _GNU_SOURCE
#include "ckks_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------------------------
 * Scalar modular arithmetic: src/math/modarith/modarith.hpp, modarith.cpp
 * ---------------------------------------------------------------------------------------- */

/* barrett_const_computation, modarith.cpp:3-8: floor((2^128 - 1) / q) split in two words. */
void orc_barrett_const(uint64_t q, uint64_t* mu_lo, uint64_t* mu_hi) {
    u128 ratio = (~(u128)0) / q;
    *mu_lo = (uint64_t)ratio;
    *mu_hi = (uint64_t)(ratio >> 64);
}

/* barrett_reduce, modarith.hpp:16-32.  One conditional subtraction: the result can be in
 * [q, 2q) for some inputs, exactly as in the reference. */
uint64_t orc_barrett_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t mu_lo, uint64_t mu_hi) {
    u128 z = (u128)a * b;
    uint64_t z_lo = (uint64_t)z, z_hi = (uint64_t)(z >> 64);
    u128 t = (u128)z_hi * mu_lo + (((u128)z_lo * mu_lo) >> 64);
    uint64_t carry = (uint64_t)(t >> 64);
    uint64_t q_hat = (uint64_t)((u128)z_hi * mu_hi + (((u128)z_lo * mu_hi) >> 64) + carry);
    uint64_t res = z_lo - q_hat * q;
    if (res >= q) res -= q;
    return res;
}

/* barrett_reduce_u64, modarith.hpp:53-58. */
static uint64_t barrett_u64(uint64_t a, uint64_t q, uint64_t mu_hi) {
    uint64_t q_hat = (uint64_t)(((u128)a * mu_hi) >> 64);
    uint64_t res = a - q_hat * q;
    if (res >= q) res -= q;
    return res;
}

/* compute_shoup, modarith.cpp:10-13 (truncated to 64 bits like the reference). */
uint64_t orc_shoup_const(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

/* mul_mod_shoup, modarith.hpp:93-99. */
static inline uint64_t mul_shoup(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t u = (uint64_t)(((u128)a * ws) >> 64);
    uint64_t res = a * w - u * q;
    if (res >= q) res -= q;
    return res;
}

/* reduce_u64_mod_q_shoup, modarith.hpp:34-41. */
static inline uint64_t reduce_shoup(uint64_t x, uint64_t q, uint64_t one_shoup) {
    uint64_t u = (uint64_t)(((u128)x * one_shoup) >> 64);
    uint64_t r = x - u * q;
    if (r >= q) r -= q;
    if (r >= q) r -= q;
    return r;
}

/* reduce_mod_4q, add_mod_q, sub_mod_q: modarith.hpp:43-81. */
static inline uint64_t red4q(uint64_t x, uint64_t q) {
    uint64_t two_q = q << 1;
    if (x >= two_q) x -= two_q;
    if (x >= q) x -= q;
    return x;
}
static inline uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t r = a + b;
    if (r >= q) r -= q;
    return r;
}
static inline uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t r = a - b;
    uint64_t mask = (uint64_t)0 - (uint64_t)(a < b);
    return r + (mask & q);
}

/* ckks_montgomery_neg_inverse64 / ckks_montgomery_mul_normal_by_montgomery,
 * modarith.hpp:101-130. */
static uint64_t mont_neg_inv(uint64_t q) {
    uint64_t inv = 1;
    for (int i = 0; i < 6; ++i) inv *= (uint64_t)2 - q * inv;
    return (uint64_t)0 - inv;
}
static inline uint64_t mont_mul(uint64_t normal, uint64_t mont, uint64_t q, uint64_t qninv) {
    u128 t = (u128)normal * mont;
    uint64_t m = (uint64_t)t * qninv;
    uint64_t u = (uint64_t)((t + (u128)m * q) >> 64);
    if (u >= q) u -= q;
    return u;
}
static uint64_t radix_mod(uint64_t q) { return (uint64_t)(((u128)1 << 64) % q); }

/* naive_mul_mod_u64, powmod, mod_inverse: modarith.hpp:62-65, modarith.cpp:15-40. */
static inline uint64_t mulmod_naive(uint64_t a, uint64_t b, uint64_t m) {
    return (uint64_t)(((u128)a * b) % m);
}
static uint64_t powmod(uint64_t a, uint64_t b, uint64_t m) {
    a %= m;
    uint64_t r = 1;
    while (b) {
        if (b & 1) r = mulmod_naive(r, a, m);
        a = mulmod_naive(a, a, m);
        b >>= 1;
    }
    return r;
}
static uint64_t mod_inverse(uint64_t a, uint64_t m) {
    int64_t m0 = (int64_t)m, t, qq;
    int64_t x0 = 0, x1 = 1;
    if (m == 1) return 0;
    while (a > 1) {
        qq = (int64_t)(a / m);
        t = (int64_t)m;
        m = a % m;
        a = (uint64_t)t;
        t = x0;
        x0 = x1 - qq * x0;
        x1 = t;
    }
    if (x1 < 0) x1 += m0;
    return (uint64_t)x1;
}

/* ------------------------------------------------------------------------------------------
 * Prime chain: src/util/random.cpp:9-131 (descending k*2N+1 per bit size, Miller-Rabin with
 * the first twelve prime bases, P primes first, then Q primes).
 * ---------------------------------------------------------------------------------------- */
static int mr_composite(uint64_t n, uint64_t base, uint64_t d, int s) {
    uint64_t v = powmod(base, d, n);
    if (v == 1 || v == n - 1) return 0;
    for (int r = 1; r < s; ++r) {
        v = mulmod_naive(v, v, n);
        if (v == n - 1) return 0;
    }
    return 1;
}
static int is_prime(uint64_t n) {
    static const uint64_t bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    int s = 0;
    uint64_t d = n - 1;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    for (int i = 0; i < 12; ++i) {
        if (n == bases[i]) return 1;
        if (mr_composite(n, bases[i], d, s)) return 0;
    }
    return 1;
}

int orc_find_primes(const uint64_t* p_bits, size_t np, const uint64_t* q_bits, size_t nq,
                    uint64_t N, uint64_t* p_out, uint64_t* q_out) {
    /* next_k per bit size (bit sizes are < 64, so a flat array replaces the std::map). */
    uint64_t next_k[64];
    memset(next_k, 0, sizeof(next_k));
    for (size_t idx = 0; idx < np + nq; ++idx) {
        uint64_t bits = idx < np ? p_bits[idx] : q_bits[idx - np];
        if (bits < 2 || bits > 63) return -1;
        uint64_t start = ((uint64_t)1 << (bits - 1)) / (2 * N);
        if (next_k[bits] == 0) next_k[bits] = ((uint64_t)1 << bits) / (2 * N);
        uint64_t found = 0;
        while (next_k[bits]-- > start) {
            uint64_t cand = next_k[bits] * 2 * N + 1;
            if (is_prime(cand)) {
                found = cand;
                break;
            }
        }
        if (!found) return -2;
        if (idx < np)
            p_out[idx] = found;
        else
            q_out[idx - np] = found;
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------
 * Negacyclic NTT: src/math/ntt/ntt.cpp
 * ---------------------------------------------------------------------------------------- */
static uint64_t bit_reverse(uint64_t x, unsigned bits) {
    uint64_t r = 0;
    for (unsigned i = 0; i < bits; ++i)
        if (x & ((uint64_t)1 << i)) r |= (uint64_t)1 << (bits - 1 - i);
    return r;
}
static unsigned ilog2u(uint64_t x) {
    unsigned r = 0;
    while (((uint64_t)1 << r) < x) ++r;
    return r;
}

/* find_root_of_unity (ntt.cpp:28-42) + generate_negacyclic_ntt_twiddles (ntt.cpp:54-148). */
int orc_ntt_tables(uint64_t N, uint64_t q, uint64_t* fwd, uint64_t* fwd_shoup, uint64_t* inv,
                   uint64_t* inv_shoup_np1, uint64_t* n_inv) {
    if ((q - 1) % (2 * N) != 0) return -1;
    uint64_t e = (q - 1) / (2 * N), psi = 0;
    for (uint64_t a = 2; a <= q - 2; ++a) {
        uint64_t cand = powmod(a, e, q);
        if (powmod(cand, N, q) == q - 1) {
            psi = cand;
            break;
        }
    }
    if (!psi) return -2;
    const uint64_t w = mulmod_naive(psi, psi, q);
    const unsigned logn = ilog2u(N);
    uint64_t* psi_pow = malloc(N * sizeof(uint64_t));
    uint64_t* psi_inv_pow = malloc(N * sizeof(uint64_t));
    uint64_t* stage = malloc((N / 2 + 1) * sizeof(uint64_t));
    psi_pow[0] = 1;
    for (uint64_t i = 1; i < N; ++i) psi_pow[i] = mulmod_naive(psi_pow[i - 1], psi, q);
    const uint64_t psi_inv = powmod(psi, q - 2, q);
    psi_inv_pow[0] = 1;
    for (uint64_t i = 1; i < N; ++i) psi_inv_pow[i] = mulmod_naive(psi_inv_pow[i - 1], psi_inv, q);

    for (uint64_t i = 0; i < N; ++i) fwd[i] = 1, inv[i] = 1;
    stage[0] = 1;
    for (uint64_t i = 1; i < N / 2; ++i) stage[i] = mulmod_naive(stage[i - 1], w, q);
    for (uint64_t m = 1; m < N; m <<= 1) {
        uint64_t step = N / (m << 1);
        unsigned sb = ilog2u(m);
        for (uint64_t i = 0; i < m; ++i) fwd[m + i] = stage[bit_reverse(i, sb) * step];
    }
    for (uint64_t m = 1, k = N >> 1; m < N; m <<= 1, k >>= 1)
        for (uint64_t i = 0; i < m; ++i) fwd[m + i] = mulmod_naive(fwd[m + i], psi_pow[k], q);

    const uint64_t w_inv = powmod(w, q - 2, q);
    stage[0] = 1;
    for (uint64_t i = 1; i < N / 2; ++i) stage[i] = mulmod_naive(stage[i - 1], w_inv, q);
    for (uint64_t m = 1; m < N; m <<= 1) {
        uint64_t step = N / (m << 1);
        unsigned sb = ilog2u(m);
        for (uint64_t i = 0; i < m; ++i) inv[m + i] = stage[bit_reverse(i, sb) * step];
    }
    for (uint64_t m = N >> 1, k = 1; m > 0; m >>= 1, k <<= 1)
        for (uint64_t i = 0; i < m; ++i) inv[m + i] = mulmod_naive(inv[m + i], psi_inv_pow[k], q);

    for (uint64_t i = 0; i < N; ++i) {
        fwd_shoup[i] = orc_shoup_const(fwd[i], q);
        inv_shoup_np1[i] = orc_shoup_const(inv[i], q);
    }
    *n_inv = powmod(N, q - 2, q);
    inv_shoup_np1[N] = orc_shoup_const(*n_inv, q);
    (void)logn;
    free(psi_pow);
    free(psi_inv_pow);
    free(stage);
    return 0;
}

/* ntt_forward_dit2_lazy (ntt.cpp:235-285): Harvey butterflies, output in [0,4q). */
static void ntt_fwd_lazy(uint64_t* a, uint64_t N, uint64_t q, const uint64_t* tw, const uint64_t* tws) {
    const uint64_t two_q = q << 1;
    for (uint64_t m = 1, k = N >> 1; m < N; m <<= 1, k >>= 1) {
        for (uint64_t i = 0; i < m; ++i) {
            const uint64_t w = tw[m + i], ws = tws[m + i];
            uint64_t* x0 = a + (i << 1) * k;
            uint64_t* x1 = x0 + k;
            for (uint64_t j = 0; j < k; ++j) {
                uint64_t t = x0[j];
                if (t >= two_q) t -= two_q;
                uint64_t v = x1[j];
                uint64_t uh = (uint64_t)(((u128)v * ws) >> 64);
                uint64_t u = v * w - uh * q;
                x0[j] = t + u;
                x1[j] = t + two_q - u;
            }
        }
    }
}

/* ntt_inverse_dif2_butterflies + final N^-1 scaling (ntt.cpp:331-386). */
static void ntt_inv(uint64_t* a, uint64_t N, uint64_t q, const uint64_t* tw, const uint64_t* tws,
                    uint64_t n_inv, int lazy) {
    const uint64_t two_q = q << 1;
    for (uint64_t m = N >> 1, k = 1; m > 0; m >>= 1, k <<= 1) {
        for (uint64_t i = 0; i < m; ++i) {
            uint64_t* x0 = a + (i << 1) * k;
            uint64_t* x1 = x0 + k;
            const uint64_t psi = tw[m + i], pss = tws[m + i];
            for (uint64_t j = 0; j < k; ++j) {
                uint64_t t = x0[j], u = x1[j];
                uint64_t sum = t + u;
                if (sum >= two_q) sum -= two_q;
                x0[j] = sum;
                uint64_t diff = t - u + two_q;
                uint64_t hi = (uint64_t)(((u128)diff * pss) >> 64);
                x1[j] = diff * psi - hi * q;
            }
        }
    }
    for (uint64_t i = 0; i < N; ++i) {
        uint64_t r = mul_shoup(a[i], n_inv, tws[N], q);
        a[i] = lazy ? r : red4q(r, q);
    }
}

/* ------------------------------------------------------------------------------------------
 * Context: moduli, twiddles and precomputed constants.
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    uint64_t q, mu_lo, mu_hi, qninv, n_inv;
    uint64_t *fwd, *fwds, *inv, *invs; /* invs has N+1 entries */
} modulus_t;

/* ApproxCrtModUpPrecomp, built as in build_approx_crt_modup_precomp
 * (src/ckks/context/relinearization_key_generation.cpp:45-129). */
typedef struct {
    size_t src_count, dst_count;
    uint64_t* src;        /* src moduli */
    uint64_t* dst;        /* dst moduli */
    uint64_t* qhat_inv;   /* [src] */
    uint64_t* qhat_inv_s; /* [src] */
    double* src_inv;      /* [src] 1.0 / q_i */
    uint64_t* qhat;       /* [dst][src] */
    uint64_t* qhat_s;     /* [dst][src] */
    uint64_t* corr;       /* [dst][src+1] alpha * prod(src) mod dst */
} modup_t;

struct orc_ctx {
    uint64_t N;
    size_t nq, np, dnum, alpha;
    modulus_t* qm; /* nq */
    modulus_t* pm; /* np */
    modup_t** modup; /* [level][part] */
    size_t* parts;   /* active parts per level */
    uint64_t** fold_inv;   /* [level] -> [(level+1)*np] */
    uint64_t** fold_inv_s;
    /* rescale constants per dropped limb d: [d] -> arrays of length d (and d*N) */
    uint64_t** rs_one_s;
    uint64_t** rs_inv_p;
    uint64_t** rs_inv_p_s;
    uint64_t** rs_half_ntt;
};

static void modulus_init(modulus_t* m, uint64_t N, uint64_t q) {
    m->q = q;
    orc_barrett_const(q, &m->mu_lo, &m->mu_hi);
    m->qninv = mont_neg_inv(q);
    m->fwd = malloc(N * 8);
    m->fwds = malloc(N * 8);
    m->inv = malloc(N * 8);
    m->invs = malloc((N + 1) * 8);
    orc_ntt_tables(N, q, m->fwd, m->fwds, m->inv, m->invs, &m->n_inv);
}
static void modulus_free(modulus_t* m) {
    free(m->fwd);
    free(m->fwds);
    free(m->inv);
    free(m->invs);
}

static void modup_build(modup_t* mu, const uint64_t* src, size_t sc, const uint64_t* dst, size_t dc) {
    mu->src_count = sc;
    mu->dst_count = dc;
    mu->src = malloc(sc * 8);
    mu->dst = malloc((dc ? dc : 1) * 8);
    memcpy(mu->src, src, sc * 8);
    memcpy(mu->dst, dst, dc * 8);
    mu->qhat_inv = malloc(sc * 8);
    mu->qhat_inv_s = malloc(sc * 8);
    mu->src_inv = malloc(sc * sizeof(double));
    mu->qhat = calloc(dc * sc + 1, 8);
    mu->qhat_s = calloc(dc * sc + 1, 8);
    mu->corr = calloc(dc * (sc + 1) + 1, 8);
    for (size_t i = 0; i < sc; ++i) {
        const uint64_t qi = src[i];
        uint64_t lo, hi;
        orc_barrett_const(qi, &lo, &hi);
        mu->src_inv[i] = 1.0 / (double)qi;
        uint64_t acc = 1;
        for (size_t j = 0; j < sc; ++j)
            if (j != i) acc = orc_barrett_mul(acc, src[j] % qi, qi, lo, hi);
        mu->qhat_inv[i] = mod_inverse(acc, qi);
        mu->qhat_inv_s[i] = orc_shoup_const(mu->qhat_inv[i], qi);
        for (size_t t = 0; t < dc; ++t) {
            const uint64_t m = dst[t];
            uint64_t mlo, mhi;
            orc_barrett_const(m, &mlo, &mhi);
            uint64_t a2 = 1;
            for (size_t j = 0; j < sc; ++j)
                if (j != i) a2 = orc_barrett_mul(a2, src[j] % m, m, mlo, mhi);
            mu->qhat[t * sc + i] = a2;
            mu->qhat_s[t * sc + i] = orc_shoup_const(a2, m);
        }
    }
    for (size_t t = 0; t < dc; ++t) {
        const uint64_t m = dst[t];
        uint64_t mlo, mhi;
        orc_barrett_const(m, &mlo, &mhi);
        uint64_t prod = 1;
        for (size_t j = 0; j < sc; ++j) prod = orc_barrett_mul(prod, src[j] % m, m, mlo, mhi);
        uint64_t corr = 0;
        mu->corr[t * (sc + 1)] = 0;
        for (size_t al = 1; al <= sc; ++al) {
            corr = add_mod(corr, prod, m);
            mu->corr[t * (sc + 1) + al] = corr;
        }
    }
}
static void modup_free(modup_t* mu) {
    free(mu->src);
    free(mu->dst);
    free(mu->qhat_inv);
    free(mu->qhat_inv_s);
    free(mu->src_inv);
    free(mu->qhat);
    free(mu->qhat_s);
    free(mu->corr);
}

size_t orc_ctx_alpha(const orc_ctx* c) { return c->alpha; }

orc_ctx* orc_ctx_create(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np,
                        size_t dnum) {
    if (dnum == 0 || dnum > nq || np == 0) return NULL;
    orc_ctx* c = calloc(1, sizeof(orc_ctx));
    c->N = N;
    c->nq = nq;
    c->np = np;
    c->dnum = dnum;
    c->alpha = (nq + dnum - 1) / dnum;
    c->qm = calloc(nq, sizeof(modulus_t));
    c->pm = calloc(np, sizeof(modulus_t));
    for (size_t i = 0; i < nq; ++i) modulus_init(&c->qm[i], N, q[i]);
    for (size_t i = 0; i < np; ++i) modulus_init(&c->pm[i], N, p[i]);

    /* ModUp precompute per level / part: ckks_context.cpp:468-514. */
    c->modup = calloc(nq, sizeof(modup_t*));
    c->parts = calloc(nq, sizeof(size_t));
    uint64_t* dst = malloc((nq + np) * 8);
    for (size_t lev = 0; lev < nq; ++lev) {
        const size_t L = lev + 1;
        size_t parts = (L + c->alpha - 1) / c->alpha;
        if (parts > dnum) parts = dnum;
        c->parts[lev] = parts;
        c->modup[lev] = calloc(parts, sizeof(modup_t));
        for (size_t part = 0; part < parts; ++part) {
            size_t s0 = part * c->alpha, s1 = s0 + c->alpha < L ? s0 + c->alpha : L;
            size_t dc = 0;
            for (size_t i = 0; i < s0; ++i) dst[dc++] = q[i];
            for (size_t i = s1; i < L; ++i) dst[dc++] = q[i];
            for (size_t i = 0; i < np; ++i) dst[dc++] = p[i];
            modup_build(&c->modup[lev][part], q + s0, s1 - s0, dst, dc);
        }
    }
    free(dst);

    /* Folded P^-1 mod q tables: ckks_context.cpp:540-560. */
    c->fold_inv = calloc(nq, sizeof(uint64_t*));
    c->fold_inv_s = calloc(nq, sizeof(uint64_t*));
    for (size_t lev = 0; lev < nq; ++lev) {
        c->fold_inv[lev] = malloc((lev + 1) * np * 8);
        c->fold_inv_s[lev] = malloc((lev + 1) * np * 8);
        for (size_t qi = 0; qi <= lev; ++qi)
            for (size_t pi = 0; pi < np; ++pi) {
                uint64_t inv = mod_inverse(p[pi] % q[qi], q[qi]);
                c->fold_inv[lev][qi * np + pi] = inv;
                c->fold_inv_s[lev][qi * np + pi] = orc_shoup_const(inv, q[qi]);
            }
    }

    /* Rescale constants: ckks_context.cpp:565-599. */
    c->rs_one_s = calloc(nq, sizeof(uint64_t*));
    c->rs_inv_p = calloc(nq, sizeof(uint64_t*));
    c->rs_inv_p_s = calloc(nq, sizeof(uint64_t*));
    c->rs_half_ntt = calloc(nq, sizeof(uint64_t*));
    for (size_t d = 1; d < nq; ++d) {
        const uint64_t pd = q[d], half = pd >> 1;
        c->rs_one_s[d] = malloc(d * 8);
        c->rs_inv_p[d] = malloc(d * 8);
        c->rs_inv_p_s[d] = malloc(d * 8);
        c->rs_half_ntt[d] = malloc(d * N * 8);
        for (size_t i = 0; i < d; ++i) {
            const modulus_t* m = &c->qm[i];
            uint64_t one_s = orc_shoup_const(1, m->q);
            uint64_t p_mod = reduce_shoup(pd, m->q, one_s);
            uint64_t inv_p = mod_inverse(p_mod, m->q);
            uint64_t half_mod = reduce_shoup(half, m->q, one_s);
            uint64_t* h = c->rs_half_ntt[d] + i * N;
            for (uint64_t j = 0; j < N; ++j) h[j] = half_mod;
            ntt_fwd_lazy(h, N, m->q, m->fwd, m->fwds);
            for (uint64_t j = 0; j < N; ++j) h[j] = red4q(h[j], m->q);
            c->rs_one_s[d][i] = one_s;
            c->rs_inv_p[d][i] = inv_p;
            c->rs_inv_p_s[d][i] = orc_shoup_const(inv_p, m->q);
        }
    }
    return c;
}

void orc_ctx_destroy(orc_ctx* c) {
    if (!c) return;
    for (size_t i = 0; i < c->nq; ++i) modulus_free(&c->qm[i]);
    for (size_t i = 0; i < c->np; ++i) modulus_free(&c->pm[i]);
    for (size_t lev = 0; lev < c->nq; ++lev) {
        for (size_t part = 0; part < c->parts[lev]; ++part) modup_free(&c->modup[lev][part]);
        free(c->modup[lev]);
        free(c->fold_inv[lev]);
        free(c->fold_inv_s[lev]);
        free(c->rs_one_s[lev]);
        free(c->rs_inv_p[lev]);
        free(c->rs_inv_p_s[lev]);
        free(c->rs_half_ntt[lev]);
    }
    free(c->modup);
    free(c->parts);
    free(c->fold_inv);
    free(c->fold_inv_s);
    free(c->rs_one_s);
    free(c->rs_inv_p);
    free(c->rs_inv_p_s);
    free(c->rs_half_ntt);
    free(c->qm);
    free(c->pm);
    free(c);
}

static void fwd_limb(const modulus_t* m, uint64_t* a, uint64_t N, int lazy) {
    ntt_fwd_lazy(a, N, m->q, m->fwd, m->fwds);
    if (!lazy)
        for (uint64_t i = 0; i < N; ++i) a[i] = red4q(a[i], m->q);
}
static void inv_limb(const modulus_t* m, uint64_t* a, uint64_t N, int lazy) {
    ntt_inv(a, N, m->q, m->inv, m->invs, m->n_inv, lazy);
}

void orc_ntt(const orc_ctx* c, uint64_t* poly, size_t first, size_t limbs, int which, int inverse,
             int lazy) {
    const modulus_t* ms = which ? c->pm : c->qm;
    for (size_t i = 0; i < limbs; ++i) {
        if (inverse)
            inv_limb(&ms[first + i], poly + i * c->N, c->N, lazy);
        else
            fwd_limb(&ms[first + i], poly + i * c->N, c->N, lazy);
    }
}

/* ------------------------------------------------------------------------------------------
 * Hybrid key switching: src/ckks/operations/keyswitch/ckks_keyswitch.cpp
 * ---------------------------------------------------------------------------------------- */

/* apply_hps_crt_base_change (ckks_keyswitch.cpp:278-332).  The alpha estimate is a separate
 * multiply and add: the reference build does not contract this one into an FMA. */
static void hps_modup(const modup_t* mu, const uint64_t* const* src, uint64_t* const* dst, uint64_t N) {
    uint64_t scaled[64];
    for (uint64_t coeff = 0; coeff < N; ++coeff) {
        double alpha_est = 0.0;
        for (size_t i = 0; i < mu->src_count; ++i) {
            const uint64_t qi = mu->src[i];
            const uint64_t x = red4q(src[i][coeff], qi);
            const uint64_t s = mul_shoup(x, mu->qhat_inv[i], mu->qhat_inv_s[i], qi);
            scaled[i] = s;
            alpha_est = alpha_est + (double)s * mu->src_inv[i];
        }
        uint64_t hps_alpha = (uint64_t)(alpha_est + 0.5);
        if (hps_alpha > mu->src_count) hps_alpha = mu->src_count;
        for (size_t t = 0; t < mu->dst_count; ++t) {
            const uint64_t m = mu->dst[t];
            uint64_t acc = 0;
            for (size_t i = 0; i < mu->src_count; ++i) {
                const size_t k = t * mu->src_count + i;
                acc = add_mod(acc, mul_shoup(scaled[i], mu->qhat[k], mu->qhat_s[k], m), m);
            }
            const uint64_t corr = mu->corr[t * (mu->src_count + 1) + hps_alpha];
            dst[t][coeff] = sub_mod(acc, corr, m);
        }
    }
}

/* ckks_apply_folded_approx_crt_moddown_pair_eval_q (ckks_keyswitch.cpp:521-607), for one of
 * the two polynomials (the pair runs the same per-polynomial arithmetic).  The alpha estimate
 * is fused (fma), as the reference build contracts it here. */
static void folded_moddown(const orc_ctx* c, size_t level, const uint64_t* src_p, uint64_t* dst_q) {
    const uint64_t N = c->N;
    const size_t np = c->np;
    const uint64_t* invs = c->fold_inv[level];
    const uint64_t* inv_s = c->fold_inv_s[level];
    double p_inv[16];
    for (size_t pi = 0; pi < np; ++pi) p_inv[pi] = 1.0 / (double)c->pm[pi].q;
    uint64_t* contrib = malloc(N * 8);
    for (size_t qi = 0; qi <= level; ++qi) {
        const modulus_t* m = &c->qm[qi];
        const uint64_t q = m->q;
        for (uint64_t coeff = 0; coeff < N; ++coeff) {
            uint64_t acc = 0;
            double alpha_est = 0.0;
            for (size_t pi = 0; pi < np; ++pi) {
                const uint64_t s = red4q(src_p[pi * N + coeff], c->pm[pi].q);
                alpha_est = fma((double)s, p_inv[pi], alpha_est);
                const uint64_t term = mul_shoup(barrett_u64(s, q, m->mu_hi), invs[qi * np + pi],
                                                inv_s[qi * np + pi], q);
                acc = add_mod(acc, term, q);
            }
            uint64_t hps_alpha = (uint64_t)(alpha_est + 0.5);
            if (hps_alpha > np) hps_alpha = np;
            contrib[coeff] = sub_mod(acc, hps_alpha, q);
        }
        fwd_limb(m, contrib, N, 0);
        uint64_t* d = dst_q + qi * N;
        for (uint64_t coeff = 0; coeff < N; ++coeff) d[coeff] = sub_mod(d[coeff], contrib[coeff], q);
    }
    free(contrib);
}

/* ckks_hybrid_key_switch_inplace (ckks_keyswitch.cpp:1330-1641) with folded keys in Montgomery
 * form (the reference defaults: fold_hybrid_keyswitch = montgomery = true). */
int orc_keyswitch(const orc_ctx* c, size_t level, const uint64_t* key_term, const uint64_t* key,
                  size_t key_level, uint64_t* b, uint64_t* a, int b_add, int a_add) {
    const uint64_t N = c->N;
    const size_t L = level + 1, K = c->np, T = L + K;
    const size_t key_limbs = key_level + 1 + K;
    if (level >= c->nq || key_level < level) return -1;
    const size_t parts = c->parts[level];
    uint64_t* coeff = malloc(L * N * 8);
    uint64_t* acc_a = calloc(T * N, 8);
    uint64_t* acc_b = calloc(T * N, 8);
    uint64_t* digit = malloc(T * N * 8);
    memcpy(coeff, key_term, L * N * 8);
    for (size_t i = 0; i < L; ++i) inv_limb(&c->qm[i], coeff + i * N, N, 1);

    for (size_t part = 0; part < parts; ++part) {
        const size_t s0 = part * c->alpha, s1 = s0 + c->alpha < L ? s0 + c->alpha : L;
        const modup_t* mu = &c->modup[level][part];
        const uint64_t* srcp[64];
        uint64_t* dstp[128];
        size_t dc = 0;
        for (size_t s = s0; s < s1; ++s) srcp[s - s0] = coeff + s * N;
        for (size_t i = 0; i < s0; ++i) dstp[dc++] = digit + i * N;
        for (size_t i = s1; i < L; ++i) dstp[dc++] = digit + i * N;
        for (size_t i = 0; i < K; ++i) dstp[dc++] = digit + (L + i) * N;
        if (dc) hps_modup(mu, srcp, dstp, N);

        const uint64_t* ka = key + (part * 2 + 0) * key_limbs * N;
        const uint64_t* kb = key + (part * 2 + 1) * key_limbs * N;
        for (size_t i = 0; i < T; ++i) {
            const int is_p = i >= L;
            const modulus_t* m = is_p ? &c->pm[i - L] : &c->qm[i];
            const size_t key_limb = is_p ? key_level + 1 + (i - L) : i;
            const uint64_t* dig;
            if (!is_p && i >= s0 && i < s1) {
                dig = key_term + i * N;
            } else {
                fwd_limb(m, digit + i * N, N, 1);
                dig = digit + i * N;
            }
            const uint64_t* kap = ka + key_limb * N;
            const uint64_t* kbp = kb + key_limb * N;
            uint64_t* aa = acc_a + i * N;
            uint64_t* bb = acc_b + i * N;
            for (uint64_t j = 0; j < N; ++j) {
                aa[j] = add_mod(aa[j], mont_mul(dig[j], kap[j], m->q, m->qninv), m->q);
                bb[j] = add_mod(bb[j], mont_mul(dig[j], kbp[j], m->q, m->qninv), m->q);
            }
        }
    }
    for (size_t pi = 0; pi < K; ++pi) {
        inv_limb(&c->pm[pi], acc_a + (L + pi) * N, N, 1);
        inv_limb(&c->pm[pi], acc_b + (L + pi) * N, N, 1);
    }
    folded_moddown(c, level, acc_a + L * N, acc_a);
    folded_moddown(c, level, acc_b + L * N, acc_b);
    for (size_t i = 0; i < L; ++i) {
        const uint64_t q = c->qm[i].q;
        for (uint64_t j = 0; j < N; ++j) {
            const size_t k = i * N + j;
            b[k] = b_add ? add_mod(b[k], acc_b[k], q) : acc_b[k];
            a[k] = a_add ? add_mod(a[k], acc_a[k], q) : acc_a[k];
        }
    }
    free(coeff);
    free(acc_a);
    free(acc_b);
    free(digit);
    return 0;
}

/* build_ntt_automorphism_map (src/ckks/context/rotation_key_generation.cpp:80-90). */
void orc_automorphism_map(uint64_t N, uint64_t g, uint64_t* dst_to_src) {
    const unsigned logn = ilog2u(N);
    const uint64_t ring = N << 1;
    for (uint64_t d = 0; d < N; ++d) {
        uint64_t src_exp = ((2 * d + 1) * g) % ring;
        uint64_t s = (src_exp - 1) >> 1;
        dst_to_src[bit_reverse(d, logn)] = bit_reverse(s, logn);
    }
}

/* rotation_automorphism_index (rotation_key_generation.cpp:73-78). */
uint64_t orc_rotation_galois(uint64_t N, int64_t rotation) {
    const int64_t slots = (int64_t)(N >> 1);
    int64_t r = rotation % slots;
    if (r < 0) r += slots;
    return powmod(5, (uint64_t)r, N << 1);
}

static void apply_map(uint64_t* poly, uint64_t N, size_t limbs, const uint64_t* map) {
    uint64_t* tmp = malloc(N * 8);
    for (size_t l = 0; l < limbs; ++l) {
        uint64_t* p = poly + l * N;
        for (uint64_t i = 0; i < N; ++i) tmp[i] = p[map[i]];
        memcpy(p, tmp, N * 8);
    }
    free(tmp);
}

/* ckks_rotate_inplace (src/ckks/operations/keyswitch/ckks_rotation.cpp:41-96). */
int orc_rotate(const orc_ctx* c, size_t level, uint64_t* b, uint64_t* a, const uint64_t* key,
               size_t key_level, int64_t rotation) {
    const int64_t slots = (int64_t)(c->N >> 1);
    int64_t r = rotation % slots;
    if (r < 0) r += slots;
    if (r == 0) return 0;
    uint64_t* kt = malloc((level + 1) * c->N * 8);
    memcpy(kt, a, (level + 1) * c->N * 8);
    int rc = orc_keyswitch(c, level, kt, key, key_level, b, a, 1, 0);
    free(kt);
    if (rc) return rc;
    uint64_t* map = malloc(c->N * 8);
    orc_automorphism_map(c->N, orc_rotation_galois(c->N, r), map);
    apply_map(b, c->N, level + 1, map);
    apply_map(a, c->N, level + 1, map);
    free(map);
    return 0;
}

/* ckks_conjugate_inplace (src/ckks/operations/keyswitch/ckks_conjugate.cpp:16-61):
 * automorphism X -> X^(2N-1) first, then the switch. */
int orc_conjugate(const orc_ctx* c, size_t level, uint64_t* b, uint64_t* a, const uint64_t* key,
                  size_t key_level) {
    uint64_t* map = malloc(c->N * 8);
    orc_automorphism_map(c->N, 2 * c->N - 1, map);
    apply_map(b, c->N, level + 1, map);
    apply_map(a, c->N, level + 1, map);
    free(map);
    uint64_t* kt = malloc((level + 1) * c->N * 8);
    memcpy(kt, a, (level + 1) * c->N * 8);
    int rc = orc_keyswitch(c, level, kt, key, key_level, b, a, 1, 0);
    free(kt);
    return rc;
}

/* ckks_mul_inplace(ct, ct) (src/ckks/operations/arith/ckks_mul.cpp:90-157): Barrett products
 * c2 = a1 a2, c0 = b1 b2, c1 = a1 b2 + b1 a2. */
int orc_mul(const orc_ctx* c, size_t level, uint64_t* b1, uint64_t* a1, const uint64_t* b2,
            const uint64_t* a2, uint64_t* c2) {
    const uint64_t N = c->N;
    for (size_t i = 0; i <= level; ++i) {
        const modulus_t* m = &c->qm[i];
        for (uint64_t j = 0; j < N; ++j) {
            const size_t k = i * N + j;
            const uint64_t x_a = a1[k], x_b = b1[k];
            c2[k] = orc_barrett_mul(x_a, a2[k], m->q, m->mu_lo, m->mu_hi);
            const uint64_t tmp = orc_barrett_mul(x_b, a2[k], m->q, m->mu_lo, m->mu_hi);
            b1[k] = orc_barrett_mul(x_b, b2[k], m->q, m->mu_lo, m->mu_hi);
            const uint64_t t2 = orc_barrett_mul(x_a, b2[k], m->q, m->mu_lo, m->mu_hi);
            a1[k] = add_mod(t2, tmp, m->q);
        }
    }
    return 0;
}

/* ckks_relin_hybrid_inplace (src/ckks/operations/keyswitch/ckks_relin.cpp:8-44). */
int orc_relin(const orc_ctx* c, size_t level, uint64_t* c0, uint64_t* c1, const uint64_t* c2,
              const uint64_t* key, size_t key_level) {
    return orc_keyswitch(c, level, c2, key, key_level, c0, c1, 1, 1);
}

/* ckks_rescale (src/ckks/operations/arith/ckks_rescale.cpp:68-148).  Polynomials keep their
 * (level+1)*N stride; only the first level*N residues are meaningful afterwards. */
int orc_rescale(const orc_ctx* c, size_t level, size_t npolys, uint64_t* polys) {
    if (level == 0 || level >= c->nq) return -1;
    const uint64_t N = c->N;
    const size_t stride = (level + 1) * N;
    const modulus_t* last = &c->qm[level];
    const uint64_t p = last->q, half_p = p >> 1;
    uint64_t* rem = malloc(N * 8);
    for (size_t k = 0; k < npolys; ++k) inv_limb(last, polys + k * stride + level * N, N, 0);
    for (size_t i = 0; i < level; ++i) {
        const modulus_t* m = &c->qm[i];
        const uint64_t one_s = c->rs_one_s[level][i];
        const uint64_t inv_p = c->rs_inv_p[level][i], inv_p_s = c->rs_inv_p_s[level][i];
        const uint64_t* half_ntt = c->rs_half_ntt[level] + i * N;
        for (size_t k = 0; k < npolys; ++k) {
            const uint64_t* drop = polys + k * stride + level * N;
            for (uint64_t j = 0; j < N; ++j) {
                uint64_t shift = drop[j] + half_p;
                if (shift >= p) shift -= p;
                rem[j] = reduce_shoup(shift, m->q, one_s);
            }
            fwd_limb(m, rem, N, 0);
            uint64_t* poly = polys + k * stride + i * N;
            for (uint64_t j = 0; j < N; ++j) {
                uint64_t num = add_mod(poly[j], half_ntt[j], m->q);
                uint64_t diff = sub_mod(num, rem[j], m->q);
                poly[j] = mul_shoup(diff, inv_p, inv_p_s, m->q);
            }
        }
    }
    free(rem);
    return 0;
}

/* Hoisted rotations (ckks_hoist_ciphertext_a_qp_eval, ckks_keyswitch.cpp:344-373, and
 * ckks_hybrid_key_switch_hoisted_inplace, :1072-1328).  The hoisted digits are exactly the
 * digits the plain switch builds, so each output equals a plain rotation of the input.
 * out layout: [rot][b, a][limb][N]. */
int orc_hoisted_rotations(const orc_ctx* c, size_t level, const uint64_t* b, const uint64_t* a,
                          const uint64_t* const* keys, size_t key_level, const int64_t* rots,
                          size_t nrot, uint64_t* out) {
    const size_t n = (level + 1) * c->N;
    for (size_t r = 0; r < nrot; ++r) {
        uint64_t* ob = out + (r * 2 + 0) * n;
        uint64_t* oa = out + (r * 2 + 1) * n;
        memcpy(ob, b, n * 8);
        memcpy(oa, a, n * 8);
        int rc = orc_rotate(c, level, ob, oa, keys[r], key_level, rots[r]);
        if (rc) return rc;
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------
 * Seeded test-data generation (key material follows generate_rotation_key_hybrid,
 * src/ckks/context/rotation_key_generation.cpp:92-199, with a seeded generator).
 * ---------------------------------------------------------------------------------------- */
static uint64_t splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t uniform_below(uint64_t* s, uint64_t q) {
    const uint64_t lim = UINT64_MAX - UINT64_MAX % q;
    uint64_t x;
    do x = splitmix(s);
    while (x >= lim);
    return x % q;
}
static int64_t gauss_int(uint64_t* s, double sigma) {
    double u1 = ((splitmix(s) >> 11) + 1) * (1.0 / 9007199254740993.0);
    double u2 = (splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
    double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    return (int64_t)llround(g * sigma);
}

void orc_sample_ternary(uint64_t N, size_t h, uint64_t seed, int8_t* out) {
    uint64_t s = seed;
    memset(out, 0, N);
    size_t placed = 0;
    while (placed < h) {
        uint64_t idx = splitmix(&s) % N;
        if (out[idx]) continue;
        out[idx] = (splitmix(&s) & 1) ? 1 : -1;
        ++placed;
    }
}

void orc_secret_automorphism(uint64_t N, uint64_t g, const int8_t* s, int8_t* out) {
    memset(out, 0, N);
    for (uint64_t i = 0; i < N; ++i) {
        uint64_t mapped = (i * g) % (2 * N);
        if (mapped >= N)
            out[mapped - N] = (int8_t)-s[i];
        else
            out[mapped] = s[i];
    }
}

static void small_to_ntt(const modulus_t* m, const int8_t* s, uint64_t N, uint64_t* out) {
    for (uint64_t j = 0; j < N; ++j) out[j] = s[j] < 0 ? m->q - (uint64_t)(-s[j]) : (uint64_t)s[j];
    fwd_limb(m, out, N, 0);
}

int orc_keygen_switch(const orc_ctx* c, const int8_t* src, int src_square, const int8_t* dst,
                      double sigma, uint64_t seed, uint64_t* key_out) {
    const uint64_t N = c->N;
    const size_t L = c->nq, K = c->np, T = L + K;
    uint64_t st = seed;
    uint64_t* s_src = malloc(T * N * 8);
    uint64_t* s_dst = malloc(T * N * 8);
    const modulus_t** ms = malloc(T * sizeof(modulus_t*));
    for (size_t i = 0; i < T; ++i) ms[i] = i < L ? &c->qm[i] : &c->pm[i - L];
    for (size_t i = 0; i < T; ++i) {
        small_to_ntt(ms[i], src, N, s_src + i * N);
        small_to_ntt(ms[i], dst, N, s_dst + i * N);
        if (src_square)
            for (uint64_t j = 0; j < N; ++j)
                s_src[i * N + j] = mulmod_naive(s_src[i * N + j], s_src[i * N + j], ms[i]->q);
    }
    for (size_t part = 0; part < c->dnum; ++part) {
        const size_t s0 = part * c->alpha, s1 = s0 + c->alpha < L ? s0 + c->alpha : L;
        if (s0 >= s1) break;
        uint64_t* ka = key_out + (part * 2 + 0) * T * N;
        uint64_t* kb = key_out + (part * 2 + 1) * T * N;
        for (size_t i = 0; i < T; ++i) {
            const modulus_t* m = ms[i];
            const uint64_t q = m->q;
            uint64_t p_mod = 1;
            for (size_t pi = 0; pi < K; ++pi) p_mod = mulmod_naive(p_mod, c->pm[pi].q % q, q);
            uint64_t* e = malloc(N * 8);
            for (uint64_t j = 0; j < N; ++j) {
                int64_t v = gauss_int(&st, sigma);
                e[j] = v < 0 ? q - (uint64_t)(-v) : (uint64_t)v;
            }
            fwd_limb(m, e, N, 0);
            for (uint64_t j = 0; j < N; ++j) {
                const uint64_t av = uniform_below(&st, q);
                uint64_t bv = sub_mod(e[j], mulmod_naive(av, s_dst[i * N + j], q), q);
                if (i >= s0 && i < s1) bv = add_mod(bv, mulmod_naive(s_src[i * N + j], p_mod, q), q);
                ka[i * N + j] = av;
                kb[i * N + j] = bv;
            }
            free(e);
            /* fold (hybrid_key_folding.hpp:50-77) and convert to Montgomery form
             * (hybrid_key_montgomery.hpp:12-36). */
            uint64_t fold;
            if (i < L) {
                fold = mod_inverse(p_mod, q);
            } else {
                uint64_t phat = 1;
                for (size_t pj = 0; pj < K; ++pj)
                    if (pj != i - L) phat = mulmod_naive(phat, c->pm[pj].q % q, q);
                fold = mod_inverse(phat, q);
            }
            const uint64_t scale = mulmod_naive(fold, radix_mod(q), q);
            for (uint64_t j = 0; j < N; ++j) {
                ka[i * N + j] = mulmod_naive(ka[i * N + j], scale, q);
                kb[i * N + j] = mulmod_naive(kb[i * N + j], scale, q);
            }
        }
    }
    free(s_src);
    free(s_dst);
    free(ms);
    return 0;
}

void orc_uniform_poly(const orc_ctx* c, size_t limbs, uint64_t seed, uint64_t* out) {
    uint64_t st = seed;
    for (size_t i = 0; i < limbs; ++i)
        for (uint64_t j = 0; j < c->N; ++j) out[i * c->N + j] = uniform_below(&st, c->qm[i].q);
}

int orc_encrypt(const orc_ctx* c, size_t level, const uint64_t* m_ntt, const int8_t* s,
                double sigma, uint64_t seed, uint64_t* b, uint64_t* a) {
    const uint64_t N = c->N;
    uint64_t st = seed;
    uint64_t* sn = malloc(N * 8);
    uint64_t* e = malloc(N * 8);
    for (size_t i = 0; i <= level; ++i) {
        const modulus_t* m = &c->qm[i];
        small_to_ntt(m, s, N, sn);
        uint64_t st_e = seed ^ 0x5bd1e995u;
        for (uint64_t j = 0; j < N; ++j) {
            int64_t v = gauss_int(&st_e, sigma);
            e[j] = v < 0 ? m->q - (uint64_t)(-v) : (uint64_t)v;
        }
        fwd_limb(m, e, N, 0);
        for (uint64_t j = 0; j < N; ++j) {
            const uint64_t av = uniform_below(&st, m->q);
            a[i * N + j] = av;
            b[i * N + j] = add_mod(sub_mod(e[j], mulmod_naive(av, sn[j], m->q), m->q),
                                   m_ntt[i * N + j] % m->q, m->q);
        }
    }
    free(sn);
    free(e);
    return 0;
}

int orc_decrypt_coeffs(const orc_ctx* c, size_t level, const uint64_t* b, const uint64_t* a,
                       const int8_t* s, double* out) {
    const uint64_t N = c->N;
    const size_t use = level >= 1 ? 2 : 1;
    uint64_t* sn = malloc(N * 8);
    uint64_t* m = malloc(use * N * 8);
    for (size_t i = 0; i < use; ++i) {
        const modulus_t* md = &c->qm[i];
        small_to_ntt(md, s, N, sn);
        for (uint64_t j = 0; j < N; ++j)
            m[i * N + j] = add_mod(red4q(b[i * N + j], md->q) % md->q,
                                   mulmod_naive(a[i * N + j] % md->q, sn[j], md->q), md->q);
        inv_limb(md, m + i * N, N, 0);
    }
    if (use == 1) {
        const uint64_t q = c->qm[0].q;
        for (uint64_t j = 0; j < N; ++j)
            out[j] = m[j] > q / 2 ? -(double)(q - m[j]) : (double)m[j];
    } else {
        const uint64_t q0 = c->qm[0].q, q1 = c->qm[1].q;
        const u128 Q = (u128)q0 * q1;
        const uint64_t q0_inv_q1 = mod_inverse(q0 % q1, q1);
        for (uint64_t j = 0; j < N; ++j) {
            uint64_t x0 = m[j], x1 = m[N + j];
            uint64_t t = mulmod_naive((x1 + q1 - x0 % q1) % q1, q0_inv_q1, q1);
            u128 x = (u128)x0 + (u128)t * q0;
            out[j] = x > Q / 2 ? -(double)(Q - x) : (double)x;
        }
    }
    free(sn);
    free(m);
    return 0;
}

/* The batched-ops workload (mul, relin, rescale, rotate per ciphertext) on the CPU, with
 * OpenMP over ciphertexts like the reference parallelizes independent ciphertexts. */
int orc_batched_ops(const orc_ctx* c, size_t count, const size_t* levels, uint64_t* x_b,
                    uint64_t* x_a, const uint64_t* y_b, const uint64_t* y_a,
                    const uint64_t* relin_key, const uint64_t* const* rot_keys,
                    const int64_t* rots, size_t key_level, size_t stride, int threads) {
    int err = 0;
#pragma omp parallel for schedule(dynamic) num_threads(threads)
    for (long i = 0; i < (long)count; ++i) {
        const size_t lev = levels[i];
        const size_t n = (lev + 1) * c->N;
        uint64_t* b = x_b + (size_t)i * stride;
        uint64_t* a = x_a + (size_t)i * stride;
        uint64_t* c2 = malloc(n * 8);
        uint64_t* buf = malloc(2 * n * 8);
        int rc = orc_mul(c, lev, b, a, y_b + (size_t)i * stride, y_a + (size_t)i * stride, c2);
        rc |= orc_relin(c, lev, b, a, c2, relin_key, key_level);
        memcpy(buf, b, n * 8);
        memcpy(buf + n, a, n * 8);
        rc |= orc_rescale(c, lev, 2, buf);
        const size_t n2 = lev * c->N;
        memcpy(b, buf, n2 * 8);
        memcpy(a, buf + n, n2 * 8);
        rc |= orc_rotate(c, lev - 1, b, a, rot_keys[i], key_level, rots[i]);
        if (rc) {
#pragma omp atomic write
            err = rc;
        }
        free(c2);
        free(buf);
    }
    return err;
}

/* ------------------------------------------------------------------------------------------
 * QP-domain baby-step / giant-step linear-transform stage:
 * ckks_apply_linear_transform_owned_stage_qp
 * (src/ckks/operations/bootstrap/ckks_linear_transform.cpp:1174-1407).
 * ---------------------------------------------------------------------------------------- */

/* single-polynomial folded ModDown (ckks_keyswitch.cpp:609-673): alpha as multiply + add */
static void folded_moddown_single(const orc_ctx* c, size_t level, const uint64_t* src_p, uint64_t* dst_q) {
    const uint64_t N = c->N;
    const size_t np = c->np;
    const uint64_t* invs = c->fold_inv[level];
    const uint64_t* inv_s = c->fold_inv_s[level];
    double p_inv[16];
    for (size_t pi = 0; pi < np; ++pi) p_inv[pi] = 1.0 / (double)c->pm[pi].q;
    uint64_t* contrib = malloc(N * 8);
    for (size_t qi = 0; qi <= level; ++qi) {
        const modulus_t* m = &c->qm[qi];
        const uint64_t q = m->q;
        for (uint64_t coeff = 0; coeff < N; ++coeff) {
            uint64_t acc = 0;
            double alpha_est = 0.0;
            for (size_t pi = 0; pi < np; ++pi) {
                const uint64_t s = red4q(src_p[pi * N + coeff], c->pm[pi].q);
                alpha_est = alpha_est + (double)s * p_inv[pi];
                acc = add_mod(acc, mul_shoup(barrett_u64(s, q, m->mu_hi), invs[qi * np + pi], inv_s[qi * np + pi], q), q);
            }
            uint64_t hps_alpha = (uint64_t)(alpha_est + 0.5);
            if (hps_alpha > np) hps_alpha = np;
            contrib[coeff] = sub_mod(acc, hps_alpha, q);
        }
        fwd_limb(m, contrib, N, 0);
        uint64_t* d = dst_q + qi * N;
        for (uint64_t coeff = 0; coeff < N; ++coeff) d[coeff] = sub_mod(d[coeff], contrib[coeff], q);
    }
    free(contrib);
}

static const modulus_t* qp_mod(const orc_ctx* c, size_t L, size_t i) { return i < L ? &c->qm[i] : &c->pm[i - L]; }

/* Digits of a QP key switch of `key_term` (Q eval, level): digit[part] holds every QP limb in
 * evaluation form (source limbs: the key term itself). */
static uint64_t* qp_digits(const orc_ctx* c, size_t level, const uint64_t* key_term) {
    const uint64_t N = c->N;
    const size_t L = level + 1, K = c->np, T = L + K;
    const size_t parts = c->parts[level];
    uint64_t* coeff = malloc(L * N * 8);
    uint64_t* digits = malloc(parts * T * N * 8);
    memcpy(coeff, key_term, L * N * 8);
    for (size_t i = 0; i < L; ++i) inv_limb(&c->qm[i], coeff + i * N, N, 1);
    for (size_t part = 0; part < parts; ++part) {
        const size_t s0 = part * c->alpha, s1 = s0 + c->alpha < L ? s0 + c->alpha : L;
        uint64_t* dg = digits + part * T * N;
        const uint64_t* srcp[64];
        uint64_t* dstp[128];
        size_t dc = 0;
        for (size_t s = s0; s < s1; ++s) srcp[s - s0] = coeff + s * N;
        for (size_t i = 0; i < s0; ++i) dstp[dc++] = dg + i * N;
        for (size_t i = s1; i < L; ++i) dstp[dc++] = dg + i * N;
        for (size_t i = 0; i < K; ++i) dstp[dc++] = dg + (L + i) * N;
        if (dc) hps_modup(&c->modup[level][part], srcp, dstp, N);
        for (size_t i = 0; i < T; ++i) {
            if (i >= s0 && i < s1) {
                memcpy(dg + i * N, key_term + i * N, N * 8);
            } else {
                fwd_limb(qp_mod(c, L, i), dg + i * N, N, 1);
            }
        }
    }
    free(coeff);
    return digits;
}

/* acc_{a,b} (+)= sum_parts REDC(digit * key) over all QP limbs. */
static void qp_mac(const orc_ctx* c, size_t level, const uint64_t* digits, const uint64_t* key, size_t key_level,
                   uint64_t* acc_a, uint64_t* acc_b) {
    const uint64_t N = c->N;
    const size_t L = level + 1, K = c->np, T = L + K;
    const size_t key_limbs = key_level + 1 + K;
    for (size_t part = 0; part < c->parts[level]; ++part) {
        const uint64_t* ka = key + (part * 2 + 0) * key_limbs * N;
        const uint64_t* kb = key + (part * 2 + 1) * key_limbs * N;
        for (size_t i = 0; i < T; ++i) {
            const modulus_t* m = qp_mod(c, L, i);
            const size_t kl = i < L ? i : key_level + 1 + (i - L);
            const uint64_t* d = digits + (part * T + i) * N;
            for (uint64_t j = 0; j < N; ++j) {
                acc_a[i * N + j] = add_mod(acc_a[i * N + j], mont_mul(d[j], ka[kl * N + j], m->q, m->qninv), m->q);
                acc_b[i * N + j] = add_mod(acc_b[i * N + j], mont_mul(d[j], kb[kl * N + j], m->q, m->qninv), m->q);
            }
        }
    }
}

static void apply_map_qp(uint64_t* poly, uint64_t N, size_t limbs, const uint64_t* map) { apply_map(poly, N, limbs, map); }

int orc_lt_stage(const orc_ctx* c, size_t level, size_t nterms, const uint64_t* indices, const uint64_t* diags,
                 size_t baby, size_t slots, int rescale, const uint64_t* const* keys, const int64_t* key_rots,
                 size_t nkeys, size_t key_level, uint64_t* b, uint64_t* a) {
    const uint64_t N = c->N;
    const size_t L = level + 1, K = c->np, T = L + K;
    const size_t full = N / 2;
    if (!slots) slots = full;
    const size_t ngiant = (slots + baby - 1) / baby;
    /* key lookup by normalized rotation */
#define FIND_KEY(rot, out)                                                   \
    do {                                                                     \
        out = NULL;                                                          \
        for (size_t kk = 0; kk < nkeys; ++kk)                                \
            if ((uint64_t)(((key_rots[kk] % (int64_t)full) + full) % full) == (uint64_t)((rot) % full)) out = keys[kk]; \
    } while (0)
    /* babies */
    char* need = calloc(baby, 1);
    for (size_t t = 0; t < nterms; ++t) need[indices[t] % baby] = 1;
    uint64_t** ba = calloc(baby, sizeof(uint64_t*));
    uint64_t** bb = calloc(baby, sizeof(uint64_t*));
    uint64_t* digits = NULL;
    uint64_t* map = malloc(N * 8);
    for (size_t r = 0; r < baby; ++r) {
        if (!need[r]) continue;
        ba[r] = calloc(T * N, 8);
        bb[r] = calloc(T * N, 8);
        if (r == 0) {
            memcpy(ba[r], a, L * N * 8);
            memcpy(bb[r], b, L * N * 8);
            continue;
        }
        if (!digits) digits = qp_digits(c, level, a);
        const uint64_t* key;
        FIND_KEY(r, key);
        if (!key) return -3;
        memcpy(bb[r], b, L * N * 8);
        qp_mac(c, level, digits, key, key_level, ba[r], bb[r]);
        orc_automorphism_map(N, orc_rotation_galois(N, (int64_t)r), map);
        apply_map_qp(ba[r], N, T, map);
        apply_map_qp(bb[r], N, T, map);
    }
    uint64_t* out_a = calloc(T * N, 8);
    uint64_t* out_b = calloc(T * N, 8);
    uint64_t* in_a = malloc(T * N * 8);
    uint64_t* in_b = malloc(T * N * 8);
    uint64_t* sw_a = malloc(T * N * 8);
    uint64_t* sw_b = malloc(T * N * 8);
    for (size_t g = 0; g < ngiant; ++g) {
        int have = 0;
        memset(in_a, 0, T * N * 8);
        memset(in_b, 0, T * N * 8);
        for (size_t t = 0; t < nterms; ++t) {
            if (indices[t] / baby != g) continue;
            have = 1;
            const size_t r = indices[t] % baby;
            const uint64_t* d = diags + t * T * N;
            for (size_t i = 0; i < T; ++i) {
                const modulus_t* m = qp_mod(c, L, i);
                for (uint64_t j = 0; j < N; ++j) {
                    const size_t k = i * N + j;
                    in_a[k] = add_mod(in_a[k], mont_mul(ba[r][k], d[k], m->q, m->qninv), m->q);
                    in_b[k] = add_mod(in_b[k], mont_mul(bb[r][k], d[k], m->q, m->qninv), m->q);
                }
            }
        }
        if (!have) continue;
        if (g == 0) {
            for (size_t i = 0; i < T; ++i) {
                const modulus_t* m = qp_mod(c, L, i);
                for (uint64_t j = 0; j < N; ++j) {
                    const size_t k = i * N + j;
                    out_a[k] = add_mod(out_a[k], in_a[k], m->q);
                    out_b[k] = add_mod(out_b[k], in_b[k], m->q);
                }
            }
            continue;
        }
        /* single ModDown of the inner a, then a QP key switch of that key term */
        for (size_t pi = 0; pi < K; ++pi) inv_limb(&c->pm[pi], in_a + (L + pi) * N, N, 1);
        folded_moddown_single(c, level, in_a + L * N, in_a);
        uint64_t* dg = qp_digits(c, level, in_a);
        const uint64_t* key;
        FIND_KEY(g * baby, key);
        if (!key) return -3;
        memset(sw_a, 0, T * N * 8);
        memset(sw_b, 0, T * N * 8);
        qp_mac(c, level, dg, key, key_level, sw_a, sw_b);
        free(dg);
        orc_automorphism_map(N, orc_rotation_galois(N, (int64_t)(g * baby)), map);
        for (size_t i = 0; i < T; ++i) {
            const modulus_t* m = qp_mod(c, L, i);
            for (uint64_t j = 0; j < N; ++j) {
                const size_t k = i * N + j, s = i * N + map[j];
                out_a[k] = add_mod(out_a[k], sw_a[s], m->q);
                out_b[k] = add_mod(out_b[k], add_mod(sw_b[s], in_b[s], m->q), m->q);
            }
        }
    }
#undef FIND_KEY
    /* pair ModDown */
    for (size_t pi = 0; pi < K; ++pi) {
        inv_limb(&c->pm[pi], out_a + (L + pi) * N, N, 1);
        inv_limb(&c->pm[pi], out_b + (L + pi) * N, N, 1);
    }
    folded_moddown(c, level, out_a + L * N, out_a);
    folded_moddown(c, level, out_b + L * N, out_b);
    memcpy(b, out_b, L * N * 8);
    memcpy(a, out_a, L * N * 8);
    int rc = 0;
    if (rescale) {
        uint64_t* buf = malloc(2 * L * N * 8);
        memcpy(buf, b, L * N * 8);
        memcpy(buf + L * N, a, L * N * 8);
        rc = orc_rescale(c, level, 2, buf);
        memcpy(b, buf, level * N * 8);
        memcpy(a, buf + L * N, level * N * 8);
        free(buf);
    }
    for (size_t r = 0; r < baby; ++r) {
        free(ba[r]);
        free(bb[r]);
    }
    free(ba);
    free(bb);
    free(need);
    free(digits);
    free(map);
    free(out_a);
    free(out_b);
    free(in_a);
    free(in_b);
    free(sw_a);
    free(sw_b);
    return rc;
}

/* ------------------------------------------------------------------------------------------
 * Bootstrapping boundary steps
 * ------------------------------------------------------------------------------------------ */

/* center_lift_mod_q / signed_to_mod_q (src/ckks/operations/bootstrap/ckks_modraise.cpp:12-29). */
static int64_t center_lift(uint64_t v, uint64_t q) {
    const uint64_t half = q >> 1;
    return v > half ? -(int64_t)(q - v) : (int64_t)v;
}
static uint64_t signed_mod(int64_t v, uint64_t q) {
    if (v >= 0) return (uint64_t)v % q;
    const uint64_t m = (uint64_t)(-v) % q;
    return m == 0 ? 0 : q - m;
}

/* ckks_modraise_inplace / modraise_eval_poly_from_q0 (ckks_modraise.cpp:31-110): the q0 limb
 * of b and a (limb 0 of each buffer) is lifted to target_level+1 limbs, in place. */
int orc_modraise(const orc_ctx* c, size_t target_level, uint64_t* b, uint64_t* a) {
    const uint64_t N = c->N;
    if (target_level == 0 || target_level >= c->nq) return -1;
    uint64_t* coeff = malloc(N * 8);
    uint64_t* polys[2] = {b, a};
    for (int k = 0; k < 2; ++k) {
        uint64_t* x = polys[k];
        memcpy(coeff, x, N * 8);
        inv_limb(&c->qm[0], coeff, N, 0);
        for (size_t l = 0; l <= target_level; ++l) {
            const uint64_t q = c->qm[l].q;
            for (uint64_t i = 0; i < N; ++i) x[l * N + i] = signed_mod(center_lift(coeff[i], c->qm[0].q), q);
        }
        for (size_t l = 0; l <= target_level; ++l) fwd_limb(&c->qm[l], x + l * N, N, 0);
    }
    free(coeff);
    return 0;
}

/* hps_base_change_single_limb (src/ckks/operations/keyswitch/ckks_keyswitch.cpp:1645-1659). */
static uint64_t base_change_single(uint64_t v, uint64_t src, const modulus_t* dst) {
    const uint64_t reduced = red4q(v, src);
    const uint64_t r = barrett_u64(reduced, dst->q, dst->mu_hi);
    const uint64_t s = barrett_u64(src, dst->q, dst->mu_hi);
    return reduced >= (src >> 1) + 1 ? sub_mod(r, s, dst->q) : r;
}

/* ckks_q0p0_key_switch_level0_inplace (ckks_keyswitch.cpp:1661-1816), folded Montgomery key
 * (the reference defaults): key = [a: q0 limb, p0 limb][b: q0 limb, p0 limb].  Level-0
 * (b, a) updated in place. */
int orc_q0p0_switch(const orc_ctx* c, const uint64_t* key, uint64_t* b, uint64_t* a) {
    const uint64_t N = c->N;
    const modulus_t* q0 = &c->qm[0];
    const modulus_t* p0 = &c->pm[0];
    uint64_t* dc = malloc(N * 8);
    uint64_t* dp = malloc(N * 8);
    uint64_t* acc = calloc(4 * N, 8); /* a_q0, a_p0, b_q0, b_p0 */
    memcpy(dc, a, N * 8);
    inv_limb(q0, dc, N, 1);
    for (uint64_t i = 0; i < N; ++i) dp[i] = base_change_single(dc[i], q0->q, p0);
    fwd_limb(p0, dp, N, 1);
    for (uint64_t i = 0; i < N; ++i) {
        acc[i] = add_mod(0, mont_mul(a[i], key[i], q0->q, q0->qninv), q0->q);
        acc[2 * N + i] = add_mod(0, mont_mul(a[i], key[2 * N + i], q0->q, q0->qninv), q0->q);
        acc[N + i] = add_mod(0, mont_mul(dp[i], key[N + i], p0->q, p0->qninv), p0->q);
        acc[3 * N + i] = add_mod(0, mont_mul(dp[i], key[3 * N + i], p0->q, p0->qninv), p0->q);
    }
    inv_limb(p0, acc + N, N, 1);
    inv_limb(p0, acc + 3 * N, N, 1);
    /* ckks_apply_folded_approx_crt_moddown_pair_eval_q with P = {p0}, Q = {q0}, inverse p0^-1 */
    const uint64_t inv = mod_inverse(p0->q % q0->q, q0->q);
    const uint64_t inv_s = orc_shoup_const(inv, q0->q);
    const double p_inv = 1.0 / (double)p0->q;
    for (int poly = 0; poly < 2; ++poly) {
        const uint64_t* src = acc + (2 * poly + 1) * N;
        uint64_t* dst = acc + 2 * poly * N;
        for (uint64_t i = 0; i < N; ++i) {
            const uint64_t s = red4q(src[i], p0->q);
            const double alpha = fma((double)s, p_inv, 0.0);
            const uint64_t term = mul_shoup(barrett_u64(s, q0->q, q0->mu_hi), inv, inv_s, q0->q);
            uint64_t hps = (uint64_t)(alpha + 0.5);
            if (hps > 1) hps = 1;
            dc[i] = sub_mod(add_mod(0, term, q0->q), hps, q0->q);
        }
        fwd_limb(q0, dc, N, 0);
        for (uint64_t i = 0; i < N; ++i) dst[i] = sub_mod(dst[i], dc[i], q0->q);
    }
    for (uint64_t i = 0; i < N; ++i) {
        b[i] = add_mod(b[i], acc[2 * N + i], q0->q);
        a[i] = acc[i];
    }
    free(dc);
    free(dp);
    free(acc);
    return 0;
}
