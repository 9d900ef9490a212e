// Host-side table generation for one parameter set.
//
// References:
//   ModUp precompute        build_approx_crt_modup_precomp,
//                           src/ckks/context/relinearization_key_generation.cpp:45-129,
//                           per level/digit as in src/ckks/context/ckks_context.cpp:468-514
//   folded P^-1 mod q       src/ckks/context/ckks_context.cpp:540-560
//   rescale constants       src/ckks/context/ckks_context.cpp:565-599
#include <algorithm>
#include <cstring>

#include "wg_internal.hpp"
#include "wg_tables.hpp"

namespace wg {
namespace {

struct TableImage {
    std::vector<uint64_t>& words;
    size_t put(const std::vector<uint64_t>& v) {
        const size_t off = words.size();
        words.insert(words.end(), v.begin(), v.end());
        return off;
    }
    size_t put(const std::vector<double>& v) {
        const size_t off = words.size();
        for (double d : v) {
            uint64_t w;
            std::memcpy(&w, &d, 8);
            words.push_back(w);
        }
        return off;
    }
    size_t put(const std::vector<int>& v) {  // two ints per word
        const size_t off = words.size();
        words.resize(off + (v.size() + 1) / 2, 0);
        std::memcpy(words.data() + off, v.data(), v.size() * sizeof(int));
        return off;
    }
};

}  // namespace

size_t parts_at(size_t level, size_t nq, size_t alpha, size_t dnum) {
    if (level >= nq) return 0;
    const size_t p_ = (level + 1 + alpha - 1) / alpha;
    return p_ < dnum ? p_ : dnum;
}

HostTables build_tables(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np, size_t dnum) {
    HostTables H;
    H.N = N;
    H.nq = nq;
    H.np = np;
    H.dnum = dnum;
    H.alpha = (nq + dnum - 1) / dnum;
    // Per-modulus constants and twiddles.
    const size_t nm = nq + np;
    H.mods.resize(nm);
    H.tw.assign(nm * 4 * N, 0);
    for (size_t i = 0; i < nm; ++i) {
        const uint64_t m = i < nq ? q[i] : p[i - nq];
        Modulus& md = H.mods[i];
        std::memset(&md, 0, sizeof(md));
        md.q = m;
        host::barrett_const(m, md.mu_lo, md.mu_hi);
        md.qninv = host::mont_neg_inv(m);
        uint64_t* t = H.tw.data() + i * 4 * N;
        host::ntt_tables(N, m, t, t + N, t + 2 * N, t + 3 * N, md.n_inv);
        md.n_inv_shoup = host::shoup(md.n_inv, m);
        md.inv_q = 1.0 / (double)m;
    }

    TableImage img{H.words};
    // ModUp descriptors for every level and digit.
    H.modup.resize(nq);
    for (size_t level = 0; level < nq; ++level) {
        const size_t L = level + 1;
        const size_t parts = parts_at(level, nq, H.alpha, dnum);
        for (size_t part = 0; part < parts; ++part) {
            const size_t s0 = part * H.alpha, s1 = std::min(s0 + H.alpha, L);
            std::vector<uint64_t> src(q + s0, q + s1), dst;
            std::vector<int> dst_limb, dst_mod;
            for (size_t i = 0; i < s0; ++i) dst.push_back(q[i]), dst_limb.push_back((int)i), dst_mod.push_back((int)i);
            for (size_t i = s1; i < L; ++i) dst.push_back(q[i]), dst_limb.push_back((int)i), dst_mod.push_back((int)i);
            for (size_t i = 0; i < np; ++i)
                dst.push_back(p[i]), dst_limb.push_back((int)(L + i)), dst_mod.push_back((int)(nq + i));
            const size_t sc = src.size(), dc = dst.size();
            std::vector<uint64_t> qhat_inv(sc), qhat_inv_s(sc), qhat(dc * sc), qhat_s(dc * sc), corr(dc * (sc + 1));
            std::vector<double> src_inv(sc);
            for (size_t i = 0; i < sc; ++i) {
                const uint64_t qi = src[i];
                uint64_t lo, hi;
                host::barrett_const(qi, lo, hi);
                src_inv[i] = 1.0 / (double)qi;
                uint64_t acc = 1;
                for (size_t j = 0; j < sc; ++j)
                    if (j != i) acc = host::barrett_mul(acc, src[j] % qi, qi, lo, hi);
                qhat_inv[i] = host::inverse(acc, qi);
                qhat_inv_s[i] = host::shoup(qhat_inv[i], qi);
                for (size_t t = 0; t < dc; ++t) {
                    const uint64_t m = dst[t];
                    uint64_t mlo, mhi;
                    host::barrett_const(m, mlo, mhi);
                    uint64_t a2 = 1;
                    for (size_t j = 0; j < sc; ++j)
                        if (j != i) a2 = host::barrett_mul(a2, src[j] % m, m, mlo, mhi);
                    qhat[t * sc + i] = a2;
                    qhat_s[t * sc + i] = host::shoup(a2, m);
                }
            }
            for (size_t t = 0; t < dc; ++t) {
                const uint64_t m = dst[t];
                uint64_t mlo, mhi;
                host::barrett_const(m, mlo, mhi);
                uint64_t prod = 1;
                for (size_t j = 0; j < sc; ++j) prod = host::barrett_mul(prod, src[j] % m, m, mlo, mhi);
                uint64_t run = 0;
                corr[t * (sc + 1)] = 0;
                for (size_t al = 1; al <= sc; ++al) {
                    run += prod;
                    if (run >= m) run -= m;
                    corr[t * (sc + 1) + al] = run;
                }
            }
            ModUpOffsets o;
            o.src_count = (int)sc;
            o.dst_count = (int)dc;
            o.src_first = (int)s0;
            o.qhat_inv = img.put(qhat_inv);
            o.qhat_inv_s = img.put(qhat_inv_s);
            o.src_inv = img.put(src_inv);
            o.qhat = img.put(qhat);
            o.qhat_s = img.put(qhat_s);
            o.corr = img.put(corr);
            o.dst_limb = img.put(dst_limb);
            o.dst_mod = img.put(dst_mod);
            H.modup[level].push_back(o);
        }
    }
    // Folded ModDown constants per level.
    H.fold_inv.resize(nq);
    H.fold_inv_s.resize(nq);
    for (size_t level = 0; level < nq; ++level) {
        std::vector<uint64_t> inv((level + 1) * np), inv_s((level + 1) * np);
        for (size_t qi = 0; qi <= level; ++qi)
            for (size_t pi = 0; pi < np; ++pi) {
                const uint64_t v = host::inverse(p[pi] % q[qi], q[qi]);
                inv[qi * np + pi] = v;
                inv_s[qi * np + pi] = host::shoup(v, q[qi]);
            }
        H.fold_inv[level] = img.put(inv);
        H.fold_inv_s[level] = img.put(inv_s);
    }
    // Rescale constants per dropped limb.
    H.rescale.assign(nq, 0);
    for (size_t d = 1; d < nq; ++d) {
        std::vector<uint64_t> v(4 * d);
        const uint64_t pd = q[d];
        for (size_t i = 0; i < d; ++i) {
            const uint64_t qi = q[i];
            const uint64_t one_s = host::shoup(1, qi);
            const uint64_t p_mod = pd % qi;
            const uint64_t inv_p = host::inverse(p_mod, qi);
            v[i] = one_s;
            v[d + i] = inv_p;
            v[2 * d + i] = host::shoup(inv_p, qi);
            v[3 * d + i] = (pd >> 1) % qi;
        }
        H.rescale[d] = img.put(v);
    }

    return H;
}

}  // namespace wg
