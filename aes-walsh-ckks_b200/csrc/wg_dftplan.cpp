// Factorized homomorphic DFT plans (CoeffToSlot / SlotToCoeff) on the host.
//
// Reference: ckks_generate_bootstrap_dft_plan and its helpers,
// src/ckks/operations/bootstrap/ckks_bootstrap_dft.cpp:122-1079.  The special FFT of the
// slot vector (SlotsToCoeffs, fft_plain_vectors :334) or its inverse (CoeffsToSlots,
// ifft_plain_vectors :379) is written as log2(slots) sparse levels, each three diagonals
// (a: identity part, b and c: the rotated butterfly halves, powers of the 4*slots-th roots at
// the 5^j rotation group's exponents).  Consecutive levels are merged into one stage (the
// merge depths; by default as even as possible, the larger factors first for CoeffsToSlots),
// multiplying diagonal maps: (A * B)[d1 + d2] += A[d1] * rot(B[d2], d1).  Each stage is
// scaled by transform_scale^(1/stages) (CoeffsToSlots: (transform_scale / slots)^(1/stages)),
// gets its plaintext scale (q_drop^(bits / group bits) of its scale group, or
// q_drop / (2.01 max|diagonal|) without groups), its baby-step count (the cheapest
// BSGS split, giant steps weighted 2^log_bsgs_ratio) and the zero diagonals dropped.
//
// The diagonal values depend on floating-point operation order, and their encodings round
// them (llrint after the FFT), so the reference's order is kept: levels and merges in its
// sequence, map entries visited in ascending index order with the a, b, c terms added in that
// order, and every complex product as the reference's compiler forms it with fused
// multiply-adds (re = fma(x.re, y.re, -(x.im y.im)), im = fma(x.re, y.im, x.im y.re)); this
// file is built without any other contraction.
#include <algorithm>
#include <bit>
#include <cmath>
#include <limits>
#include <map>
#include <stdexcept>

#include "wg_dftplan.hpp"

namespace wg {
namespace dft {
namespace {

using Map = std::map<size_t, std::vector<cplx>>;

inline cplx cmul(const cplx& x, const cplx& y) {
    return {std::fma(x.real(), y.real(), -(x.imag() * y.imag())), std::fma(x.real(), y.imag(), x.imag() * y.real())};
}

struct Levels {
    std::vector<std::vector<cplx>> a, b, c;  // [level index], slots values each
};

// The three diagonals of every FFT level, in processing order (level index k <-> FFT level
// log_slots - k).
Levels fft_levels(size_t log_slots, bool inverse) {
    const size_t slots = size_t{1} << log_slots;
    const size_t nroots = slots << 2;
    constexpr double pi = 3.141592653589793238462643383279502884;
    std::vector<cplx> roots(nroots + 1);
    for (size_t i = 0; i <= nroots; ++i) {
        const double ang = 2.0 * pi * (double)i / (double)nroots;
        roots[i] = cplx(std::cos(ang), std::sin(ang));
    }
    std::vector<size_t> pow5(2 * slots + 1);
    pow5[0] = 1;
    for (size_t i = 1; i < pow5.size(); ++i) pow5[i] = (pow5[i - 1] * 5) & (nroots - 1);
    Levels L;
    L.a.assign(log_slots, {});
    L.b.assign(log_slots, {});
    L.c.assign(log_slots, {});
    for (size_t k = 0; k < log_slots; ++k) {
        // forward: block size m = 2, 4, ..., slots; inverse: m = slots, ..., 2
        const size_t m = inverse ? (slots >> k) : (size_t{2} << k);
        std::vector<cplx> a(slots), b(slots), c(slots);
        const size_t hm = m >> 1, gap = slots / m, mask = (m << 2) - 1;
        for (size_t i = 0; i < slots; i += m)
            for (size_t j = 0; j < hm; ++j) {
                const size_t e = pow5[j] & mask;
                const cplx w = roots[(inverse ? (m << 2) - e : e) * gap];
                const size_t i1 = i + j, i2 = i1 + hm;
                a[i1] = cplx(1.0, 0.0);
                a[i2] = -w;
                if (inverse) {
                    b[i1] = cplx(1.0, 0.0);
                    c[i2] = w;
                } else {
                    b[i1] = w;
                    c[i2] = cplx(1.0, 0.0);
                }
            }
        L.a[k] = std::move(a);
        L.b[k] = std::move(b);
        L.c[k] = std::move(c);
    }
    return L;
}

// Rotation of FFT level `level` (1..log_slots) in the diagonal index space.
size_t level_rotation(size_t log_slots, size_t level, bool c2s) {
    const size_t slots = size_t{1} << log_slots;
    const size_t r = c2s ? (size_t{1} << (level - 1)) : (size_t{1} << (log_slots - level));
    return r & (slots - 1);
}

void accumulate(Map& m, size_t idx, std::vector<cplx>&& v) {
    auto it = m.find(idx);
    if (it == m.end()) {
        m.emplace(idx, std::move(v));
        return;
    }
    auto& d = it->second;
    for (size_t i = 0; i < d.size(); ++i) d[i] += v[i];
}

// out[i] = mult[i] * v[(i + rot) mod n]
std::vector<cplx> rotate_times(const std::vector<cplx>& v, int64_t rot, const std::vector<cplx>& mult) {
    const size_t n = v.size(), mask = n - 1;
    const size_t off = (size_t)(((rot % (int64_t)n) + (int64_t)n) % (int64_t)n);
    std::vector<cplx> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = cmul(mult[i], v[(i + off) & mask]);
    return out;
}

// Diagonal map of one stage: its first FFT level, then its further levels merged in.
Map stage_map(const Levels& L, size_t log_slots, bool c2s, const std::vector<size_t>& merge, size_t stage,
              double scale) {
    const size_t slots = size_t{1} << log_slots;
    size_t level = log_slots;
    for (size_t i = 0; i < stage; ++i) level -= merge[i];
    Map m;
    {
        const size_t k = log_slots - level;
        const size_t r = level_rotation(log_slots, level, c2s);
        accumulate(m, 0, std::vector<cplx>(L.a[k]));
        accumulate(m, r, std::vector<cplx>(L.b[k]));
        accumulate(m, (slots - r) & (slots - 1), std::vector<cplx>(L.c[k]));
    }
    size_t next = level - 1;
    for (size_t j = 0; j + 1 < merge[stage]; ++j, --next) {
        const size_t k = log_slots - next;
        const size_t r = level_rotation(log_slots, next, c2s);
        Map merged;
        for (const auto& [idx, v] : m) {
            accumulate(merged, idx, rotate_times(v, 0, L.a[k]));
            accumulate(merged, (idx + r) & (slots - 1), rotate_times(v, (int64_t)r, L.b[k]));
            accumulate(merged, (idx + slots - r) & (slots - 1), rotate_times(v, -(int64_t)r, L.c[k]));
        }
        m = std::move(merged);
    }
    for (auto& [idx, v] : m) {
        if (idx >= slots || v.size() != slots) throw std::invalid_argument("dft plan: invalid diagonal");
        for (cplx& x : v) x *= scale;
    }
    return m;
}

std::vector<size_t> balanced_merge(size_t log_slots, size_t factors, bool c2s) {
    if (factors == 0 || factors > log_slots) throw std::invalid_argument("dft plan: invalid factor count");
    std::vector<size_t> merge(factors);
    size_t level = log_slots;
    for (size_t i = 0; i < factors; ++i) {
        const size_t rem = factors - i;
        const size_t depth = (level + rem - 1) / rem;
        merge[c2s ? i : factors - 1 - i] = depth;
        level -= depth;
    }
    return merge;
}

}  // namespace

size_t auto_baby_steps(size_t slots, const std::vector<size_t>& indices, int log_bsgs_ratio) {
    if (slots == 0 || indices.empty()) throw std::invalid_argument("dft plan: empty diagonal set");
    if (indices.size() <= 1) return 1;
    size_t best = 1, best_cost = std::numeric_limits<size_t>::max(), best_giants = best_cost;
    const size_t giant_weight = size_t{1} << std::max(0, log_bsgs_ratio);
    for (size_t n1 = 1; n1 < slots; n1 <<= 1) {
        std::vector<char> seen_giant(slots, 0), seen_baby(slots, 0);
        size_t giants = 0, babies = 0;
        for (size_t d : indices) {
            if (d >= slots) throw std::invalid_argument("dft plan: diagonal index exceeds slot count");
            const size_t r = d & (slots - 1);
            const size_t g = ((r / n1) * n1) & (slots - 1), b = r & (n1 - 1);
            if (!seen_giant[g]) {
                seen_giant[g] = 1;
                ++giants;
            }
            if (!seen_baby[b]) {
                seen_baby[b] = 1;
                ++babies;
            }
        }
        const size_t nz_g = giants > 0 && seen_giant[0] ? giants - 1 : giants;
        const size_t nz_b = babies > 0 && seen_baby[0] ? babies - 1 : babies;
        const size_t cost = giant_weight * nz_g + nz_b;
        if (cost < best_cost || (cost == best_cost && nz_g < best_giants)) {
            best_cost = cost;
            best_giants = nz_g;
            best = n1;
        }
    }
    return best;
}

std::vector<Stage> generate_plan(const Literal& lit, size_t N, const std::vector<uint64_t>& q) {
    const size_t full = N / 2;
    const size_t slots = lit.active_slots == 0 ? full : lit.active_slots;
    if (slots == 0 || slots > full || full % slots || !std::has_single_bit(slots))
        throw std::invalid_argument("dft plan: invalid active slot count");
    // factor schedule: (group, log scale, ends group)
    struct Factor {
        size_t group, bits;
        bool ends;
    };
    std::vector<Factor> sched;
    std::vector<size_t> group_bits;
    if (lit.scale_groups.empty()) {
        for (size_t i = 0; i < lit.stage_count; ++i) sched.push_back({i, 0, true});
    } else {
        for (size_t g = 0; g < lit.scale_groups.size(); ++g) {
            const auto& grp = lit.scale_groups[g];
            if (grp.empty()) throw std::invalid_argument("dft plan: empty scale group");
            size_t sum = 0;
            for (size_t f = 0; f < grp.size(); ++f) {
                if (grp[f] == 0) throw std::invalid_argument("dft plan: scale schedule entries must be positive");
                sum += grp[f];
                sched.push_back({g, grp[f], f + 1 == grp.size()});
            }
            group_bits.push_back(sum);
        }
    }
    const size_t factors = sched.size();
    const size_t log_slots = (size_t)std::countr_zero(slots);
    const size_t groups = lit.scale_groups.empty() ? lit.stage_count : lit.scale_groups.size();
    if (factors == 0 || factors > log_slots) throw std::invalid_argument("dft plan: invalid factorized stage count");
    if (lit.level >= q.size()) throw std::invalid_argument("dft plan: invalid matrix level");
    if (groups > lit.level) throw std::invalid_argument("dft plan: the stages consume more levels than available");
    if (!(lit.transform_scale > 0.0)) throw std::invalid_argument("dft plan: transform scale must be positive");
    if (lit.input_selector_size != 0 &&
        (lit.coeffs_to_slots || lit.input_selector_start >= slots || lit.input_selector_size > slots))
        throw std::invalid_argument("dft plan: invalid input selector");
    std::vector<size_t> merge;
    if (lit.merge_depths.empty()) {
        merge = balanced_merge(log_slots, factors, lit.coeffs_to_slots);
    } else {
        if (lit.merge_depths.size() != factors) throw std::invalid_argument("dft plan: merge-depth count mismatch");
        size_t total = 0;
        for (size_t d : lit.merge_depths) {
            if (d == 0) throw std::invalid_argument("dft plan: merge depths must be positive");
            total += d;
        }
        if (total != log_slots) throw std::invalid_argument("dft plan: merge depths must sum to log2(slots)");
        merge = lit.merge_depths;
    }
    const Levels L = fft_levels(log_slots, lit.coeffs_to_slots);
    const double stage_scale =
        lit.coeffs_to_slots ? std::pow(lit.transform_scale / (double)slots, 1.0 / (double)factors)
                            : std::pow(lit.transform_scale, 1.0 / (double)factors);
    std::vector<Stage> out;
    size_t level = lit.level;
    for (size_t s = 0; s < factors; ++s) {
        Map m = stage_map(L, log_slots, lit.coeffs_to_slots, merge, s, stage_scale);
        if (s == 0 && lit.input_selector_size != 0) {
            for (auto& [idx, v] : m)
                for (size_t row = 0; row < slots; ++row) {
                    const size_t col = (row + idx) % slots;
                    if ((col + slots - lit.input_selector_start) % slots >= lit.input_selector_size)
                        v[row] = cplx(0.0, 0.0);
                }
        }
        double max_abs = 0.0;
        for (const auto& [idx, v] : m)
            for (const cplx& x : v) max_abs = std::max(max_abs, std::abs(x));
        if (!(max_abs > 0.0)) throw std::runtime_error("dft plan: generated an empty stage");
        const double q_drop = (double)q[level];
        Stage st;
        st.level = level;
        st.plaintext_scale = lit.scale_groups.empty()
                                 ? q_drop / (2.01 * max_abs)
                                 : std::pow(q_drop, (double)sched[s].bits / (double)group_bits[sched[s].group]);
        st.rescale_after = sched[s].ends;
        st.slots = slots;
        for (auto& [idx, v] : m) {
            bool zero = true;
            for (const cplx& x : v)
                if (x.real() != 0.0 || x.imag() != 0.0) {
                    zero = false;
                    break;
                }
            if (zero) continue;
            st.indices.push_back(idx);
            st.diagonals.push_back(std::move(v));
        }
        if (st.indices.empty()) throw std::runtime_error("dft plan: generated stage has no nonzero diagonals");
        st.baby = lit.baby_step_count == 0 ? auto_baby_steps(slots, st.indices, lit.log_bsgs_ratio) : lit.baby_step_count;
        if (st.baby == 0 || st.baby > slots) throw std::invalid_argument("dft plan: invalid baby-step count");
        out.push_back(std::move(st));
        if (sched[s].ends && s + 1 < factors) {
            if (level == 0) throw std::runtime_error("dft plan: stage levels exhausted");
            --level;
        }
    }
    return out;
}

}  // namespace dft
}  // namespace wg
