// Host image of every table the kernels read (moduli, twiddles, ModUp / ModDown / rescale
// constants).  Built once per parameter set; the device library uploads it, the CPU emulation
// test reads it in place.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "wg_arith.cuh"

namespace wg {

struct ModUpOffsets {
    int src_count, dst_count, src_first;
    size_t qhat_inv, qhat_inv_s, src_inv, qhat, qhat_s, corr, dst_limb, dst_mod;
};

struct HostTables {
    uint64_t N = 0;
    size_t nq = 0, np = 0, dnum = 0, alpha = 0;
    std::vector<Modulus> mods;                     // nq + np
    std::vector<uint64_t> tw;                      // [mod][4][N]
    std::vector<uint64_t> words;                   // small tables, addressed by word offsets
    std::vector<std::vector<ModUpOffsets>> modup;  // [level][part]
    std::vector<size_t> fold_inv, fold_inv_s;      // [level] -> [(level+1)][np]
    std::vector<size_t> rescale;                   // [d] -> one_s[d], inv_p[d], inv_p_s[d], half[d]
};

size_t parts_at(size_t level, size_t nq, size_t alpha, size_t dnum);
HostTables build_tables(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np, size_t dnum);

}  // namespace wg
