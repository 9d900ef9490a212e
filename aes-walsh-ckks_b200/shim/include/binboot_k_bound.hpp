// EvalMod K bound of sparse-secret bootstrapping (the reference's src/math/binboot_k_bound.hpp):
// computed by the device library's host code (wg_evalmod_k_bound).
#ifndef BINBOOT_K_BOUND_HPP
#define BINBOOT_K_BOUND_HPP

#include <cstddef>

struct BinBootKBound {
    size_t mathematical_k = 0;
    size_t evalmod_k = 0;
    // Not computed by this build (0): only the K values steer the bootstrap.
    long double failure_probability = 0.0L;
};

BinBootKBound required_binboot_k_bound(size_t coefficient_count, size_t hamming_weight,
                                       long double target_failure_probability);

#endif  // BINBOOT_K_BOUND_HPP
