// Bootstrapping DFT plans on the host (wg_dftplan.cpp): the factorized homomorphic DFT's
// diagonals, before they are encoded into QP plaintexts on the device (wg_dftplan_dev.cu).
#pragma once
#include <complex>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace wg {
namespace dft {

using cplx = std::complex<double>;

// One transform to factorize (the reference's CKKSBootstrapDftMatrixLiteral fields this path
// uses, src/ckks/operations/bootstrap/ckks_bootstrap_dft.hpp).
struct Literal {
    bool coeffs_to_slots = false;     // CoeffsToSlots (else SlotsToCoeffs)
    size_t level = 0;                 // level of the first stage
    size_t baby_step_count = 0;       // 0: chosen per stage from its diagonals
    int log_bsgs_ratio = 1;
    size_t stage_count = 0;           // factors when no scale groups are given
    std::vector<std::vector<size_t>> scale_groups;  // log2 plaintext scales, one group per rescale
    std::vector<size_t> merge_depths;              // FFT levels per factor (empty: balanced)
    size_t active_slots = 0;          // 0: N/2
    double transform_scale = 1.0;
    size_t input_selector_start = 0, input_selector_size = 0;  // SlotsToCoeffs only
};

// One generated stage: its nonzero diagonals (active_slots values each, ascending index).
struct Stage {
    size_t level = 0;
    double plaintext_scale = 0.0;
    bool rescale_after = true;
    size_t baby = 0;
    size_t slots = 0;
    std::vector<size_t> indices;
    std::vector<std::vector<cplx>> diagonals;
};

// Stages of the factorized DFT for a ring of degree N whose Q moduli are q (the plaintext scale
// of a stage depends on the modulus it will drop).
std::vector<Stage> generate_plan(const Literal& lit, size_t N, const std::vector<uint64_t>& q);

// The baby-step count the reference picks for a set of diagonal indices.
size_t auto_baby_steps(size_t slots, const std::vector<size_t>& indices, int log_bsgs_ratio);

}  // namespace dft
}  // namespace wg
