// Host-side CKKS slot encoding (wg_encode.cpp).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace wg {
namespace host {

// Coefficient-form plaintext of the N/2 slot values re[i] + i im[i] at `scale`, one limb per
// modulus: out[l * N + k].
void encode_slots(size_t N, const double* re, const double* im, double scale, const uint64_t* moduli, size_t limbs,
                  uint64_t* out);

// The tables encode_slots uses: the DIF twiddles with the twist folded in (interleaved re, im;
// N entries, stage m at [m, 2m)) and the slot permutation (slot i -> evaluation index), for the
// device encoder, which repeats the same operations.
void encode_tables(size_t N, std::vector<double>& twiddles, std::vector<uint32_t>& perm);

// Calls of encode_slots so far and their summed wall time (ns).
void encode_stats(uint64_t* calls, uint64_t* ns);

}  // namespace host
}  // namespace wg
