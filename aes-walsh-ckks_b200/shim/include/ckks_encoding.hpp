// Decryption of the reference API (src/ckks/encoding/ckks_encoding.hpp), on the device.
#ifndef CKKS_ENCODING_HPP
#define CKKS_ENCODING_HPP

#include <complex>
#include <cstddef>

#include "aligned_vector.hpp"
#include "ckks_ciphertext.hpp"
#include "ckks_context.hpp"

using Complex = std::complex<double>;

// The N/2 slot values of `ct` under the context's secret (the sparse bootstrapping secret when
// use_low_secret or when the ciphertext is labelled with it), decrypted and decoded on the
// device (wg_decrypt_decode): equal to the reference's to FP64 rounding.  Only the Slots domain
// is provided; Coefficients throws std::invalid_argument.
MyVector<Complex> ckks_decrypt(const CKKSContext& context, const CKKSCiphertext& ct,
                               CKKSDecryptDomain domain = CKKSDecryptDomain::Slots, bool use_low_secret = false);

#endif  // CKKS_ENCODING_HPP
