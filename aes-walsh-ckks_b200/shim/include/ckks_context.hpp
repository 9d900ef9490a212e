// The CKKS context of the reference API (src/ckks/context/ckks_context.hpp), built on the device.
//
// The constructor does what the reference's does for a bootstrapping AES parameter set, with
// the device library doing the work: the modulus chain and NTT tables (wg_ctx_create), the
// EvalMod series (wg_evalmod_fit), the SlotToCoeff / CoeffToSlot plans (wg_dft_plan_create),
// a dense secret of the configured Hamming weight and the sparse bootstrapping secret (drawn
// from the operating system's random source), and every switching key its bootstraps and AES
// circuits use (wg_keygen_switch_key, wg_keygen_secret_switch), generated and kept on the
// device.  Secrets stay in host memory (decryption and key generation use them).
//
// Interface: the reference's accessors that code outside the library needs (parameters, key
// availability and counts, the EvalMod polynomial); the reference's accessors that hand out
// host copies of tables and keys (twiddles, ModUp precomputation, key ciphertexts) are not
// provided, because those live on the device here.
#ifndef CKKS_CONTEXT_HPP
#define CKKS_CONTEXT_HPP

#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>

#include "aligned_vector.hpp"
#include "ckks_ciphertext.hpp"
#include "ckks_params.hpp"
#include "poly_approx.hpp"

using Complex = std::complex<double>;

enum class CKKSDecryptDomain {
    Slots,
    Coefficients,
};

class CKKSContext {
public:
    CKKSContext(CKKSParams ckks_params);
    ~CKKSContext();
    CKKSContext(const CKKSContext&) = delete;
    CKKSContext& operator=(const CKKSContext&) = delete;
    CKKSContext(CKKSContext&&) noexcept;
    CKKSContext& operator=(CKKSContext&&) noexcept;

    const CKKSParams& getParams() const;
    bool hasSparseSecretEncapsulationKeys() const;
    bool hasConjugationKey() const;
    size_t getRotationKeyCount() const;
    bool hasRotationKey(int64_t rotation) const;
    bool hasEvalModBootstrapDftPlans() const;
    double getEvalModScaledC2STransformScale() const;
    const PolynomialApproximation& getEvalModPolynomial() const;

    // The device engine behind this context (this build's circuits and decryption use it).
    struct Engine;
    Engine& engine() const;

private:
    std::unique_ptr<Engine> eng;
};

#endif  // CKKS_CONTEXT_HPP
