// ckks_decrypt of the reference API, decrypted and decoded on the device.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "ckks_encoding.hpp"
#include "context_engine.hpp"

MyVector<Complex> ckks_decrypt(const CKKSContext& context, const CKKSCiphertext& ct, CKKSDecryptDomain domain,
                               bool use_low_secret) {
    if (domain != CKKSDecryptDomain::Slots)
        throw std::invalid_argument("ckks_decrypt: only slot-domain decryption is provided by this build");
    CKKSContext::Engine& e = context.engine();
    const bool low = use_low_secret || ct.getSecretOwner() == CKKSSecretOwner::BootstrapSparse;
    const std::vector<int8_t>& s = low ? e.low_secret : e.secret;
    if (s.empty()) throw std::runtime_error("ckks_decrypt: sparse bootstrap secret key is unavailable");
    const size_t half = e.params.getN() / 2;
    if (ct.getNumPolys() < 2 || ct.getNumPolys() > 3)
        throw std::invalid_argument("ckks_decrypt: ciphertext must have two or three polynomials");
    std::vector<double> re(half), im(half);
    const double scale = (double)ct.getScale();
    const uint64_t* b = ct.devicePoly(0);
    const uint64_t* a = ct.devicePoly(1);
    const uint64_t* c2 = ct.getNumPolys() == 3 ? ct.devicePoly(2) : nullptr;
    const int rc = wg_decrypt_decode(e.ctx, 1, ct.getLevel(), &scale, &b, &a, c2 ? &c2 : nullptr, s.data(), re.data(),
                                     im.data(), nullptr);
    if (rc != WG_OK) throw std::runtime_error(std::string("ckks_decrypt: ") + wg_last_error());
    MyVector<Complex> out(half);
    for (size_t i = 0; i < half; ++i) out[i] = Complex(re[i], im[i]);
    return out;
}
