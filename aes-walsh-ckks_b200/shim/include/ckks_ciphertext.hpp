// Ciphertexts and plaintexts of the reference API (src/ckks/ciphertext/ckks_ciphertext.hpp) with
// the residues kept in device memory.
//
// A CKKSCiphertext owns one device allocation holding its polynomials ([poly][level+1][N]
// uint64 residues, evaluation form), is move-only with an explicit clone(), and carries the
// reference's scale / level / secret-owner / encoding-state labels.  The host accessors
// (getA, getB, getPoly and their mutable forms) download the residues on first use into a
// host copy; after a mutable host access the next device use uploads the host copy again.
// Circuits of this build read and write the device copy directly.
#ifndef CKKS_CIPHERTEXT_HPP
#define CKKS_CIPHERTEXT_HPP

#include <cstddef>
#include <cstdint>
#include <memory>

#include "aligned_vector.hpp"

enum class CKKSSecretOwner {
    Dense,
    BootstrapSparse,
};

enum class CKKSMessageEncodingState {
    Slots,
    Coefficients,
};

class CKKSCiphertext {
public:
    CKKSCiphertext(size_t N, MyVector<uint64_t> a, MyVector<uint64_t> b, long double scale, size_t level,
                   CKKSSecretOwner secret_owner = CKKSSecretOwner::Dense,
                   CKKSMessageEncodingState message_encoding_state = CKKSMessageEncodingState::Slots);
    CKKSCiphertext(size_t N, MyVector<MyVector<uint64_t>> polys, long double scale, size_t level,
                   CKKSSecretOwner secret_owner = CKKSSecretOwner::Dense,
                   CKKSMessageEncodingState message_encoding_state = CKKSMessageEncodingState::Slots);

    CKKSCiphertext(const CKKSCiphertext&) = delete;
    CKKSCiphertext& operator=(const CKKSCiphertext&) = delete;
    CKKSCiphertext(CKKSCiphertext&&) noexcept;
    CKKSCiphertext& operator=(CKKSCiphertext&&) noexcept;
    ~CKKSCiphertext();

    CKKSCiphertext clone() const;

    long double getScale() const;
    size_t getLevel() const;
    size_t getN() const;
    size_t getNumPolys() const;
    CKKSSecretOwner getSecretOwner() const;
    CKKSMessageEncodingState getMessageEncodingState() const;

    const MyVector<uint64_t>& getA() const;
    const MyVector<uint64_t>& getB() const;
    MyVector<uint64_t>& getAMutable();
    MyVector<uint64_t>& getBMutable();
    const MyVector<uint64_t>& getPoly(size_t idx) const;
    MyVector<uint64_t>& getPolyMutable(size_t idx);
    MyVector<MyVector<uint64_t>>& getPolysMutable();
    void addPoly(MyVector<uint64_t> poly);
    void setScale(long double new_scale);
    void setLevel(size_t new_level);
    void setSecretOwner(CKKSSecretOwner new_secret_owner);
    void setMessageEncodingState(CKKSMessageEncodingState new_message_encoding_state);

    // Device storage (this build): `polys` polynomials of `capacity_limbs` limbs each, laid out
    // [poly][limb][N]; a ciphertext made by a circuit keeps room for the parameter set's top
    // level.  The pointers stay valid until the ciphertext is destroyed or moved from.
    struct Device;
    CKKSCiphertext(size_t N, long double scale, size_t level, size_t polys, size_t capacity_limbs,
                   CKKSSecretOwner secret_owner = CKKSSecretOwner::Dense,
                   CKKSMessageEncodingState message_encoding_state = CKKSMessageEncodingState::Slots);
    uint64_t* devicePoly(size_t idx);              // uploads a pending host copy first
    const uint64_t* devicePoly(size_t idx) const;  // likewise
    size_t deviceCapacityLimbs() const;
    void markDeviceWritten();                      // a device write invalidates the host copy

private:
    size_t N = 0;
    long double scale = 0.0L;
    size_t level = 0;
    CKKSSecretOwner secret_owner = CKKSSecretOwner::Dense;
    CKKSMessageEncodingState message_encoding_state = CKKSMessageEncodingState::Slots;
    std::unique_ptr<Device> dev;
    void syncHost() const;
    void syncDevice() const;
};

class CKKSEncoding {
public:
    CKKSEncoding(size_t N, MyVector<uint64_t> plaintext, long double scale, size_t level, bool montgomery_form = false);
    CKKSEncoding(const CKKSEncoding&) = delete;
    CKKSEncoding& operator=(const CKKSEncoding&) = delete;
    CKKSEncoding(CKKSEncoding&&) noexcept = default;
    CKKSEncoding& operator=(CKKSEncoding&&) noexcept = default;
    ~CKKSEncoding() = default;

    const MyVector<uint64_t>& getPlaintext() const;
    bool isMontgomeryForm() const;
    long double getScale() const;
    size_t getLevel() const;
    size_t getN() const;

private:
    size_t N;
    long double scale;
    size_t level;
    MyVector<uint64_t> plaintext;
    bool montgomery_form = false;
};

#endif  // CKKS_CIPHERTEXT_HPP
