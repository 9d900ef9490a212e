// Device-backed CKKSCiphertext and host CKKSEncoding of the reference API.
#include <cuda_runtime.h>

#include <cstring>
#include <stdexcept>
#include <string>

#include "ckks_ciphertext.hpp"

struct CKKSCiphertext::Device {
    uint64_t* d = nullptr;     // [poly][cap][N]
    size_t polys = 0, cap = 0, N = 0;
    // host copy ([poly][(level + 1) N]) and which side is current
    MyVector<MyVector<uint64_t>> host;
    bool host_valid = false;   // host copy equals the device words
    bool host_dirty = false;   // host copy written; device must be refreshed before its next use
    ~Device() {
        if (d) cudaFree(d);
    }
};

namespace {

uint64_t* device_alloc(size_t words) {
    void* p = nullptr;
    if (cudaMalloc(&p, words * 8) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("CKKSCiphertext: device allocation failed");
    }
    return static_cast<uint64_t*>(p);
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CKKSCiphertext: ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace

CKKSCiphertext::CKKSCiphertext(size_t n, MyVector<uint64_t> a, MyVector<uint64_t> b, long double sc, size_t lv,
                               CKKSSecretOwner owner, CKKSMessageEncodingState st) {
    MyVector<MyVector<uint64_t>> polys;
    polys.emplace_back(std::move(b));  // poly 0 is the constant term b
    polys.emplace_back(std::move(a));
    *this = CKKSCiphertext(n, std::move(polys), sc, lv, owner, st);
}

CKKSCiphertext::CKKSCiphertext(size_t n, MyVector<MyVector<uint64_t>> polys, long double sc, size_t lv,
                               CKKSSecretOwner owner, CKKSMessageEncodingState st)
    : N(n), scale(sc), level(lv), secret_owner(owner), message_encoding_state(st), dev(new Device) {
    if (polys.empty()) throw std::invalid_argument("CKKSCiphertext: no polynomials");
    const size_t words = (lv + 1) * n;
    for (const auto& p : polys)
        if (p.size() != words) throw std::invalid_argument("CKKSCiphertext: polynomial size does not match the level");
    dev->N = n;
    dev->polys = polys.size();
    dev->cap = lv + 1;
    dev->d = device_alloc(dev->polys * words);
    dev->host = std::move(polys);
    dev->host_valid = true;
    dev->host_dirty = true;
}

CKKSCiphertext::CKKSCiphertext(size_t n, long double sc, size_t lv, size_t polys, size_t cap, CKKSSecretOwner owner,
                               CKKSMessageEncodingState st)
    : N(n), scale(sc), level(lv), secret_owner(owner), message_encoding_state(st), dev(new Device) {
    if (cap < lv + 1 || polys == 0) throw std::invalid_argument("CKKSCiphertext: capacity below the level");
    dev->N = n;
    dev->polys = polys;
    dev->cap = cap;
    dev->d = device_alloc(polys * cap * n);
}

CKKSCiphertext::CKKSCiphertext(CKKSCiphertext&&) noexcept = default;
CKKSCiphertext& CKKSCiphertext::operator=(CKKSCiphertext&&) noexcept = default;
CKKSCiphertext::~CKKSCiphertext() = default;

void CKKSCiphertext::syncHost() const {
    if (dev->host_valid) return;
    const size_t words = (level + 1) * N;
    dev->host.assign(dev->polys, MyVector<uint64_t>(words));
    for (size_t p = 0; p < dev->polys; ++p)
        check(cudaMemcpy(dev->host[p].data(), dev->d + p * dev->cap * N, words * 8, cudaMemcpyDeviceToHost), "download");
    dev->host_valid = true;
    dev->host_dirty = false;
}

void CKKSCiphertext::syncDevice() const {
    if (!dev->host_dirty) return;
    if (dev->host.size() > dev->polys) {
        // polynomials were added on the host: grow the device store
        uint64_t* d = device_alloc(dev->host.size() * dev->cap * N);
        cudaFree(dev->d);
        dev->d = d;
        dev->polys = dev->host.size();
    }
    const size_t words = (level + 1) * N;
    for (size_t p = 0; p < dev->host.size(); ++p) {
        if (dev->host[p].size() != words) throw std::invalid_argument("CKKSCiphertext: polynomial size does not match the level");
        if (level + 1 > dev->cap) throw std::invalid_argument("CKKSCiphertext: level above the device capacity");
        check(cudaMemcpy(dev->d + p * dev->cap * N, dev->host[p].data(), words * 8, cudaMemcpyHostToDevice), "upload");
    }
    dev->host_dirty = false;
}

CKKSCiphertext CKKSCiphertext::clone() const {
    CKKSCiphertext c(N, scale, level, dev->polys, dev->cap, secret_owner, message_encoding_state);
    syncDevice();
    check(cudaMemcpy(c.dev->d, dev->d, dev->polys * dev->cap * N * 8, cudaMemcpyDeviceToDevice), "clone");
    return c;
}

long double CKKSCiphertext::getScale() const { return scale; }
size_t CKKSCiphertext::getLevel() const { return level; }
size_t CKKSCiphertext::getN() const { return N; }
size_t CKKSCiphertext::getNumPolys() const { return dev->host_dirty ? dev->host.size() : dev->polys; }
CKKSSecretOwner CKKSCiphertext::getSecretOwner() const { return secret_owner; }
CKKSMessageEncodingState CKKSCiphertext::getMessageEncodingState() const { return message_encoding_state; }

const MyVector<uint64_t>& CKKSCiphertext::getPoly(size_t idx) const {
    syncHost();
    if (idx >= dev->host.size()) throw std::runtime_error("CKKSCiphertext: missing polynomial");
    return dev->host[idx];
}
MyVector<uint64_t>& CKKSCiphertext::getPolyMutable(size_t idx) {
    syncHost();
    if (idx >= dev->host.size()) throw std::runtime_error("CKKSCiphertext: missing polynomial");
    dev->host_dirty = true;
    return dev->host[idx];
}
const MyVector<uint64_t>& CKKSCiphertext::getA() const { return getPoly(1); }
const MyVector<uint64_t>& CKKSCiphertext::getB() const { return getPoly(0); }
MyVector<uint64_t>& CKKSCiphertext::getAMutable() { return getPolyMutable(1); }
MyVector<uint64_t>& CKKSCiphertext::getBMutable() { return getPolyMutable(0); }
MyVector<MyVector<uint64_t>>& CKKSCiphertext::getPolysMutable() {
    syncHost();
    dev->host_dirty = true;
    return dev->host;
}
void CKKSCiphertext::addPoly(MyVector<uint64_t> poly) {
    syncHost();
    dev->host.push_back(std::move(poly));
    dev->host_dirty = true;
}
void CKKSCiphertext::setScale(long double s) { scale = s; }
void CKKSCiphertext::setLevel(size_t l) {
    if (dev->host_valid && l != level) {
        syncDevice();
        dev->host_valid = false;
    }
    level = l;
}
void CKKSCiphertext::setSecretOwner(CKKSSecretOwner o) { secret_owner = o; }
void CKKSCiphertext::setMessageEncodingState(CKKSMessageEncodingState s) { message_encoding_state = s; }

uint64_t* CKKSCiphertext::devicePoly(size_t idx) {
    syncDevice();
    if (idx >= dev->polys) throw std::runtime_error("CKKSCiphertext: missing polynomial");
    return dev->d + idx * dev->cap * N;
}
const uint64_t* CKKSCiphertext::devicePoly(size_t idx) const {
    syncDevice();
    if (idx >= dev->polys) throw std::runtime_error("CKKSCiphertext: missing polynomial");
    return dev->d + idx * dev->cap * N;
}
size_t CKKSCiphertext::deviceCapacityLimbs() const { return dev->cap; }
void CKKSCiphertext::markDeviceWritten() {
    dev->host_valid = false;
    dev->host_dirty = false;
}

CKKSEncoding::CKKSEncoding(size_t n, MyVector<uint64_t> pt, long double sc, size_t lv, bool mont)
    : N(n), scale(sc), level(lv), plaintext(std::move(pt)), montgomery_form(mont) {}
const MyVector<uint64_t>& CKKSEncoding::getPlaintext() const { return plaintext; }
bool CKKSEncoding::isMontgomeryForm() const { return montgomery_form; }
long double CKKSEncoding::getScale() const { return scale; }
size_t CKKSEncoding::getLevel() const { return level; }
size_t CKKSEncoding::getN() const { return N; }
