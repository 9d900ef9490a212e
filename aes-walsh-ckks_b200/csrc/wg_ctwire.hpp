// Ciphertext wire format (host-only): one ciphertext as a self-checking byte record, so
// ciphertexts can leave one process and enter another (a client's encryptions, a server's
// results).  No counterpart in the reference, which keeps ciphertexts in memory only.
//
// Layout, integers little-endian:
//   "WGC1" (4 bytes), version (u32) = 1
//   N, level, npolys (u64 each), scale (IEEE double), secret owner (u8: 0 dense, 1 sparse
//   bootstrap), encoding state (u8: 0 slots, 1 coefficients), 6 zero bytes
//   q[0 .. level] (u64): the moduli the residues are reduced by
//   residues [poly][level + 1][N] (u64), evaluation form
//   FNV-1a 64 of every preceding byte
// The reader checks the magic, version, sizes against the bytes given, that every residue is
// below its modulus, that the moduli are the receiving context's, and the checksum; any mismatch
// throws std::invalid_argument.
#pragma once
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "wg_bundle.hpp"

namespace wg {

struct CtRecord {
    uint64_t N = 0, level = 0, npolys = 0;
    double scale = 0.0;
    uint8_t owner = 0, state = 0;
    std::vector<uint64_t> q;      // level + 1 moduli
    std::vector<uint64_t> polys;  // npolys * (level + 1) * N residues
};

inline size_t ct_wire_bytes(uint64_t N, uint64_t level, uint64_t npolys) {
    return 4 + 4 + 3 * 8 + 8 + 8 + (level + 1) * 8 + npolys * (level + 1) * N * 8 + 8;
}

inline void ct_wire_encode(const CtRecord& r, uint8_t* out, size_t cap) {
    const size_t need = ct_wire_bytes(r.N, r.level, r.npolys);
    if (cap < need) throw std::invalid_argument("ciphertext wire: output buffer too small");
    if (r.q.size() != r.level + 1 || r.polys.size() != r.npolys * (r.level + 1) * r.N)
        throw std::invalid_argument("ciphertext wire: inconsistent record");
    uint8_t* p = out;
    auto put = [&](const void* s, size_t n) {
        std::memcpy(p, s, n);
        p += n;
    };
    const uint32_t version = 1;
    put("WGC1", 4);
    put(&version, 4);
    put(&r.N, 8);
    put(&r.level, 8);
    put(&r.npolys, 8);
    put(&r.scale, 8);
    const uint8_t flags[8] = {r.owner, r.state, 0, 0, 0, 0, 0, 0};
    put(flags, 8);
    put(r.q.data(), r.q.size() * 8);
    put(r.polys.data(), r.polys.size() * 8);
    const uint64_t h = bundle_fnv1a(out, (size_t)(p - out));
    put(&h, 8);
}

inline CtRecord ct_wire_decode(const uint8_t* in, size_t len) {
    auto bad = [](const char* m) { throw std::invalid_argument(std::string("ciphertext wire: ") + m); };
    if (len < 4 + 4 + 3 * 8 + 16 + 8) bad("record too short");
    if (std::memcmp(in, "WGC1", 4) != 0) bad("not a ciphertext record");
    uint32_t version;
    std::memcpy(&version, in + 4, 4);
    if (version != 1) bad("unsupported version");
    CtRecord r;
    std::memcpy(&r.N, in + 8, 8);
    std::memcpy(&r.level, in + 16, 8);
    std::memcpy(&r.npolys, in + 24, 8);
    std::memcpy(&r.scale, in + 32, 8);
    r.owner = in[40];
    r.state = in[41];
    if (r.N == 0 || r.N > (uint64_t{1} << 17) || (r.N & (r.N - 1))) bad("invalid ring degree");
    if (r.level > 256 || r.npolys == 0 || r.npolys > 3) bad("invalid level or polynomial count");
    if (r.owner > 1 || r.state > 1) bad("invalid labels");
    if (len != ct_wire_bytes(r.N, r.level, r.npolys)) bad("length does not match the header");
    uint64_t h;
    std::memcpy(&h, in + len - 8, 8);
    if (bundle_fnv1a(in, len - 8) != h) bad("checksum mismatch");
    const uint8_t* p = in + 48;
    r.q.resize(r.level + 1);
    std::memcpy(r.q.data(), p, r.q.size() * 8);
    p += r.q.size() * 8;
    r.polys.resize(r.npolys * (r.level + 1) * r.N);
    std::memcpy(r.polys.data(), p, r.polys.size() * 8);
    for (uint64_t k = 0; k < r.npolys; ++k)
        for (uint64_t l = 0; l <= r.level; ++l) {
            const uint64_t* x = r.polys.data() + (k * (r.level + 1) + l) * r.N;
            for (uint64_t i = 0; i < r.N; ++i)
                if (x[i] >= r.q[l]) bad("residue not below its modulus");
        }
    return r;
}

}  // namespace wg
