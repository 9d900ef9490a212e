// A file format for a context's switching keys and linear-transform plans, so that a server
// loads them instead of regenerating them (host-only; wg_capi.cu moves the payloads to and from
// the device).  No counterpart in the reference, which builds keys and plans in its context
// constructor every time.
//
// Layout, all integers little-endian 64-bit words unless noted:
//   "WGB1" (4 bytes), version (u32) = 1
//   N, dnum, nq, np, q[nq], p[np]
//   key count; per key: kind, rotation (i64), parts, key_level, words, data[words]
//   stage count; per stage: level, baby, slots, rescale, nterms, indices[nterms], words, diagonals[words]
//   FNV-1a 64 of every preceding byte
// The reader checks the magic, the version, every length against the bytes left, and the
// checksum, and throws std::invalid_argument on any mismatch.
#pragma once
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace wg {

struct BundleKey {
    int64_t kind = 0, rotation = 0;
    uint64_t parts = 0, key_level = 0;
    std::vector<uint64_t> data;
};

struct BundleStage {
    uint64_t level = 0, baby = 0, slots = 0, rescale = 0;
    std::vector<uint64_t> indices, diagonals;
};

struct Bundle {
    uint64_t N = 0, dnum = 0;
    std::vector<uint64_t> q, p;
    std::vector<BundleKey> keys;
    std::vector<BundleStage> stages;
};

inline uint64_t bundle_fnv1a(const uint8_t* d, size_t n) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= d[i];
        h *= 0x100000001b3ull;
    }
    return h;
}

inline std::vector<uint8_t> bundle_encode(const Bundle& b) {
    std::vector<uint8_t> out;
    auto put = [&](const void* p, size_t n) {
        const auto* c = static_cast<const uint8_t*>(p);
        out.insert(out.end(), c, c + n);
    };
    auto word = [&](uint64_t v) { put(&v, 8); };
    auto words = [&](const std::vector<uint64_t>& v) {
        word(v.size());
        if (!v.empty()) put(v.data(), v.size() * 8);
    };
    put("WGB1", 4);
    const uint32_t version = 1;
    put(&version, 4);
    word(b.N);
    word(b.dnum);
    words(b.q);
    words(b.p);
    word(b.keys.size());
    for (const auto& k : b.keys) {
        word((uint64_t)k.kind);
        word((uint64_t)k.rotation);
        word(k.parts);
        word(k.key_level);
        words(k.data);
    }
    word(b.stages.size());
    for (const auto& s : b.stages) {
        word(s.level);
        word(s.baby);
        word(s.slots);
        word(s.rescale);
        words(s.indices);
        words(s.diagonals);
    }
    word(bundle_fnv1a(out.data(), out.size()));
    return out;
}

inline Bundle bundle_decode(const uint8_t* d, size_t n) {
    if (n < 16 || std::memcmp(d, "WGB1", 4) != 0) throw std::invalid_argument("wg_bundle: not a bundle file");
    uint32_t version = 0;
    std::memcpy(&version, d + 4, 4);
    if (version != 1) throw std::invalid_argument("wg_bundle: unsupported bundle version");
    uint64_t stored = 0;
    std::memcpy(&stored, d + n - 8, 8);
    if (bundle_fnv1a(d, n - 8) != stored) throw std::invalid_argument("wg_bundle: checksum mismatch");
    size_t pos = 8;
    const size_t end = n - 8;
    auto word = [&]() {
        if (end - pos < 8) throw std::invalid_argument("wg_bundle: truncated bundle");
        uint64_t v;
        std::memcpy(&v, d + pos, 8);
        pos += 8;
        return v;
    };
    auto words = [&]() {
        const uint64_t count = word();
        if (count > (end - pos) / 8) throw std::invalid_argument("wg_bundle: truncated bundle");
        std::vector<uint64_t> v(count);
        if (count) std::memcpy(v.data(), d + pos, count * 8);
        pos += count * 8;
        return v;
    };
    Bundle b;
    b.N = word();
    b.dnum = word();
    b.q = words();
    b.p = words();
    const uint64_t nkeys = word();
    if (nkeys > (end - pos) / 40) throw std::invalid_argument("wg_bundle: truncated bundle");
    for (uint64_t i = 0; i < nkeys; ++i) {
        BundleKey k;
        k.kind = (int64_t)word();
        k.rotation = (int64_t)word();
        k.parts = word();
        k.key_level = word();
        k.data = words();
        b.keys.push_back(std::move(k));
    }
    const uint64_t nstages = word();
    if (nstages > (end - pos) / 48) throw std::invalid_argument("wg_bundle: truncated bundle");
    for (uint64_t i = 0; i < nstages; ++i) {
        BundleStage s;
        s.level = word();
        s.baby = word();
        s.slots = word();
        s.rescale = word();
        s.indices = words();
        s.diagonals = words();
        b.stages.push_back(std::move(s));
    }
    if (pos != end) throw std::invalid_argument("wg_bundle: trailing bytes");
    return b;
}

}  // namespace wg
