// Prints the modulus chains, P moduli, scale and depth of the reference-API presets as built by
// the device library's reference-API layer (libckks_b200.so), one JSON object per line, for the
// CPU test that compares them with the reference's own CKKSParams presets.
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "ckks_aes_params.hpp"
#include "ckks_params.hpp"

int main() {
    const std::vector<std::pair<std::string, std::function<CKKSParams()>>> presets = {
        {"walsh15", [] { return CKKSParams::AESWalsh15(); }},
        {"xboot13", [] { return CKKSParams::XBootParamAes13Reference(); }},
        {"xboot14", [] { return CKKSParams::AESXBoot14Secure(); }},
        {"xboot14-sparse", [] { return CKKSParams::AESXBoot14SecureSparse1024(); }},
        {"xboot15", [] { return CKKSParams::AESXBoot15(); }},
        {"xboot15-sparse", [] { return CKKSParams::AESXBoot15Sparse1024(); }},
    };
    for (const auto& [name, make] : presets) {
        const CKKSParams p = make();
        std::printf("{\"name\": \"%s\", \"q\": [", name.c_str());
        for (size_t i = 0; i < p.getModuli().size(); ++i)
            std::printf("%s%llu", i ? ", " : "", (unsigned long long)p.getModuli()[i]);
        std::printf("], \"p\": [");
        for (size_t i = 0; i < p.getPModuli().size(); ++i)
            std::printf("%s%llu", i ? ", " : "", (unsigned long long)p.getPModuli()[i]);
        std::printf("], \"scale\": %.17g, \"depth\": %zu, \"active\": %zu, \"k\": %zu, \"s2c\": %zu, \"c2s\": %zu}\n",
                    p.getScale(), p.getDepth(), p.getBootstrapActiveSlotCount(), p.getBootstrapEvalModK(),
                    p.getBootstrapS2CDepth(), p.getBootstrapC2SDepth());
    }
    return 0;
}
