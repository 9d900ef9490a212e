// Optional host-time spans for locating host-side cost in the batched paths.  Compiled in only
// with -DWG_HOST_SPANS (the shipped library has none): each WG_SPAN("name") adds the wall time
// of its scope to a per-name total, read back by wg_host_spans() in such builds.
#pragma once

#ifdef WG_HOST_SPANS
#include <chrono>
#include <cstdint>

namespace wg {
void host_span_add(const char* name, uint64_t ns);

struct HostSpan {
    const char* name;
    std::chrono::steady_clock::time_point t0;
    explicit HostSpan(const char* n) : name(n), t0(std::chrono::steady_clock::now()) {}
    ~HostSpan() {
        host_span_add(name, (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                                std::chrono::steady_clock::now() - t0)
                                .count());
    }
};
}  // namespace wg

#define WG_SPAN_CAT2(a, b) a##b
#define WG_SPAN_CAT(a, b) WG_SPAN_CAT2(a, b)
#define WG_SPAN(name) ::wg::HostSpan WG_SPAN_CAT(wg_span_, __LINE__)(name)
#else
#define WG_SPAN(name) ((void)0)
#endif
