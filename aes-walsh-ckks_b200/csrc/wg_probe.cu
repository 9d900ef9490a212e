// Launch counting and optional CUDA-event timing of one kernel class (see Probe in
// wg_internal.hpp).  Timing is off unless wg_probe_begin() enables it; counting is always on.
#include <atomic>
#include <mutex>
#include <vector>

#include "../../include/walsh_gpu.h"
#include "wg_encode.hpp"
#include "wg_internal.hpp"

namespace wg {
namespace {

constexpr int kMaxEvents = 1 << 16;

struct ProbeState {
    std::mutex mu;
    std::atomic<uint64_t> launches[kClsCount] = {};
    int timed_class = -1;
    std::vector<cudaEvent_t> begin, end;
    std::vector<double> bytes;
    int used = 0;
};

ProbeState& state() {
    static ProbeState s;
    return s;
}

}  // namespace

Probe::Probe(int cls, double nbytes, cudaStream_t s) : stream(s) {
    ProbeState& st = state();
    st.launches[cls].fetch_add(1, std::memory_order_relaxed);
    if (st.timed_class != cls) return;
    std::lock_guard<std::mutex> g(st.mu);
    if (st.used >= (int)st.begin.size()) return;
    slot = st.used++;
    st.bytes[slot] = nbytes;
    cudaEventRecord(st.begin[slot], s);
}

Probe::~Probe() {
    if (slot >= 0) cudaEventRecord(state().end[slot], stream);
}

void probe_counts(uint64_t* out) {
    for (int i = 0; i < kClsCount; ++i) out[i] = state().launches[i].load();
}

void probe_add(const uint64_t* counts) {
    for (int i = 0; i < kClsCount; ++i) state().launches[i].fetch_add(counts[i], std::memory_order_relaxed);
}

}  // namespace wg

#ifdef WG_HOST_SPANS
#include <cstdio>
#include <map>
#include <string>
namespace wg {
namespace {
std::mutex g_span_mu;
std::map<std::string, std::pair<uint64_t, uint64_t>> g_spans;  // name -> (count, ns)
}  // namespace
void host_span_add(const char* name, uint64_t ns) {
    std::lock_guard<std::mutex> g(g_span_mu);
    auto& e = g_spans[name];
    e.first += 1;
    e.second += ns;
}
}  // namespace wg
extern "C" int wg_host_spans(char* buf, size_t n) {
    std::lock_guard<std::mutex> g(wg::g_span_mu);
    std::string out;
    for (const auto& kv : wg::g_spans) {
        char line[256];
        std::snprintf(line, sizeof line, "%s %llu %.3f\n", kv.first.c_str(), (unsigned long long)kv.second.first,
                      kv.second.second / 1e6);
        out += line;
    }
    wg::g_spans.clear();
    std::snprintf(buf, n, "%s", out.c_str());
    return 0;
}
#endif

extern "C" {

int wg_host_stats(uint64_t* out, size_t n) {
    if (!out) return WG_ERR_INVALID;
    uint64_t v[5] = {};
    wg::host::encode_stats(&v[0], &v[1]);
    wg::stage_stats(&v[2], &v[3], &v[4]);
    for (size_t i = 0; i < n && i < 5; ++i) out[i] = v[i];
    return WG_OK;
}

uint64_t wg_launch_count(int kernel_class) {
    auto& st = wg::state();
    if (kernel_class < 0) {
        uint64_t t = 0;
        for (int i = 0; i < wg::kClsCount; ++i) t += st.launches[i].load();
        return t;
    }
    if (kernel_class >= wg::kClsCount) return 0;
    return st.launches[kernel_class].load();
}

int wg_probe_begin(int kernel_class, int max_launches) {
    auto& st = wg::state();
    std::lock_guard<std::mutex> g(st.mu);
    if (kernel_class < 0 || kernel_class >= wg::kClsCount) return WG_ERR_INVALID;
    if (max_launches <= 0 || max_launches > wg::kMaxEvents) return WG_ERR_INVALID;
    for (auto e : st.begin) cudaEventDestroy(e);
    for (auto e : st.end) cudaEventDestroy(e);
    st.begin.assign(max_launches, nullptr);
    st.end.assign(max_launches, nullptr);
    st.bytes.assign(max_launches, 0.0);
    for (int i = 0; i < max_launches; ++i) {
        if (cudaEventCreate(&st.begin[i]) != cudaSuccess || cudaEventCreate(&st.end[i]) != cudaSuccess)
            return WG_ERR_CUDA;
    }
    st.used = 0;
    st.timed_class = kernel_class;
    return WG_OK;
}

int wg_probe_end(uint64_t* launches, double* total_ms, double* total_bytes) {
    auto& st = wg::state();
    std::lock_guard<std::mutex> g(st.mu);
    st.timed_class = -1;
    double ms = 0, by = 0;
    for (int i = 0; i < st.used; ++i) {
        if (cudaEventSynchronize(st.end[i]) != cudaSuccess) return WG_ERR_CUDA;
        float t = 0;
        if (cudaEventElapsedTime(&t, st.begin[i], st.end[i]) != cudaSuccess) return WG_ERR_CUDA;
        ms += t;
        by += st.bytes[i];
    }
    if (launches) *launches = (uint64_t)st.used;
    if (total_ms) *total_ms = ms;
    if (total_bytes) *total_bytes = by;
    st.used = 0;
    return WG_OK;
}

}  // extern "C"
