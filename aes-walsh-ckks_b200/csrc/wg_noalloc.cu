// Rotation that allocates nothing: the key-switch scratch lives in a fixed static device array.
//
// Some callers cannot call cudaMalloc at the moment they need a rotation: an application whose
// device memory was reserved up front by another allocator (a serving engine that claims most
// of HBM at start-up), or latency-sensitive loops that must avoid the device-wide
// synchronisation cudaMalloc/cudaFree can cause.  wg_rotate_noalloc serves them: apart from the
// context's own tables and keys (allocated once at creation) it uses only the array below.
//
// Limits and sharing rules:
//   * the array holds kScratchWords 64-bit words (32 MiB); a switch needing more fails with
//     WG_ERR_INVALID.  Every GPU that loads the library keeps the array until the process exits;
//   * every call shares the one array and it keeps the last call's contents.  The switch writes
//     every scratch word it later reads, so nothing has to be cleared between calls;
//   * calls that overlap on the GPU (different streams, or concurrent host threads) race on the
//     array; serialise them.
//   * every call makes the context's device current and leaves it current;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current; make that first call before any stream capture.
#include <mutex>

#include "../../include/walsh_gpu.h"
#include "wg_internal.hpp"

namespace wg {
namespace {

constexpr size_t kScratchWords = size_t{4} << 20;  // 32 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint64_t g_rotation_scratch[kScratchWords];

std::mutex g_setup_mutex;
uint64_t* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device`, looked up once per device.  The caller has
// made `device` current; the lookup itself allocates nothing.
uint64_t* scratch_on(int device) {
    if (device < 0 || device >= kMaxDevices) fail(kInvalid, "rotate_noalloc: device index out of range");
    std::lock_guard<std::mutex> g(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        void* ptr = nullptr;
        check_cuda(cudaGetSymbolAddress(&ptr, g_rotation_scratch), "rotate_noalloc: cudaGetSymbolAddress");
        g_scratch_ptr[device] = static_cast<uint64_t*>(ptr);
    }
    return g_scratch_ptr[device];
}

}  // namespace
}  // namespace wg

extern "C" int wg_rotate_noalloc(wg_context* ctx, size_t level, uint64_t* b, uint64_t* a, int64_t rotation,
                                 void* stream);

extern "C" int wg_rotate_noalloc(wg_context* ctx, size_t level, uint64_t* b, uint64_t* a, int64_t rotation,
                                 void* stream) {
    try {
        if (!ctx || !ctx->c) wg::fail(wg::kInvalid, "rotate_noalloc: null context");
        wg::Context& c = *ctx->c;
        if (level >= c.nq) wg::fail(wg::kInvalid, "rotate_noalloc: invalid ciphertext level");
        if (!b || !a) wg::fail(wg::kInvalid, "rotate_noalloc: null buffer");
        const int64_t slots = (int64_t)(c.N / 2);
        int64_t r = rotation % slots;
        if (r < 0) r += slots;
        if (r == 0) return WG_OK;
        const size_t words = wg::keyswitch_workspace_words(c, level);
        if (words > wg::kScratchWords)
            wg::fail(wg::kInvalid, "rotate_noalloc: this level needs " + std::to_string(words * 8 >> 20) +
                                       " MiB of scratch, above the 32 MiB static array");
        const wg::KeyEntry& k = c.key(WG_KEY_ROTATION, r);
        // Every call makes the context's device current (and leaves it current, as the other
        // entry points do): the scratch address and the context's tables belong to that device.
        wg::check_cuda(cudaSetDevice(c.device), "rotate_noalloc: cudaSetDevice");
        uint64_t* scratch = wg::scratch_on(c.device);
        const uint64_t galois = wg::host::powmod(5, (uint64_t)r, 2 * c.N);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        wg::keyswitch(c, level, a, k, b, a, b, a, true, false, galois, scratch, s);
        wg::set_last_error("");
        return WG_OK;
    } catch (const wg::Error& e) {
        wg::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        wg::set_last_error(e.what());
        return WG_ERR_RUNTIME;
    }
}
