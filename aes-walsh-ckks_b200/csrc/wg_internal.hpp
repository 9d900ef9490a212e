// Internal declarations shared by the device library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <deque>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>

#include "wg_hostspan.hpp"
#include <vector>

#include "wg_arith.cuh"
#include "wg_ntt.cuh"

namespace wg {

// Status codes of the C ABI (walsh_gpu.h): invalid arguments mirror the reference's
// std::invalid_argument, missing keys or precomputed material its std::runtime_error.
enum Status : int { kOk = 0, kInvalid = -1, kRuntime = -2, kCuda = -3, kNoMemory = -4 };

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] inline void fail(int code, const std::string& m) { throw Error(code, m); }
// Message returned by wg_last_error() for the calling thread (wg_capi.cu).
void set_last_error(const std::string& m);
inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(kCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------
// Host-side precomputation (wg_host.cpp).  Restates the reference's context-build math.
// ---------------------------------------------------------------------------------------
namespace host {
uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m);
uint64_t powmod(uint64_t a, uint64_t e, uint64_t m);
uint64_t inverse(uint64_t a, uint64_t m);
uint64_t shoup(uint64_t w, uint64_t q);
void barrett_const(uint64_t q, uint64_t& lo, uint64_t& hi);
uint64_t barrett_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t lo, uint64_t hi);
uint64_t mont_neg_inv(uint64_t q);
void find_primes(const std::vector<uint64_t>& p_bits, const std::vector<uint64_t>& q_bits,
                 uint64_t N, std::vector<uint64_t>& p, std::vector<uint64_t>& q);
// Twiddles: fwd, fwd_shoup, inv, inv_shoup (N entries each), N^-1.
void ntt_tables(uint64_t N, uint64_t q, uint64_t* fwd, uint64_t* fwd_s, uint64_t* inv,
                uint64_t* inv_s, uint64_t& n_inv);
}  // namespace host

// ---------------------------------------------------------------------------------------
// Device-side descriptors.
// ---------------------------------------------------------------------------------------

// Base change Q-digit -> (other Q limbs, P limbs) for one (level, digit); arrays in device
// memory, row-major [dst][src] like the reference's ApproxCrtModUpPrecomp.
struct ModUpDesc {
    int src_count;
    int dst_count;
    int src_first;             // first Q limb of the digit
    int pad;
    const uint64_t* qhat_inv;  // [src]
    const uint64_t* qhat_inv_s;
    const double* src_inv;     // [src]
    const uint64_t* qhat;      // [dst][src]
    const uint64_t* qhat_s;
    const uint64_t* corr;      // [dst][src+1]
    const int* dst_limb;       // QP limb index written for each dst
    const int* dst_mod;        // modulus index (into Context::d_mod) for each dst
};

struct KeyEntry {
    uint64_t* d_data = nullptr;  // [part][a|b][key_level+1+K][N], Montgomery, folded
    size_t parts = 0;
    size_t key_level = 0;
};

struct Workspace {
    uint64_t* base = nullptr;
    size_t words = 0;
};

struct Context;
// Staging uploads so far: calls, bytes and the time spent waiting for ring space.
void stage_stats(uint64_t* calls, uint64_t* bytes, uint64_t* wait_ns);

// Per-stream buffers of the batched path: the job-table image (pinned stage + device copy)
// and a scratch arena, both grown on demand outside stream capture.
// Per-stream buffers of the batched paths.  Host-to-device staging (job tables, public
// plaintexts) goes through a ring: a pinned host buffer mirrored by a device buffer, filled
// front to back; each upload records an event, and a region is rewritten only after the
// upload that last used it has completed, so the host runs ahead of the device instead of
// waiting for every copy.  Device-side reuse is safe in stream order: a later copy into a
// region executes after every kernel queued before it on the same stream.
struct BatchBuffers {
    struct Flight {
        size_t begin, end;
        cudaEvent_t done;
    };
    unsigned char* d_ring = nullptr;
    unsigned char* h_ring = nullptr;
    size_t ring_bytes = 0;
    size_t head = 0;
    std::deque<Flight> flights;
    std::vector<cudaEvent_t> spare_events;
    uint64_t* d_arena = nullptr;
    size_t arena_words = 0;
    // Copy `bytes` of host data into the ring and onto the device (stream order); returns the
    // device address, valid for kernels queued on `s` before the ring wraps back over it.
    void* stage(const Context& c, const void* data, size_t bytes, cudaStream_t s);
    // The same in two steps, for callers that write the bytes in place: reserve() makes a
    // region of `bytes` free (waiting for old uploads as stage() does) and returns its offset;
    // the caller fills h_ring + offset; commit() uploads it and returns d_ring + offset.
    size_t reserve(const Context& c, size_t bytes, cudaStream_t s);
    void* commit(size_t offset, size_t bytes, cudaStream_t s);
    uint64_t* arena(const Context& c, size_t words, cudaStream_t s);
    void release();
};

// NTT geometries (wg_ntt.cu): 0 = 8 residues per thread, staged twiddles; 1 = 8, twiddles
// from the table; 2 = 16, staged; 3 = 16, from the table.  Device timings of each (ms, best of
// three over a scratch batch) per [direction: forward, inverse][phase: rows, columns].
constexpr int kNttGeometries = 4;
struct NttTuning {
    float ms[2][2][kNttGeometries];
    int chosen[2][2];
    int limbs;  // limbs of the timed batch
};

struct Context {
    int device = 0;
    uint64_t N = 0;
    int logN = 0;
    size_t nq = 0, np = 0, dnum = 0, alpha = 0;
    std::vector<uint64_t> q, p;
    std::vector<Modulus> mods;       // nq + np entries (P after Q)
    Modulus* d_mod = nullptr;
    uint64_t* d_tw = nullptr;        // [mod][2][N] (w, Shoup w) pairs: forward, inverse (ntt::TwPair)
    int ntt_variant[2][2] = {{0, 0}, {0, 0}};  // NTT geometry per [direction][phase: rows, columns]
    // Key switches and rescales can run their base changes fused with the adjacent NTT column
    // phases and their final element-wise steps in the last row phase's epilogue (wg_ksfuse.cu,
    // k_ntt_rows_epi).  0: always the separate launches; 1: fused when the launch fills the
    // device (fuse()); 2: always fused.  The words are the same in every mode.
    int ntt_fusion = 1;
    int sm_count = 148;  // multiprocessors of the device
    // Whether a step over `jobs` jobs runs fused: the fused kernels give one CTA of 128 threads
    // per (job, 1024-coefficient column tile) and hold several source tiles in shared memory, so
    // they only pay when the launch fills the device at least twice; smaller calls (a single
    // ciphertext) keep the separate, wider launches.
    bool fuse(size_t jobs) const {
        return ntt_fusion == 2 || (ntt_fusion == 1 && jobs * (N >= 1024 ? N / 1024 : 1) >= 2 * (size_t)sm_count);
    }
    NttTuning tuning{};
    // ModUp descriptors, host copies holding device pointers: [level][part]
    std::vector<std::vector<ModUpDesc>> modup;
    uint64_t* d_tables = nullptr;    // backing store for all small tables
    size_t tables_words = 0;
    // folded ModDown constants per level: [qi][pi] inverse and Shoup
    std::vector<const uint64_t*> fold_inv, fold_inv_s;
    const double* d_p_inv = nullptr; // [pi] 1.0 / p
    // rescale constants per dropped limb d: arrays of d entries (Shoup of 1, p^-1 and its
    // Shoup companion, floor(p/2) mod q_i)
    std::vector<const uint64_t*> rs_one_s, rs_inv_p, rs_inv_p_s, rs_half;
    std::map<std::pair<int, int64_t>, KeyEntry> keys;
    std::mutex ws_mutex;
    std::map<cudaStream_t, Workspace> workspaces;  // one per stream, allocated on first use
    std::map<cudaStream_t, BatchBuffers> batches;   // batched-path buffers per stream
    ModUpDesc* d_modup = nullptr;                  // device copy of modup, [level * dnum + part]
    // host copy of the rescale constants: for dropped limb d at rs_host_off[d]:
    // one_s[d], inv_p[d], inv_p_s[d], half[d]
    std::vector<uint64_t> rs_host;
    std::vector<size_t> rs_host_off;
    BatchBuffers& batch_buffers(cudaStream_t s);
    // Evaluation-form plaintexts of slot-constant values, kept for the context's lifetime
    // (keyed by value, scale and limb count); `ready` follows the NTT that filled them on
    // `stream`, for users on other streams.
    struct ConstPlain {
        uint64_t* d;
        cudaEvent_t ready;
        cudaStream_t stream;
        size_t bytes;
    };
    std::mutex const_mutex;
    std::map<std::tuple<double, double, double, size_t>, ConstPlain> consts;
    size_t const_bytes = 0;
    // Chunks of stream-ordered device memory that finished operation sets hand back for later
    // ones: each carries an event recorded on the stream that last used it, and a taker's stream
    // waits on that event before its first use, so reuse needs no host synchronisation and
    // works across streams.  At most kChunkCacheBytes are kept over all contexts of the
    // process together (chunk_cache_total), so many contexts on one device do not each hold
    // their own reserve; the rest is freed.
    struct CachedChunk {
        void* p;
        size_t bytes;
        cudaEvent_t done;
    };
    static constexpr size_t kChunkCacheBytes = size_t{24} << 30;
    std::mutex chunk_mutex;
    std::multimap<size_t, CachedChunk> chunk_cache;
    std::vector<cudaEvent_t> chunk_events;
    size_t chunk_cache_bytes = 0;
    // a cached chunk of at least `bytes` (at most twice that) made safe for use on s, or nullptr
    void* take_chunk(size_t bytes, cudaStream_t s, size_t* got);
    void give_chunk(void* p, size_t bytes, cudaStream_t s);
    // Give back what the context holds for stream s beyond its tables and keys: the stream's
    // batched scratch arena and staging ring, its single-operation workspace, every cached
    // chunk (waiting for their last users first) and the stream-ordered pool's unused reserve.
    // The next call on s allocates again.
    void trim(cudaStream_t s);

    ~Context();
    uint64_t* workspace(cudaStream_t s);   // scratch for one in-flight operation on stream s
    size_t workspace_words() const;
    const KeyEntry& key(int kind, int64_t rotation) const;

    size_t parts_at(size_t level) const {
        if (level >= nq) return 0;
        const size_t L = level + 1;
        const size_t p_ = (L + alpha - 1) / alpha;
        return p_ < dnum ? p_ : dnum;
    }
};

// Modulus-index rule for a batch of limbs: limb l of a polynomial uses modulus
// (l < nA ? firstA + l : firstB + l - nA).  Q moduli occupy [0, nq), P moduli [nq, nq+np).
struct LimbMap {
    int nA;
    int firstA;
    int firstB;
    __host__ __device__ int operator()(int l) const { return l < nA ? firstA + l : firstB + (l - nA); }
};

// ---------------------------------------------------------------------------------------
// Launch accounting.  Every kernel launch of the library goes through a Probe: it counts
// launches and, when event timing is enabled for the launch's class, brackets it with a pair
// of CUDA events on the launching stream and books its algorithmic bytes.
// ---------------------------------------------------------------------------------------
enum KernelClass : int {
    kClsNtt = 0,       // NTT / inverse NTT phases
    kClsModUp = 1,     // HPS base extension
    kClsKeyMac = 2,    // key inner product
    kClsModDown = 3,   // folded HPS ModDown
    kClsCombine = 4,   // combine / automorphism gathers
    kClsElementwise = 5,  // tensor, add/sub, rescale steps
    kClsWalsh = 6,     // Walsh S-box products and sums
    kClsGiant = 7,     // BSGS giant-step sums
    kClsCount = 8
};
// Per-class launch counters: snapshot, and credit of the kernels a graph replay runs.
void probe_counts(uint64_t* out);
void probe_add(const uint64_t* counts);
struct Probe {
    Probe(int cls, double bytes, cudaStream_t s);
    ~Probe();
    Probe(const Probe&) = delete;
    Probe& operator=(const Probe&) = delete;
    int slot = -1;
    cudaStream_t stream;
#ifdef WG_HOST_SPANS
    HostSpan span{"launch"};
#endif
};

// ---------------------------------------------------------------------------------------
// Kernel launchers.
// ---------------------------------------------------------------------------------------
// One limb of a job-table NTT: the first phase reads src and writes dst, the second phase
// works in place on dst (src == dst for an in-place transform).
struct NttJob {
    const uint64_t* src;
    uint64_t* dst;
    int mod;
    int pad;
};
void ntt_jobs(const Context& c, const NttJob* d_jobs, int njobs, bool forward, cudaStream_t s);
// Time every NTT geometry on the context's device and keep the fastest per direction and phase
// (cached per device and ring degree for the process).
void ntt_autotune(Context& c);
// One phase (cols: the high-bit phase) of a strided batch with a given geometry.
void ntt_phase_geometry(const Context& c, bool forward, bool cols, int variant, uint64_t* data, int limbs,
                        int polys, size_t poly_stride, LimbMap map, cudaStream_t s);

// One phase of a job-table NTT (cols: the high-bit phase) with the context's geometry; the
// inverse transform is rows then columns, the forward one columns then rows, and the first
// phase reads src and writes dst.
void ntt_jobs_phase(const Context& c, const NttJob* d_jobs, int njobs, bool forward, bool cols, cudaStream_t s);

// ModUp and ModDown jobs of the batched kernels (kb_modup, kb_moddown: coefficient-form limbs in
// and out) and of the fused key-switch steps (wg_ksfuse.cu).  A ModUp job is one digit of one
// switch: for the fused kernel src holds the switch's L Q limbs after the inverse row phase, and
// every destination limb of the digit is written after the forward column phase (the forward
// row phase follows as a job-table launch).  A ModDown job is one accumulator polynomial: for
// the fused kernel src_p holds its K P limbs after the inverse row phase, and out receives the L
// contribution limbs after the forward column phase.
struct ModUpNttJob {
    const ModUpDesc* desc;
    const uint64_t* src;
    uint64_t* digit;
};
struct ModDownNttJob {
    const uint64_t* src_p;
    uint64_t* out;
    const uint64_t* inv;  // folded P^-1 table of the level, [qi][pi]
    const uint64_t* inv_s;
    int L;
    int pad;
};
// Rescale of one polynomial at level lv (ckks_rescale): drop holds its last limb after the
// inverse row phase; the kernel finishes that inverse transform, forms the rounded remainder
// for every lower limb and writes it to rem (lv limbs) after the forward column phase.  rc: the
// device rescale constants of level lv (one_s, inv_p, inv_p_s, half; lv words each).
struct RescaleNttJob {
    const uint64_t* drop;
    uint64_t* rem;
    const uint64_t* rc;
    int lv;
    int pad;
};
// The forward row phase of job-table limbs with an element-wise epilogue (NttEpiJob, wg_ntt.cuh).
using ntt::NttEpiJob;
using ntt::kEpiRescale;
using ntt::kEpiCombine;
void ntt_rows_epilogue_jobs(const Context& c, const NttEpiJob* d_jobs, int njobs, double bytes, cudaStream_t s);
// Algorithmic bytes of such jobs: the phase's share of its transform (8 N B per limb, as every
// NTT phase is booked) plus the words the epilogue reads (acc, in) and writes (out).
inline double ntt_epilogue_bytes(const std::vector<NttEpiJob>& jobs, size_t N) {
    double words = 0.0;
    for (const NttEpiJob& j : jobs)
        words += 2.0 + (j.kind == kEpiCombine ? 1.0 : 0.0) + ((j.kind == kEpiRescale || j.c0) ? 1.0 : 0.0);
    return 8.0 * (double)N * words;
}
void rescale_ntt_jobs(const Context& c, const RescaleNttJob* d_jobs, int njobs, double bytes, cudaStream_t s);

// max_src: the largest source-limb count of the jobs (shared-memory size).
void modup_ntt_jobs(const Context& c, const ModUpNttJob* d_jobs, int njobs, int max_src, double bytes,
                    cudaStream_t s);
// fma_alpha: the alpha estimate rounded as fused multiply-adds (the key switch's pair ModDown)
// or as multiplies then adds (the single-polynomial ModDown of the QP linear transform).
void moddown_ntt_jobs(const Context& c, const ModDownNttJob* d_jobs, int njobs, double bytes, cudaStream_t s,
                      bool fma_alpha = true);

// NTT over `polys` polynomials of `limbs` limbs each, `poly_stride` words apart.
void ntt_forward(const Context& c, uint64_t* data, int limbs, int polys, size_t poly_stride,
                 LimbMap map, cudaStream_t s);
void ntt_inverse(const Context& c, uint64_t* data, int limbs, int polys, size_t poly_stride,
                 LimbMap map, cudaStream_t s);

// Key switch of key_term (level) with key `k`; b/a combine modes; optional automorphism
// (galois != 0) applied to the outputs.  `ws` must hold keyswitch_workspace_words(level).
size_t keyswitch_workspace_words(const Context& c, size_t level);
// b = (b_add ? b_in + ks_b : ks_b), a likewise; b_in/a_in may alias b/a.
void keyswitch(const Context& c, size_t level, const uint64_t* key_term, const KeyEntry& k,
               const uint64_t* b_in, const uint64_t* a_in, uint64_t* b, uint64_t* a, bool b_add,
               bool a_add, uint64_t galois, uint64_t* ws, cudaStream_t s);

// Elementwise and structural kernels (wg_ops.cu).
void automorphism(const Context& c, const uint64_t* src, uint64_t* dst, int limbs, int polys,
                  size_t poly_stride, uint64_t galois, cudaStream_t s);
void tensor(const Context& c, size_t level, uint64_t* b1, uint64_t* a1, const uint64_t* b2,
            const uint64_t* a2, uint64_t* c2, cudaStream_t s);
// Divide by the last active Q limb with rounding; ws holds npolys*level*N words.
void rescale(const Context& c, size_t level, uint64_t* polys, int npolys, size_t poly_stride,
             uint64_t* ws, cudaStream_t s);
void add_sub(const Context& c, size_t level, uint64_t* x, const uint64_t* y, int npolys,
             size_t poly_stride, bool subtract, cudaStream_t s);

}  // namespace wg

// The public context handle of include/walsh_gpu.h: a wrapper around the engine context, defined
// once here for every file that implements entry points on it.
struct wg_context {
    wg::Context* c;
};
