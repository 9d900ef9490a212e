// Continuous-batching AES-CTR transciphering service on one device (wg_serve.cu).
//
// No counterpart in the reference, whose benchmark runs one AES-CTR evaluation at a time
// (bench/aes_bench.cpp).  Requests of counter blocks queue up; each free worker takes every
// waiting request, in arrival order, that still fits into one evaluation's block slots (1024 for
// walsh15, one per active slot for the XBOOT parameter sets), runs the homomorphic AES-CTR on its
// own stream and hands every request its output bit ciphertexts.  Workers run evaluations
// concurrently (their kernels interleave on the device) as far as the device-memory budget allows.
#pragma once
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "wg_batch.hpp"

namespace wg {

// Everything an evaluation needs besides its blocks; pointers must outlive the server.
struct ServeSetup {
    BootstrapParams bp;
    std::vector<const LtStage*> s2c, s2c_x2, c2s;
    std::vector<double> coeffs;
    std::vector<const uint64_t*> key_b, key_a;  // 1408 encrypted round-key bits
    std::vector<double> key_scales;
    size_t key_level = 0, packing_block_count = 0, packed_segment_count = 0;
    // XBOOT evaluations (aes_ctr_xboot) instead of Walsh ones: key bits at key_levels, one block
    // per active slot, no packing; s2c_x2, key_level and the packing counts are unused
    bool xboot = false;
    std::vector<size_t> key_levels;
};

// Device bytes that the evaluations of several servers on one device share: a worker takes its
// evaluation's bytes before it starts (waiting while the others hold them) and returns them when
// it finishes.  An evaluation larger than the whole budget runs alone.
struct ServeBudget {
    std::mutex mu;
    std::condition_variable cv;
    size_t capacity = 0;
    size_t in_use = 0;
    size_t acquire(size_t bytes);  // returns the bytes taken (clamped to the capacity)
    void release(size_t bytes);
};

struct ServeConfig {
    size_t workers = 2;        // evaluations that may run at once
    size_t hbm_budget = 0;     // device bytes the evaluations may take together (0: no limit)
    size_t eval_bytes = 0;     // device bytes one evaluation takes (admission estimate)
    size_t max_blocks = 0;     // block slots per evaluation (0: 2 x packing block count, or the
                               // active slot count for XBOOT)
    double batch_window_ms = 0.0;  // a free worker waits this long after the oldest queued
                                   // request for more to fill its batch (0: start at once)
    int priority = 0;              // 1: the workers' streams take the device's highest scheduling
                                   // priority, so this server's kernels go first when servers
                                   // share the device (short evaluations do not wait behind long
                                   // ones); 0: default priority
    ServeBudget* budget = nullptr; // shared with other servers (null: this server's own limit);
                                   // workers then release their stream's scratch after each
                                   // evaluation (Context::trim), so idle servers hold none
};

struct ServeResult {
    int status = 0;            // WG_OK, or the error code of the failed evaluation
    std::string error;
    size_t block_offset = 0;   // first evaluation block of the request
    size_t active_blocks = 0;  // the evaluation's blocks per lane (Walsh: the packing block count;
                               // block b sits in slot b mod it, real part for b < it, imaginary
                               // otherwise.  XBOOT: the active slot count; block b in slot b)
    size_t batch_requests = 0, batch_blocks = 0;
    double queue_ms = 0.0, latency_ms = 0.0;  // submission to start, submission to completion
    size_t out_level[128] = {};
    double out_scale[128] = {};
};

// One worker's stream and its evaluation's output buffers ([bit][b, a][(depth + 1) N]).
struct ServeWorker {
    cudaStream_t stream = nullptr;
    uint64_t* out = nullptr;
};

class Server {
public:
    Server(Context& c, ServeSetup setup, const ServeConfig& cfg);
    ~Server();  // finishes every queued request, then stops the workers
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Queue a request: `blocks` counter blocks and as many ciphertext blocks (16 bytes each;
    // Walsh: blocks even, 2 <= blocks <= max_blocks; XBOOT: 1 <= blocks <= max_blocks); out_b /
    // out_a are 128 device buffers of (depth + 1) N words each that receive the output bit
    // ciphertexts.  Returns its id.
    uint64_t submit(const uint8_t* counters, const uint8_t* ciphertexts, size_t blocks, uint64_t* const* out_b,
                    uint64_t* const* out_a);
    // Wait up to timeout_s (negative: no limit) for a request; true when it has finished.
    bool wait(uint64_t id, double timeout_s, ServeResult* out);
    size_t max_blocks() const { return max_blocks_; }

private:
    using Clock = std::chrono::steady_clock;
    struct Request {
        uint64_t id;
        std::vector<uint8_t> counters, ciphertexts;
        size_t blocks;
        std::vector<uint64_t*> out_b, out_a;
        Clock::time_point submitted;
    };
    void worker(size_t w);
    size_t admitted() const;
    bool head_batch_full() const;
    void release_workers();

    Context& c_;
    ServeSetup setup_;
    ServeConfig cfg_;
    size_t max_blocks_ = 0;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::deque<Request> queue_;
    std::map<uint64_t, ServeResult> done_;
    std::set<uint64_t> pending_;  // submitted, not finished
    std::vector<ServeWorker> workers_;
    uint64_t next_id_ = 1;
    size_t running_ = 0;
    bool stop_ = false;
    std::vector<std::thread> threads_;
};

}  // namespace wg
