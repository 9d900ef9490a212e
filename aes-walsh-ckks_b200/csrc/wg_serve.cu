// Continuous-batching AES-CTR service (wg_serve.hpp).
//
// Each worker thread owns a non-blocking stream and one evaluation's output buffers.  A free
// worker waits until requests are queued and fewer evaluations run than the memory budget
// admits, takes every queued request, in arrival order, whose blocks still fit into one
// evaluation (a request never splits) and concatenates their counter and ciphertext blocks.
// An XBOOT evaluation (aes_ctr_xboot) takes them as they are, block b in slot b.  A Walsh one
// pads them with zero blocks to the evaluation's full 2 x packing-block-count slots (block b: real slot
// b for b < packing blocks, imaginary slot b - packing blocks otherwise; the circuit's final
// refresh packs by rotations of multiples of the active block count, and the walsh15 context
// holds rotation keys for the full count only, as the reference's does), runs aes_ctr_walsh on
// its stream, copies the 128 output bit ciphertexts into every
// request's buffers and publishes the results.  Requests that arrive meanwhile wait for the next
// free worker, so evaluations of later arrivals overlap the running ones on the device.
#include <algorithm>
#include <stdexcept>

#include "../../include/walsh_gpu.h"
#include "wg_batching.hpp"
#include "wg_internal.hpp"
#include "wg_serve.hpp"

namespace wg {

namespace {
constexpr size_t kStateBits = 128;
constexpr size_t kKeyBits = 11 * kStateBits;
constexpr size_t kBlockBytes = 16;
}  // namespace

size_t ServeBudget::acquire(size_t bytes) {
    std::unique_lock<std::mutex> lk(mu);
    const size_t take = capacity ? std::min(bytes, capacity) : 0;
    if (!take) return 0;
    cv.wait(lk, [&] { return in_use + take <= capacity; });
    in_use += take;
    return take;
}

void ServeBudget::release(size_t bytes) {
    {
        std::lock_guard<std::mutex> g(mu);
        in_use -= std::min(bytes, in_use);
    }
    cv.notify_all();
}

Server::Server(Context& c, ServeSetup setup, const ServeConfig& cfg) : c_(c), setup_(std::move(setup)), cfg_(cfg) {
    if (setup_.key_b.size() != kKeyBits || setup_.key_a.size() != kKeyBits || setup_.key_scales.size() != kKeyBits)
        throw std::invalid_argument("wg_serve: expected 1408 encrypted round-key bits");
    if (setup_.xboot) {
        if (setup_.key_levels.size() != kKeyBits) throw std::invalid_argument("wg_serve: expected 1408 key-bit levels");
        const size_t slots = setup_.bp.active_slots;
        max_blocks_ = cfg_.max_blocks ? cfg_.max_blocks : slots;
        if (max_blocks_ == 0 || max_blocks_ > slots)
            throw std::invalid_argument("wg_serve: block slots per evaluation must be 1..active slots");
    } else {
        if (setup_.packing_block_count == 0) throw std::invalid_argument("wg_serve: packing block count must be nonzero");
        max_blocks_ = cfg_.max_blocks ? cfg_.max_blocks : 2 * setup_.packing_block_count;
        if (max_blocks_ < 2 || (max_blocks_ & 1) || max_blocks_ > 2 * setup_.packing_block_count)
            throw std::invalid_argument("wg_serve: block slots per evaluation must be even and at most 2 x packing blocks");
    }
    if (cfg_.workers == 0) throw std::invalid_argument("wg_serve: at least one worker");
    check_cuda(cudaSetDevice(c_.device), "cudaSetDevice");
    workers_.resize(cfg_.workers);
    const size_t words = kStateBits * 2 * (setup_.bp.depth + 1) * c_.N;
    int prio = 0;
    if (cfg_.priority) {
        int least = 0, greatest = 0;
        check_cuda(cudaDeviceGetStreamPriorityRange(&least, &greatest), "wg_serve: stream priorities");
        prio = greatest;
    }
    for (auto& w : workers_) {
        if (cudaStreamCreateWithPriority(&w.stream, cudaStreamNonBlocking, prio) != cudaSuccess ||
            cudaMalloc((void**)&w.out, words * 8) != cudaSuccess) {
            cudaGetLastError();
            release_workers();
            fail(kNoMemory, "wg_serve: worker stream or output buffers");
        }
    }
    for (size_t w = 0; w < cfg_.workers; ++w) threads_.emplace_back(&Server::worker, this, w);
}

void Server::release_workers() {
    for (auto& w : workers_) {
        if (w.stream) cudaStreamSynchronize(w.stream);
        cudaFree(w.out);
        if (w.stream) cudaStreamDestroy(w.stream);
    }
    workers_.clear();
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
    release_workers();
}

// the queued requests already fill the next evaluation (wg_batching.hpp)
bool Server::head_batch_full() const {
    return batch_full(queue_, max_blocks_, [](const Request& r) { return r.blocks; });
}

size_t Server::admitted() const {
    size_t n = cfg_.workers;
    if (cfg_.hbm_budget && cfg_.eval_bytes) n = std::min(n, std::max<size_t>(1, cfg_.hbm_budget / cfg_.eval_bytes));
    return n;
}

uint64_t Server::submit(const uint8_t* counters, const uint8_t* ciphertexts, size_t blocks, uint64_t* const* out_b,
                        uint64_t* const* out_a) {
    if (!counters || !ciphertexts || !out_b || !out_a) throw std::invalid_argument("wg_serve: null argument");
    if (setup_.xboot ? (blocks == 0 || blocks > max_blocks_) : (blocks < 2 || (blocks & 1) || blocks > max_blocks_))
        throw std::invalid_argument(setup_.xboot
                                        ? "wg_serve: block count must be at least 1 and at most the evaluation's slots"
                                        : "wg_serve: block count must be even, at least 2 and at most the evaluation's slots");
    Request r;
    r.counters.assign(counters, counters + blocks * kBlockBytes);
    r.ciphertexts.assign(ciphertexts, ciphertexts + blocks * kBlockBytes);
    r.blocks = blocks;
    r.out_b.assign(out_b, out_b + kStateBits);
    r.out_a.assign(out_a, out_a + kStateBits);
    for (size_t k = 0; k < kStateBits; ++k)
        if (!r.out_b[k] || !r.out_a[k]) throw std::invalid_argument("wg_serve: null output buffer");
    r.submitted = Clock::now();
    uint64_t id;
    {
        std::lock_guard<std::mutex> g(mu_);
        if (stop_) throw std::runtime_error("wg_serve: server is stopping");
        id = r.id = next_id_++;
        pending_.insert(id);
        queue_.push_back(std::move(r));
    }
    cv_.notify_all();
    return id;
}

bool Server::wait(uint64_t id, double timeout_s, ServeResult* out) {
    std::unique_lock<std::mutex> lk(mu_);
    auto ready = [&] { return done_.count(id) != 0; };
    if (!ready() && !pending_.count(id)) throw std::invalid_argument("wg_serve: unknown or already collected request");
    if (timeout_s < 0) {
        done_cv_.wait(lk, ready);
    } else if (!done_cv_.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return false;
    }
    *out = std::move(done_[id]);
    done_.erase(id);
    return true;
}

void Server::worker(size_t w) {
    cudaSetDevice(c_.device);
    ServeWorker& me = workers_[w];
    const size_t N = c_.N, full = (setup_.bp.depth + 1) * N;
    std::vector<uint64_t*> ob(kStateBits), oa(kStateBits);
    for (size_t k = 0; k < kStateBits; ++k) {
        ob[k] = me.out + (2 * k) * full;
        oa[k] = me.out + (2 * k + 1) * full;
    }
    const S2cPlan plans[2] = {{1, setup_.s2c.data(), setup_.s2c.size()},
                              {2, setup_.s2c_x2.data(), setup_.s2c_x2.size()}};
    for (;;) {
        std::vector<Request> batch;
        size_t blocks = 0;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return (stop_ && queue_.empty()) || (!queue_.empty() && running_ < admitted()); });
            if (queue_.empty()) return;
            if (cfg_.batch_window_ms > 0.0 && !stop_) {
                // wait for more requests until the batch is full or the oldest has waited the window
                const auto deadline = queue_.front().submitted +
                                      std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double, std::milli>(cfg_.batch_window_ms));
                cv_.wait_until(lk, deadline, [&] { return stop_ || queue_.empty() || head_batch_full(); });
                if (queue_.empty() || running_ >= admitted()) continue;  // another worker took them
            }
            // every queued request that still fits, in arrival order (first fit, wg_batching.hpp)
            const std::vector<size_t> take = first_fit(queue_, max_blocks_, [](const Request& r) { return r.blocks; });
            std::deque<Request> rest;
            for (size_t k = 0, t = 0; k < queue_.size(); ++k) {
                if (t < take.size() && take[t] == k) {
                    blocks += queue_[k].blocks;
                    batch.push_back(std::move(queue_[k]));
                    ++t;
                } else {
                    rest.push_back(std::move(queue_[k]));
                }
            }
            queue_.swap(rest);
            ++running_;
        }
        // a budget shared with other servers: hold this evaluation's bytes while it runs
        const size_t held = cfg_.budget && cfg_.eval_bytes ? cfg_.budget->acquire(cfg_.eval_bytes) : 0;
        const auto started = Clock::now();
        const size_t active = setup_.xboot ? setup_.bp.active_slots : setup_.packing_block_count;
        ServeResult base;
        base.batch_requests = batch.size();
        base.batch_blocks = blocks;
        base.active_blocks = active;
        try {
            std::vector<uint8_t> counters, cts;
            counters.reserve(2 * active * kBlockBytes);
            cts.reserve(2 * active * kBlockBytes);
            for (const auto& r : batch) {
                counters.insert(counters.end(), r.counters.begin(), r.counters.end());
                cts.insert(cts.end(), r.ciphertexts.begin(), r.ciphertexts.end());
            }
            if (setup_.xboot) {
                // the XBOOT circuit takes the batch's blocks as they are (slot b = block b)
                XbootAesArgs x;
                x.key_b = setup_.key_b.data();
                x.key_a = setup_.key_a.data();
                x.key_scales = setup_.key_scales.data();
                x.key_levels = setup_.key_levels.data();
                x.counters = counters.data();
                x.ciphertexts = cts.data();
                x.blocks = blocks;
                aes_ctr_xboot(c_, setup_.bp, plans, 1, setup_.c2s.data(), setup_.c2s.size(), setup_.coeffs.data(),
                              setup_.coeffs.size(), x, ob.data(), oa.data(), base.out_level, base.out_scale,
                              me.stream);
            } else {
                counters.resize(2 * active * kBlockBytes, 0);
                cts.resize(2 * active * kBlockBytes, 0);
                AesArgs a;
                a.key_b = setup_.key_b.data();
                a.key_a = setup_.key_a.data();
                a.key_scales = setup_.key_scales.data();
                a.key_level = setup_.key_level;
                a.counters = counters.data();
                a.ciphertexts = cts.data();
                a.active_blocks = active;
                a.packing_block_count = setup_.packing_block_count;
                a.packed_segment_count = setup_.packed_segment_count;
                aes_ctr_walsh(c_, setup_.bp, plans, setup_.s2c_x2.empty() ? 1 : 2, setup_.c2s.data(), setup_.c2s.size(),
                              setup_.coeffs.data(), setup_.coeffs.size(), a, ob.data(), oa.data(), base.out_level,
                              base.out_scale, me.stream);
            }
            for (const auto& r : batch)
                for (size_t k = 0; k < kStateBits; ++k) {
                    const size_t bytes = (base.out_level[k] + 1) * N * 8;
                    check_cuda(cudaMemcpyAsync(r.out_b[k], ob[k], bytes, cudaMemcpyDeviceToDevice, me.stream), "serve out");
                    check_cuda(cudaMemcpyAsync(r.out_a[k], oa[k], bytes, cudaMemcpyDeviceToDevice, me.stream), "serve out");
                }
            check_cuda(cudaStreamSynchronize(me.stream), "serve evaluation");
            // under a budget shared with other servers the bytes held between evaluations count
            // too: give back this stream's scratch and the context's cached chunks
            if (cfg_.budget) c_.trim(me.stream);
        } catch (const Error& e) {
            base.status = e.code;
            base.error = e.what();
        } catch (const std::invalid_argument& e) {
            base.status = kInvalid;
            base.error = e.what();
        } catch (const std::exception& e) {
            base.status = kRuntime;
            base.error = e.what();
        }
        const auto finished = Clock::now();
        if (held) cfg_.budget->release(held);
        {
            std::lock_guard<std::mutex> g(mu_);
            size_t off = 0;
            for (const auto& r : batch) {
                ServeResult res = base;
                res.block_offset = off;
                off += r.blocks;
                res.queue_ms = std::chrono::duration<double, std::milli>(started - r.submitted).count();
                res.latency_ms = std::chrono::duration<double, std::milli>(finished - r.submitted).count();
                pending_.erase(r.id);
                done_.emplace(r.id, std::move(res));
            }
            --running_;
        }
        done_cv_.notify_all();
        cv_.notify_all();
    }
}

}  // namespace wg
