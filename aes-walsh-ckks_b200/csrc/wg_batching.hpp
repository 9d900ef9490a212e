// Request packing of the batching service (wg_serve.cu), host-only and free of CUDA so the CPU
// tests can drive it.  No counterpart in the reference, which evaluates one batch at a time.
#pragma once
#include <cstddef>
#include <vector>

namespace wg {

// The queued requests (arrival order) that share the next evaluation of max_blocks block slots:
// every request that still fits beside those taken before it (first fit).  The oldest request
// always fits an empty evaluation, so none waits behind later ones for ever.  size(r) is a
// request's block count (>= 1).  Returns the positions taken, ascending.
template <class Queue, class Size>
std::vector<size_t> first_fit(const Queue& queue, size_t max_blocks, Size size) {
    std::vector<size_t> take;
    size_t blocks = 0, k = 0;
    for (auto it = queue.begin(); it != queue.end() && blocks < max_blocks; ++it, ++k) {
        const size_t n = size(*it);
        if (blocks + n <= max_blocks) {
            blocks += n;
            take.push_back(k);
        }
    }
    return take;
}

// The queued requests already fill the next evaluation: one of them no longer fits beside the
// others, or the block slots are used up.
template <class Queue, class Size>
bool batch_full(const Queue& queue, size_t max_blocks, Size size) {
    size_t blocks = 0;
    bool skipped = false;
    for (const auto& r : queue) {
        const size_t n = size(r);
        if (blocks + n <= max_blocks)
            blocks += n;
        else
            skipped = true;
    }
    return skipped || blocks == max_blocks;
}

}  // namespace wg
