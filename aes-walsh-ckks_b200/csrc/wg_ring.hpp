// Placement in the staging ring (BatchBuffers in wg_internal.hpp), host-only and free of CUDA so
// the CPU tests can drive it.
//
// Regions are handed out front to back and wrap to offset 0 when the next one does not fit.  A
// region may be written by the host only after every upload still in flight over any of its
// bytes has completed.  The in-flight list is in issue order, which after an early wrap is not
// address order (old uploads at high offsets can precede newer ones at low offsets), so the whole
// list is searched; since the uploads of one ring go through one stream and complete in issue
// order, waiting for the newest overlapping one completes every older one as well.
#pragma once
#include <cstddef>

namespace wg {

// Chooses the region for `need` bytes (need <= ring_bytes): returns its offset and advances
// nothing; *wait_count = how many of the oldest flights must complete (and can then be
// released) before the region may be written.
template <class Flights>
size_t ring_place(size_t head, size_t ring_bytes, size_t need, const Flights& flights, size_t* wait_count) {
    const size_t begin = head + need > ring_bytes ? 0 : head;
    const size_t end = begin + need;
    size_t count = 0, k = 0;
    for (const auto& f : flights) {
        ++k;
        if (f.begin < end && begin < f.end) count = k;
    }
    *wait_count = count;
    return begin;
}

}  // namespace wg
