// The reference API's container type (src/util/aligned_vector.hpp): a std::vector whose storage
// is 64-byte aligned.  Code written against the reference's headers uses MyVector<T> for keys,
// ciphertext lists and decoded slots.
#ifndef ALIGNED_VECTOR_HPP
#define ALIGNED_VECTOR_HPP

#include <cstddef>
#include <limits>
#include <new>
#include <type_traits>
#include <vector>

template <class T, std::size_t Alignment = 64>
struct AlignedAllocator {
    using value_type = T;
    using is_always_equal = std::true_type;
    template <class U>
    struct rebind {
        using other = AlignedAllocator<U, Alignment>;
    };

    AlignedAllocator() noexcept = default;
    template <class U>
    AlignedAllocator(const AlignedAllocator<U, Alignment>&) noexcept {}

    [[nodiscard]] T* allocate(std::size_t n) {
        static_assert((Alignment & (Alignment - 1)) == 0 && Alignment >= alignof(T), "bad alignment");
        if (n == 0) return nullptr;
        if (n > (std::numeric_limits<std::size_t>::max)() / sizeof(T)) throw std::bad_alloc();
        return static_cast<T*>(::operator new(n * sizeof(T), std::align_val_t{Alignment}));
    }
    void deallocate(T* p, std::size_t) noexcept { ::operator delete(p, std::align_val_t{Alignment}); }

    template <class U>
    bool operator==(const AlignedAllocator<U, Alignment>&) const noexcept {
        return true;
    }
    template <class U>
    bool operator!=(const AlignedAllocator<U, Alignment>&) const noexcept {
        return false;
    }
};

template <class T>
using MyVector = std::vector<T, AlignedAllocator<T>>;

#endif  // ALIGNED_VECTOR_HPP
