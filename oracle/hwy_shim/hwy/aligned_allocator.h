// Highway-API shim (TEST INFRASTRUCTURE ONLY): the aligned-allocation names
// the reference uses (hwy::AllocateAligned, hwy::AlignedFreeUniquePtr),
// written from Highway's documented behaviour: an array of n default-
// initialised T, aligned to HWY_ALIGNMENT, released with the matching free.
#pragma once

#include <cstddef>
#include <cstdlib>
#include <memory>
#include <new>

namespace hwy {

struct ShimAlignedFreer {
    void operator()(void* p) const noexcept { std::free(p); }
};

template <typename T>
using AlignedFreeUniquePtr = std::unique_ptr<T, ShimAlignedFreer>;

template <typename T>
AlignedFreeUniquePtr<T[]> AllocateAligned(const size_t n) {
    constexpr size_t kAlign = 64;
    size_t bytes = n * sizeof(T);
    bytes = (bytes + kAlign - 1) / kAlign * kAlign;
    if (bytes == 0) bytes = kAlign;
    void* p = std::aligned_alloc(kAlign, bytes);
    if (p == nullptr) throw std::bad_alloc();
    return AlignedFreeUniquePtr<T[]>(static_cast<T*>(p));
}

}  // namespace hwy
