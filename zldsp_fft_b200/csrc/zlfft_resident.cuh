// Per-device kernel set-up shared by the launch functions.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

namespace zlfft {

constexpr int kMaxDevices = 64;

// A launch site's cache of resident CTAs per SM, one slot per device
// (0: not set up on that device yet).
using ResidentSlots = std::atomic<int>[kMaxDevices];

// Resident CTAs per SM of one kernel on the current device. `setup` raises
// the kernel's dynamic shared-memory limit and returns the count (>= 1).
// Function attributes belong to one device's context, so `setup` runs on the
// first launch on each device, not once per process. Two threads racing on a
// first launch both set the same attributes and store the same count.
template <typename Setup>
int resident_ctas(ResidentSlots& slots, Setup&& setup) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return setup();
    int b = slots[dev].load(std::memory_order_acquire);
    if (b == 0) {
        b = setup();
        slots[dev].store(b, std::memory_order_release);
    }
    return b;
}

// The common set-up: the shared-memory limit, then the occupancy query.
template <typename K>
int occupancy_setup(K kern, int threads, size_t smem) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, threads, smem) != cudaSuccess || b < 1) b = 1;
    return b;
}

}  // namespace zlfft
