// G7: one persistent launch for a mixed batch of transforms of many orders.
//
// A mixed batch (thousands of transforms of uneven order, CFFT and RFFT
// mixed) is grouped on the host by (kind, order, operation);
// each group is cut into tiles of the tile kernel's shape (TPC transforms of
// one order). The tiles form one work list per order class, sorted longest
// first: complex orders 2..11 in 128-thread CTAs, and 12..13 in 512-thread
// CTAs (two transforms of order 12 or one of order 13 per tile). Resident CTAs
// pull tiles from their class's list through an atomic counter and run the
// same TileWorker body as tile_kernel on gathered per-transform pointers. The
// grid is sized to the resident capacity, so each launch stays persistent and
// load-balanced across orders whose costs differ by 2^10; splitting the body
// by class keeps each kernel's instruction footprint and registers to the
// variants of its own class.
#pragma once

#include "zlfft_resident.cuh"
#include "zlfft_tile.cuh"

namespace zlfft {

constexpr int kMixedMinP = 2;   // smallest complex order in the persistent kernels
constexpr int kMixedMaxP = 11;  // largest of the 128-thread class: T <= 128 threads per transform
constexpr int kMixedBlock = 128;
constexpr int kMixedLargeMinP = 12;  // the 512-thread class
constexpr int kMixedLargeMaxP = 13;
constexpr int kMixedLargeBlock = 512;
constexpr int kMixedTopP = kMixedLargeMaxP;  // largest complex order of any persistent class

// Order class of a complex order (0: 128 threads, 1: 512 threads) and its CTA size.
__host__ __device__ constexpr int mixed_class(int P) { return P > kMixedMaxP ? 1 : 0; }

// operation codes handled by the persistent kernel (AoS <-> AoS)
__host__ __device__ constexpr int mixed_code(int op, int P) { return op * 32 + P; }

struct MixedGroup {
    TileArgs a;  // gathered pointers (gin0/gout0), twiddles of the group's plan, batch = group size
    int code;    // mixed_code(op, P)
};

struct MixedItem {
    int group;
    int tile;  // tile index inside the group (TPC transforms per tile)
};

template <typename F, int OP, int P, int BLOCK>
__device__ __forceinline__ bool mixed_try(int code, const MixedGroup& g, int tile, unsigned char* smem) {
    if (code != mixed_code(OP, P)) return false;
    TileWorker<F, P, OP, kAoS, kAoS, BLOCK, true> w(g.a, smem);
    w.run(g.a, tile, false, []() {});
    return true;
}

template <typename F, int OP, int BLOCK, int MINP, int... Ps>
__device__ __forceinline__ bool mixed_try_op(int code, const MixedGroup& g, int tile, unsigned char* smem,
                                             std::integer_sequence<int, Ps...>) {
    return (mixed_try<F, OP, MINP + Ps, BLOCK>(code, g, tile, smem) || ...);
}

// Resident CTAs per SM: 128 registers per thread. The union of all order and
// operation variants of the 128-thread class spills heavily at 96 (5 CTAs),
// little at 128. The 512-thread class runs one CTA per SM at 128 registers.
template <int BLOCK>
constexpr int mixed_minb() { return BLOCK == kMixedBlock ? 4 : 1; }

template <typename F, int BLOCK, int MINP, int MAXP>
__global__ void __launch_bounds__(BLOCK, mixed_minb<BLOCK>())
    mixed_kernel(const MixedGroup* __restrict__ groups, const MixedItem* __restrict__ items, int n_items,
                 int* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    using Ps = std::make_integer_sequence<int, MAXP - MINP + 1>;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const MixedItem item = items[it];
        const MixedGroup& g = groups[item.group];
        const int code = g.code;
        mixed_try_op<F, kC2CFwd, BLOCK, MINP>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kC2CBwd, BLOCK, MINP>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kR2CFwd, BLOCK, MINP>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kR2CSqrMag, BLOCK, MINP>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kC2RBwd, BLOCK, MINP>(code, g, item.tile, smem_raw, Ps{});
        __syncthreads();  // shared memory and s_item are reused by the next tile
    }
}

// Shared memory of a persistent class: the largest tile of its orders,
// TPC * N complex values = BLOCK * E = BLOCK * 16 points (orders >= 4).
template <typename F, int BLOCK>
constexpr size_t mixed_smem() {
    return (size_t)BLOCK * 16 * sizeof(Cx<F>);
}

// Transforms per tile of complex order P in its persistent class.
template <int... Ps>
constexpr int mixed_tpc_impl(int P, std::integer_sequence<int, Ps...>) {
    int r = 0;
    ((r = (P == Ps ? (mixed_class(Ps) == 0 ? TileCfg<float, Ps, kC2CFwd, kMixedBlock>::TPC
                                           : TileCfg<float, Ps, kC2CFwd, kMixedLargeBlock>::TPC)
                   : r)),
     ...);
    return r;
}
constexpr int mixed_tpc(int P) { return mixed_tpc_impl(P, std::make_integer_sequence<int, kMixedTopP + 1>{}); }

// Launch one class over n_items tiles; the caller has zeroed *counter on `stream`.
template <typename F, int BLOCK, int MINP, int MAXP>
cudaError_t launch_mixed_class(const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                               cudaStream_t stream, int num_sms) {
    auto kern = mixed_kernel<F, BLOCK, MINP, MAXP>;
    constexpr size_t smem = mixed_smem<F, BLOCK>();
    static ResidentSlots slots;
    const int blocks_per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, BLOCK, smem); });
    if (n_items <= 0) return cudaSuccess;
    const int cap = num_sms * blocks_per_sm;
    kern<<<n_items < cap ? n_items : cap, BLOCK, smem, stream>>>(groups, items, n_items, counter);
    return cudaGetLastError();
}

template <typename F>
cudaError_t launch_mixed(int cls, const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                         cudaStream_t stream, int num_sms) {
    return cls == 0 ? launch_mixed_class<F, kMixedBlock, kMixedMinP, kMixedMaxP>(groups, items, n_items, counter,
                                                                                stream, num_sms)
                    : launch_mixed_class<F, kMixedLargeBlock, kMixedLargeMinP, kMixedLargeMaxP>(
                          groups, items, n_items, counter, stream, num_sms);
}

cudaError_t launch_mixed_f32(int cls, const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                             cudaStream_t stream, int num_sms);
cudaError_t launch_mixed_f64(int cls, const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                             cudaStream_t stream, int num_sms);

}  // namespace zlfft
