// G7: one persistent launch for a mixed batch of transforms of many orders.
//
// A mixed batch (thousands of transforms of uneven order, CFFT and RFFT
// mixed) is grouped on the host by (kind, order, operation);
// each group is cut into tiles of the tile kernel's shape (TPC transforms of
// one order, 128 threads). All tiles of all groups with orders that fit a
// 128-thread CTA (complex orders <= 11) form one work list, sorted longest
// first; resident CTAs pull tiles from it through an atomic counter and run
// the same TileWorker body as tile_kernel on gathered per-transform pointers.
// The grid is sized to the resident capacity, so the launch stays persistent
// and load-balanced across orders whose costs differ by 2^10.
#pragma once

#include "zlfft_resident.cuh"
#include "zlfft_tile.cuh"

namespace zlfft {

constexpr int kMixedMinP = 2;   // smallest complex order in the persistent kernel
constexpr int kMixedMaxP = 11;  // largest: T <= 128 threads per transform
constexpr int kMixedBlock = 128;

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

template <typename F, int OP, int P>
__device__ __forceinline__ bool mixed_try(int code, const MixedGroup& g, int tile, unsigned char* smem) {
    if (code != mixed_code(OP, P)) return false;
    TileWorker<F, P, OP, kAoS, kAoS, kMixedBlock, true> w(g.a, smem);
    w.run(g.a, tile, false, []() {});
    return true;
}

template <typename F, int OP, int... Ps>
__device__ __forceinline__ bool mixed_try_op(int code, const MixedGroup& g, int tile, unsigned char* smem,
                                             std::integer_sequence<int, Ps...>) {
    return (mixed_try<F, OP, kMixedMinP + Ps>(code, g, tile, smem) || ...);
}

// Resident CTAs per SM: 128 registers per thread. The union of all order and
// operation variants in one body spills heavily at 96 (5 CTAs), little at 128.
template <typename F>
constexpr int mixed_minb() { return 4; }

template <typename F>
__global__ void __launch_bounds__(kMixedBlock, mixed_minb<F>())
    mixed_kernel(const MixedGroup* __restrict__ groups, const MixedItem* __restrict__ items, int n_items,
                 int* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    using Ps = std::make_integer_sequence<int, kMixedMaxP - kMixedMinP + 1>;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const MixedItem item = items[it];
        const MixedGroup& g = groups[item.group];
        const int code = g.code;
        mixed_try_op<F, kC2CFwd>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kC2CBwd>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kR2CFwd>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kR2CSqrMag>(code, g, item.tile, smem_raw, Ps{}) ||
            mixed_try_op<F, kC2RBwd>(code, g, item.tile, smem_raw, Ps{});
        __syncthreads();  // shared memory and s_item are reused by the next tile
    }
}

// Shared memory of the persistent kernel: the largest tile of the covered orders.
template <typename F>
constexpr size_t mixed_smem() {
    // TPC * N complex values; for T <= 128 this is 128 * E = 2048 points
    return (size_t)kMixedBlock * 16 * sizeof(Cx<F>);
}

// Transforms per tile of order P in the persistent kernel.
template <int... Ps>
constexpr int mixed_tpc_impl(int P, std::integer_sequence<int, Ps...>) {
    int r = 0;
    ((r = (P == Ps ? TileCfg<float, Ps, kC2CFwd, kMixedBlock>::TPC : r)), ...);
    return r;
}
constexpr int mixed_tpc(int P) { return mixed_tpc_impl(P, std::make_integer_sequence<int, kMixedMaxP + 1>{}); }

// Launch over n_items tiles; the caller has zeroed *counter on `stream`.
template <typename F>
cudaError_t launch_mixed(const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                         cudaStream_t stream, int num_sms) {
    auto kern = mixed_kernel<F>;
    constexpr size_t smem = mixed_smem<F>();
    static ResidentSlots slots;
    const int blocks_per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, kMixedBlock, smem); });
    if (n_items <= 0) return cudaSuccess;
    const int cap = num_sms * blocks_per_sm;
    kern<<<n_items < cap ? n_items : cap, kMixedBlock, smem, stream>>>(groups, items, n_items, counter);
    return cudaGetLastError();
}

cudaError_t launch_mixed_f32(const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                             cudaStream_t stream, int num_sms);
cudaError_t launch_mixed_f64(const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                             cudaStream_t stream, int num_sms);

}  // namespace zlfft
