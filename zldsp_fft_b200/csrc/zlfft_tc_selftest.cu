// Self-test of the tensor-core split-precision DFT-16 building block: one CTA
// computes 128 independent 16-point DFTs with tcgen05 MMAs (operands in
// shared memory, FP32 accumulators in tensor memory) so the host can check
// descriptors, swizzle and the tensor-memory protocol against FP64.
#include <cuda_runtime.h>

#include "zlfft_tc.cuh"

namespace zlfft {

constexpr size_t kTcSelftestSmem = 64 * 1024;  // A 16 KB + B 4 KB + barrier, with slack

__global__ void __launch_bounds__(128) tc_dft16_selftest_kernel(const float2* __restrict__ in,
                                                                  float2* __restrict__ out,
                                                                  const float2* __restrict__ tw16, int* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // the swizzle pattern is a function of the address bits: align the tiles to 1024 bytes
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    unsigned char* a_tile = smem;
    unsigned char* b_tile = smem + 16384;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 20480);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + 20488);
    const int r = (int)threadIdx.x;
    const int warp = r / 32;
    if (warp == 0) {
        tc::tmem_alloc(slot, 32);
        tc::tmem_relinquish();
    }
    if (r == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    // row r of A: the 16 inputs of butterfly r, split into hi | lo halves
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float2* x = in + r * 16 + 4 * c;
        const tc::HL2 p0 = tc::split_pair(x[0], x[1]);
        const tc::HL2 p1 = tc::split_pair(x[2], x[3]);
        *reinterpret_cast<uint4*>(a_tile + tc::sw128_off((uint32_t)r, (uint32_t)c)) =
            make_uint4(p0.hi.x, p0.hi.y, p1.hi.x, p1.hi.y);
        *reinterpret_cast<uint4*>(a_tile + tc::sw128_off((uint32_t)r, (uint32_t)(4 + c))) =
            make_uint4(p0.lo.x, p0.lo.y, p1.lo.x, p1.lo.y);
    }
    tc::build_dft16_b(b_tile, tw16);
    fence_proxy_async_smem();  // generic-proxy writes of A and B before the tensor core reads them
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    if (r == 0) {
        tc::issue_split_dft16(tmem, smem_u32(a_tile), smem_u32(b_tile));
        tc::mma_commit(bar);
    }
    const bool ok = mbar_wait(bar, 0);
    tc::fence_after_sync();
    if (__syncthreads_or(!ok)) {  // bounded wait ran out: report, give the MMAs a bounded chance, free TMEM
        if (r == 0) atomicOr(err, kDevErrWaitTimeout);
        mbar_wait(bar, 0);
        tc::fence_before_sync();
        __syncthreads();
        if (warp == 0) tc::tmem_dealloc(tmem, 32);
        return;
    }
    float v[32];
    tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16), v);
#pragma unroll
    for (int q = 0; q < 16; ++q) out[r * 16 + q] = make_float2(v[2 * q], v[2 * q + 1]);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 32);
}

cudaError_t tc_selftest_launch(const float2* in, float2* out, const float2* tw16, int* err, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(tc_dft16_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSelftestSmem);
    if (e != cudaSuccess) return e;
    tc_dft16_selftest_kernel<<<1, 128, kTcSelftestSmem, st>>>(in, out, tw16, err);
    return cudaGetLastError();
}

}  // namespace zlfft
