// Tensor-core building blocks (sm_100a tcgen05) for the split-precision form.
//
// A radix-16 DFT stage over 128 butterflies is one dense real contraction
//   D[128 x 32] = A[128 x 32] * B[32 x 32]
// with A's row r = the 16 complex inputs of butterfly r as (re, im) pairs and
// B the real form of the 16-point DFT matrix F (F[q][m] = exp(-2 pi i qm/16)):
//   B[2m][2q] = Re F, B[2m+1][2q] = -Im F, B[2m][2q+1] = Im F, B[2m+1][2q+1] = Re F,
// so D's row r holds the 16 outputs (re, im) of butterfly r.
//
// Split precision: every FP32 value v is carried as hi = fp16(v) and
// lo = fp16(v - hi), and the product uses the three significant terms
//   A*B ~ Ahi*Bhi + Alo*Bhi + Ahi*Blo
// accumulated in FP32 in tensor memory. A row in shared memory is 128 bytes,
// [hi: 32 halves | lo: 32 halves]; B rows the same with Bhi | Blo. Both use the
// 128-byte swizzled K-major canonical layout (16-byte chunk c of row r stored
// at chunk c ^ (r % 8); 8-row groups 1024 bytes apart; tile bases 1024-byte
// aligned). One MMA instruction covers K = 16 halves (32 bytes), so the
// six K-steps are (A chunk pair, B chunk pair): (0,0) (1,1) (2,0) (3,1) (0,2) (1,3)
// in 32-byte units of the row.
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

#include "zlfft_device.cuh"

namespace zlfft {
namespace tc {

// Shared-memory matrix descriptor: 128-byte swizzle, K-major, 8-row groups
// 1024 bytes apart (stride byte offset), leading byte offset unused (1),
// descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t smem_addr) {
    return (uint64_t)((smem_addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: FP16 A and B (K-major), FP32 D.
__host__ __device__ constexpr uint32_t idesc_f16_f32(int M, int N) {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {  // whole warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {  // whole warp
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // whole warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D (+)= A * B, issued by one thread.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive 32-bit columns of this thread's TMEM lane (32x32b shape: the
// warp reads lanes 32*(warp % 4) .. +31 of the address's column range).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// hi/lo halves of one FP32 value
__device__ __forceinline__ void split_hl(float v, __half& hi, __half& lo) {
    hi = __float2half_rn(v);
    lo = __float2half_rn(v - __half2float(hi));
}

// Packs the (re, im) pairs of two complex values into 16 bytes worth of
// halves: returns hi and lo words for complex values a and b (4 halves each).
struct HL2 {
    uint2 hi, lo;
};
__device__ __forceinline__ HL2 split_pair(float2 a, float2 b) {
    __half h0, l0, h1, l1, h2, l2, h3, l3;
    split_hl(a.x, h0, l0);
    split_hl(a.y, h1, l1);
    split_hl(b.x, h2, l2);
    split_hl(b.y, h3, l3);
    HL2 r;
    r.hi.x = (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
    r.hi.y = (uint32_t)__half_as_ushort(h2) | ((uint32_t)__half_as_ushort(h3) << 16);
    r.lo.x = (uint32_t)__half_as_ushort(l0) | ((uint32_t)__half_as_ushort(l1) << 16);
    r.lo.y = (uint32_t)__half_as_ushort(l2) | ((uint32_t)__half_as_ushort(l3) << 16);
    return r;
}

// Byte offset of 16-byte chunk c of row r in a 128-byte swizzled tile.
__device__ __forceinline__ uint32_t sw128_off(uint32_t r, uint32_t c) { return r * 128u + ((c ^ (r & 7u)) << 4); }

// The 32x32 real DFT-16 matrix as K-major rows n (output component) of
// [Bhi: 32 halves | Blo: 32 halves], rows swizzled. `tw16` holds
// exp(-2 pi i t/16), t = 0..15, in FP32 (values of the plan's twiddle table).
// Called by all threads of the block; writes 32 rows x 128 bytes.
__device__ __forceinline__ void build_dft16_b(unsigned char* b_tile, const float2* tw16) {
    for (int e = (int)threadIdx.x; e < 32 * 32; e += (int)blockDim.x) {
        const int n = e / 32, kk = e % 32;
        const int q = n >> 1, co = n & 1, m = kk >> 1, ci = kk & 1;
        const float2 w = tw16[(q * m) & 15];  // F[q][m] = w.x + i w.y
        float v;
        if (ci == 0) v = co == 0 ? w.x : w.y;    // B[2m][2q] = Re F, B[2m][2q+1] = Im F
        else v = co == 0 ? -w.y : w.x;           // B[2m+1][2q] = -Im F, B[2m+1][2q+1] = Re F
        __half hi, lo;
        split_hl(v, hi, lo);
        // half index kk in the hi part (chunk kk/8), and 32 + kk in the lo part
        __half* row = reinterpret_cast<__half*>(b_tile);
        row[(sw128_off((uint32_t)n, (uint32_t)(kk >> 3)) >> 1) + (kk & 7)] = hi;
        row[(sw128_off((uint32_t)n, (uint32_t)(4 + (kk >> 3))) >> 1) + (kk & 7)] = lo;
    }
}

// The six K-steps of one split-precision 128 x 32 x 32 product into d_tmem.
__device__ __forceinline__ void issue_split_dft16(uint32_t d_tmem, uint32_t a_addr, uint32_t b_addr) {
    constexpr uint32_t idesc = idesc_f16_f32(128, 32);
    const uint32_t ak[6] = {0, 1, 2, 3, 0, 1};
    const uint32_t bk[6] = {0, 1, 0, 1, 2, 3};
#pragma unroll
    for (int s = 0; s < 6; ++s)
        mma_f16(d_tmem, sw128_desc(a_addr + 32u * ak[s]), sw128_desc(b_addr + 32u * bk[s]), idesc, s > 0 ? 1u : 0u);
}

}  // namespace tc
}  // namespace zlfft
