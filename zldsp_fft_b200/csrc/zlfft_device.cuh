// Device building blocks shared by every FFT kernel of libzlfft_cuda.
//
// Arithmetic follows the reference's rounding exactly: each MulAdd/NegMulAdd
// of the reference is one fma here, every other multiply is an explicitly
// rounded multiply (__fmul_rn/__dmul_rn), which the compiler never contracts
// into a neighbouring add. With the same twiddle bits, a plain-form kernel
// therefore reproduces the reference's micro-only Stockham output bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace zlfft {

template <typename F>
struct CxT;
template <>
struct CxT<float> {
    using type = float2;
};
template <>
struct CxT<double> {
    using type = double2;
};
template <typename F>
using Cx = typename CxT<F>::type;

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
// cp.async copies of 4, 8 or 16 bytes from global into shared memory
// (both addresses aligned to the size), grouped by commit and awaited by
// wait_all; the data is visible to the CTA after the wait and a barrier.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src) {
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async copies 4, 8 or 16 bytes");
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    const size_t g = __cvta_generic_to_global(gmem_src);
    if constexpr (BYTES == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(g), "n"(BYTES) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

template <typename C>
__device__ __forceinline__ C cx(decltype(C::x) r, decltype(C::x) i) {
    C c;
    c.x = r;
    c.y = i;
    return c;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
    return cx<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
    return cx<C>(a.x - b.x, a.y - b.y);
}
// a - i*b
template <typename C>
__device__ __forceinline__ C csub_i(C a, C b) {
    return cx<C>(a.x + b.y, a.y - b.x);
}
// a + i*b
template <typename C>
__device__ __forceinline__ C cadd_i(C a, C b) {
    return cx<C>(a.x - b.y, a.y + b.x);
}
// x * w: re = fma(-xi, wi, xr*wr), im = fma(xi, wr, xr*wi)
// (src/common/zldsp_fft_common_radix.hpp:114-115 of the reference).
template <typename C>
__device__ __forceinline__ C cmul_tw(C x, C w) {
    return cx<C>(fma_rn(-x.y, w.y, mul_rn(x.x, w.x)), fma_rn(x.y, w.x, mul_rn(x.x, w.y)));
}
// Swap re/im: the reference's backward transform is swap(DFT(swap(x)))
// (src/common/zldsp_fft_common_structure.hpp:47-95).
template <typename C>
__device__ __forceinline__ C cswap(C a) {
    return cx<C>(a.y, a.x);
}

// Radix-4 butterfly of the first Stockham pass (no twiddles), in place:
// a_q = x[j + q*N/4] in, a_m = DFT4 output m out
// (src/common/zldsp_fft_common_radix.hpp:192-238).
template <typename C>
__device__ __forceinline__ void bfly4_first(C& a0, C& a1, C& a2, C& a3) {
    const C t0 = cadd(a0, a2), t1 = csub(a0, a2);
    const C t2 = cadd(a1, a3), t3 = csub(a1, a3);
    a0 = cadd(t0, t2);
    a1 = csub_i(t1, t3);
    a2 = csub(t0, t2);
    a3 = cadd_i(t1, t3);
}

// Twiddled radix-4 DIT butterfly, in place (src/common/zldsp_fft_common_radix.hpp:103-156).
template <typename C>
__device__ __forceinline__ void bfly4_tw(C& a0, C& a1, C& a2, C& a3, C w1, C w2, C w3) {
    const C t1 = cmul_tw(a1, w1);
    const C t3 = cmul_tw(a3, w3);
    const C s2 = cadd(t1, t3), s3 = csub(t1, t3);
    const C t2 = cmul_tw(a2, w2);
    const C s0 = cadd(a0, t2), s1 = csub(a0, t2);
    a0 = cadd(s0, s2);
    a1 = csub_i(s1, s3);
    a2 = csub(s0, s2);
    a3 = cadd_i(s1, s3);
}

// Radix-8 butterfly of the first Stockham pass, in place: a_q = x[j + q*N/8]
// in, a_p = DFT8 output p out. The W8 factors use 1/sqrt(2) formed as the
// double quotient rounded to F (src/common/zldsp_fft_common_radix.hpp:495-568).
template <typename C>
__device__ __forceinline__ void bfly8_first(C* a) {
    using F = decltype(C::x);
    const F c = (F)(1.0 / 1.4142135623730951);
    const C t0 = cadd(a[0], a[4]), t1 = csub(a[0], a[4]);
    const C t2 = cadd(a[2], a[6]), t3 = csub(a[2], a[6]);
    const C y00 = cadd(t0, t2), y02 = csub(t0, t2);
    const C y01 = csub_i(t1, t3), y03 = cadd_i(t1, t3);
    const C u0 = cadd(a[1], a[5]), u1 = csub(a[1], a[5]);
    const C u2 = cadd(a[3], a[7]), u3 = csub(a[3], a[7]);
    const C y10 = cadd(u0, u2), y12 = csub(u0, u2);
    const C y11 = csub_i(u1, u3), y13 = cadd_i(u1, u3);
    const C v1 = cx<C>(mul_rn(y11.x + y11.y, c), mul_rn(y11.y - y11.x, c));
    const C v2 = cx<C>(y12.y, -y12.x);
    const C v3 = cx<C>(mul_rn(y13.y - y13.x, c), mul_rn(-(y13.x + y13.y), c));
    a[0] = cadd(y00, y10);
    a[1] = cadd(y01, v1);
    a[2] = cadd(y02, v2);
    a[3] = cadd(y03, v3);
    a[4] = csub(y00, y10);
    a[5] = csub(y01, v1);
    a[6] = csub(y02, v2);
    a[7] = csub(y03, v3);
}

template <typename C>
__device__ __forceinline__ void bfly2(C& a0, C& a1) {
    const C t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

// Twiddle W_N^t from the unified table T[t] = exp(-2*pi*i*t/N), t < 3N/4
// (a plain cached load: the table is shared by every CTA and stays in L1/L2;
// unlike the non-coherent path it is not hoisted across barriers).
template <typename C>
__device__ __forceinline__ C tw_load(const C* tw, uint32_t t) {
    return tw[t];
}

// ---------------------------------------------------------------- TMA bulk copies
// 1-D bulk copies global -> shared completed on an mbarrier (sm_90+ PTX,
// non-multicast). Waits are bounded: after kWaitLimit polls a wait reports
// failure instead of spinning forever.
constexpr uint32_t kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// 3-D tiled tensor copy global -> shared (no multicast), completed on an
// mbarrier. The map lives in kernel parameter space (__grid_constant__).
// Coordinates: x innermost; callers keep x * element size a multiple of 16 B.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
// 2-D tiled tensor copy shared -> global (no multicast), in this thread's
// current bulk group; bulk_commit closes the group, bulk_wait_read0 waits
// until every committed group has finished reading shared memory, and
// bulk_wait0 until every committed group has completed.
__device__ __forceinline__ void tma_store_2d(const void* map, int x, int y, const void* src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(smem_u32(src))
                 : "memory");
}
// As tma_store_2d with an L2 cache-policy hint (createpolicy): keeps the
// stored lines in L2 for the next pass instead of streaming them out.
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void tma_store_2d_hint(const void* map, int x, int y, const void* src, uint64_t pol) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2}], [%3], %4;" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(smem_u32(src)), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses of shared memory. Every thread that read a
// staging buffer executes it before the barrier after which the buffer is
// refilled by TMA; without it a read still in flight may observe the refill.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the given phase parity; false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Drops one 128-byte line of global memory from L2 without writing it back
// (its contents become undefined): for intermediates that no later kernel
// reads, so that the dead data does not cost DRAM write bandwidth when L2
// evicts it. The address must be 128-byte aligned.
__device__ __forceinline__ void discard_l2_line(const void* p) {
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

// Device error word bits (read back by the host with zlfft_plan_device_status).
constexpr int kDevErrWaitTimeout = 1;

}  // namespace zlfft
