// Highway-API shim: TEST INFRASTRUCTURE ONLY.
//
// The reference (zldsp::fft) is header-only C++ written against Google
// Highway's SIMD API (src/common/zldsp_fft_common_init.hpp:3-4). Highway is
// not present in this environment, so this file supplies the subset of its
// public API that the reference names, written here from Highway's documented
// op semantics (not from Highway's sources). It lets the reference headers
// compile UNCHANGED from where they lie, so the oracle can run the reference's
// own algorithm on the CPU.
//
// Target modelled: x86 AVX2 + FMA ("-march=x86-64-v3"), i.e. full vectors of
// 256 bits (8 x float, 4 x double). Capped/fixed tags give 1..N lanes.
// Semantics that matter for correctness of the reference:
//   * InterleaveLower/Upper act independently on each 128-bit block.
//   * ConcatLowerLower/UpperUpper, Combine, Lower/UpperHalf act on halves of
//     the whole vector.
//   * MulAdd(m, x, a) = m*x + a and NegMulAdd(m, x, a) = a - m*x, each FUSED
//     (one rounding), as on Highway's AVX2 target.
// Every other op is a lane-wise IEEE operation. Build with -ffp-contract=off
// so that the compiler does not fuse a separate Mul and Add on its own.
#pragma once

#include <array>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "aligned_allocator.h"

#define HWY_NAMESPACE N_SHIM_AVX2
#define HWY_INLINE inline __attribute__((always_inline))
#define HWY_RESTRICT __restrict__
#define HWY_ALIGNMENT 64
#define HWY_ALIGN alignas(HWY_ALIGNMENT)
#define HWY_ASSUME_ALIGNED(ptr, align) __builtin_assume_aligned((ptr), (align))
#define HWY_ASSUME(expr)               \
    do {                               \
        if (!(expr)) __builtin_unreachable(); \
    } while (0)
#define HWY_SHIM_PRAGMA(tokens) _Pragma(#tokens)
#define HWY_UNROLL(factor) HWY_SHIM_PRAGMA(GCC unroll factor)

namespace hwy {
namespace HWY_NAMESPACE {

constexpr size_t kShimVectorBytes = 32;  // AVX2

template <typename T, size_t N>
struct Simd {
    using T_ = T;
    static constexpr size_t kLanes = N;
    constexpr Simd() = default;
};

template <typename T>
constexpr size_t ShimFullLanes() { return kShimVectorBytes / sizeof(T); }

template <typename T>
using ScalableTag = Simd<T, ShimFullLanes<T>()>;

template <typename T, size_t kLimit>
using CappedTag = Simd<T, (kLimit < ShimFullLanes<T>() ? kLimit : ShimFullLanes<T>())>;

template <typename T, size_t kNumLanes>
using FixedTag = Simd<T, kNumLanes>;

template <class D>
using TFromD = typename D::T_;

template <typename U, class D>
using Repartition =
    Simd<U, (D::kLanes * sizeof(TFromD<D>) / sizeof(U) > 0 ? D::kLanes * sizeof(TFromD<D>) / sizeof(U) : 1)>;

template <class D>
using Half = Simd<TFromD<D>, (D::kLanes / 2 > 0 ? D::kLanes / 2 : 1)>;

// A vector of N lanes of T: a GCC vector-extension value, so lane-wise
// arithmetic compiles to SIMD instructions.
template <typename T, size_t N>
struct VecN {
    typedef T raw_t __attribute__((vector_size(N * sizeof(T))));
    raw_t raw;
};

template <class D>
using Vec = VecN<TFromD<D>, D::kLanes>;

template <class D>
constexpr size_t MaxLanes(D) { return D::kLanes; }

template <class D>
constexpr size_t Lanes(D) { return D::kLanes; }

// ---------------------------------------------------------------- load/store
template <class D>
HWY_INLINE Vec<D> LoadU(D, const TFromD<D>* HWY_RESTRICT p) {
    Vec<D> v;
    std::memcpy(&v.raw, p, sizeof(v.raw));
    return v;
}

template <class D>
HWY_INLINE Vec<D> Load(D d, const TFromD<D>* HWY_RESTRICT p) {
    return LoadU(d, p);
}

template <class D>
HWY_INLINE void StoreU(const Vec<D> v, D, TFromD<D>* HWY_RESTRICT p) {
    std::memcpy(p, &v.raw, sizeof(v.raw));
}

template <class D>
HWY_INLINE void Store(const Vec<D> v, D d, TFromD<D>* HWY_RESTRICT p) {
    StoreU(v, d, p);
}

template <class D>
HWY_INLINE Vec<D> Set(D, const TFromD<D> x) {
    Vec<D> v;
    for (size_t i = 0; i < D::kLanes; ++i) v.raw[i] = x;
    return v;
}

// ---------------------------------------------------------------- arithmetic
template <typename T, size_t N>
HWY_INLINE VecN<T, N> Add(const VecN<T, N> a, const VecN<T, N> b) { return {a.raw + b.raw}; }

template <typename T, size_t N>
HWY_INLINE VecN<T, N> Sub(const VecN<T, N> a, const VecN<T, N> b) { return {a.raw - b.raw}; }

template <typename T, size_t N>
HWY_INLINE VecN<T, N> Mul(const VecN<T, N> a, const VecN<T, N> b) { return {a.raw * b.raw}; }

template <typename T, size_t N>
HWY_INLINE VecN<T, N> Neg(const VecN<T, N> a) { return {-a.raw}; }

HWY_INLINE float ShimFma(float a, float b, float c) { return __builtin_fmaf(a, b, c); }
HWY_INLINE double ShimFma(double a, double b, double c) { return __builtin_fma(a, b, c); }

// m * x + a, one rounding.
template <typename T, size_t N>
HWY_INLINE VecN<T, N> MulAdd(const VecN<T, N> m, const VecN<T, N> x, const VecN<T, N> a) {
    VecN<T, N> r;
    for (size_t i = 0; i < N; ++i) r.raw[i] = ShimFma(m.raw[i], x.raw[i], a.raw[i]);
    return r;
}

// a - m * x, one rounding.
template <typename T, size_t N>
HWY_INLINE VecN<T, N> NegMulAdd(const VecN<T, N> m, const VecN<T, N> x, const VecN<T, N> a) {
    VecN<T, N> r;
    for (size_t i = 0; i < N; ++i) r.raw[i] = ShimFma(-m.raw[i], x.raw[i], a.raw[i]);
    return r;
}

// ---------------------------------------------------------------- shuffles
// Lanes per 128-bit block for element type T within a vector of N lanes.
template <typename T, size_t N>
constexpr size_t ShimBlockLanes() {
    return (N * sizeof(T) > 16) ? 16 / sizeof(T) : N;
}

// Per 128-bit block: lower halves of a and b, interleaved (a first).
// A one-lane vector has no pairs to interleave and returns a.
template <class D>
HWY_INLINE Vec<D> InterleaveLower(D, const Vec<D> a, const Vec<D> b) {
    using T = TFromD<D>;
    constexpr size_t N = D::kLanes;
    constexpr size_t B = ShimBlockLanes<T, N>();
    if constexpr (B == 1) {
        return a;
    } else {
        Vec<D> r;
        for (size_t blk = 0; blk < N; blk += B) {
            for (size_t i = 0; i < B / 2; ++i) {
                r.raw[blk + 2 * i] = a.raw[blk + i];
                r.raw[blk + 2 * i + 1] = b.raw[blk + i];
            }
        }
        return r;
    }
}

// Per 128-bit block: upper halves of a and b, interleaved (a first).
template <class D>
HWY_INLINE Vec<D> InterleaveUpper(D, const Vec<D> a, const Vec<D> b) {
    using T = TFromD<D>;
    constexpr size_t N = D::kLanes;
    constexpr size_t B = ShimBlockLanes<T, N>();
    Vec<D> r;
    for (size_t blk = 0; blk < N; blk += B) {
        for (size_t i = 0; i < B / 2; ++i) {
            r.raw[blk + 2 * i] = a.raw[blk + B / 2 + i];
            r.raw[blk + 2 * i + 1] = b.raw[blk + B / 2 + i];
        }
    }
    return r;
}

// Result: lower half = lower half of lo, upper half = lower half of hi.
template <class D>
HWY_INLINE Vec<D> ConcatLowerLower(D, const Vec<D> hi, const Vec<D> lo) {
    constexpr size_t N = D::kLanes;
    Vec<D> r;
    for (size_t i = 0; i < N / 2; ++i) {
        r.raw[i] = lo.raw[i];
        r.raw[N / 2 + i] = hi.raw[i];
    }
    return r;
}

// Result: lower half = upper half of lo, upper half = upper half of hi.
template <class D>
HWY_INLINE Vec<D> ConcatUpperUpper(D, const Vec<D> hi, const Vec<D> lo) {
    constexpr size_t N = D::kLanes;
    Vec<D> r;
    for (size_t i = 0; i < N / 2; ++i) {
        r.raw[i] = lo.raw[N / 2 + i];
        r.raw[N / 2 + i] = hi.raw[N / 2 + i];
    }
    return r;
}

template <class DH, typename T, size_t N>
HWY_INLINE Vec<DH> LowerHalf(DH, const VecN<T, N> v) {
    static_assert(DH::kLanes * 2 == N, "LowerHalf: tag must be half of the vector");
    Vec<DH> r;
    for (size_t i = 0; i < DH::kLanes; ++i) r.raw[i] = v.raw[i];
    return r;
}

template <class DH, typename T, size_t N>
HWY_INLINE Vec<DH> UpperHalf(DH, const VecN<T, N> v) {
    static_assert(DH::kLanes * 2 == N, "UpperHalf: tag must be half of the vector");
    Vec<DH> r;
    for (size_t i = 0; i < DH::kLanes; ++i) r.raw[i] = v.raw[DH::kLanes + i];
    return r;
}

// Full vector with lower half = lo and upper half = hi.
template <class D>
HWY_INLINE Vec<D> Combine(D, const Vec<Half<D>> hi, const Vec<Half<D>> lo) {
    constexpr size_t N = D::kLanes;
    Vec<D> r;
    for (size_t i = 0; i < N / 2; ++i) {
        r.raw[i] = lo.raw[i];
        r.raw[N / 2 + i] = hi.raw[i];
    }
    return r;
}

template <class D, typename T, size_t N>
HWY_INLINE Vec<D> BitCast(D, const VecN<T, N> v) {
    static_assert(sizeof(Vec<D>) == sizeof(VecN<T, N>), "BitCast: size mismatch");
    Vec<D> r;
    std::memcpy(&r.raw, &v.raw, sizeof(r.raw));
    return r;
}

template <class D>
HWY_INLINE Vec<D> Reverse(D, const Vec<D> v) {
    constexpr size_t N = D::kLanes;
    Vec<D> r;
    for (size_t i = 0; i < N; ++i) r.raw[i] = v.raw[N - 1 - i];
    return r;
}

// a = p[0], p[2], ...; b = p[1], p[3], ...
template <class D>
HWY_INLINE void LoadInterleaved2(D, const TFromD<D>* HWY_RESTRICT p, Vec<D>& a, Vec<D>& b) {
    for (size_t i = 0; i < D::kLanes; ++i) {
        a.raw[i] = p[2 * i];
        b.raw[i] = p[2 * i + 1];
    }
}

template <class D>
HWY_INLINE void StoreInterleaved2(const Vec<D> a, const Vec<D> b, D, TFromD<D>* HWY_RESTRICT p) {
    for (size_t i = 0; i < D::kLanes; ++i) {
        p[2 * i] = a.raw[i];
        p[2 * i + 1] = b.raw[i];
    }
}

template <class D>
HWY_INLINE void StoreInterleaved4(const Vec<D> v0, const Vec<D> v1, const Vec<D> v2, const Vec<D> v3, D,
                                  TFromD<D>* HWY_RESTRICT p) {
    for (size_t i = 0; i < D::kLanes; ++i) {
        p[4 * i] = v0.raw[i];
        p[4 * i + 1] = v1.raw[i];
        p[4 * i + 2] = v2.raw[i];
        p[4 * i + 3] = v3.raw[i];
    }
}

}  // namespace HWY_NAMESPACE
}  // namespace hwy
