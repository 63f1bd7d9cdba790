// G2: CTA-resident Stockham FFT ("tile" kernel), plain form, FP32 or FP64.
//
// One CTA holds TPC whole transforms of N = 2^P points. Each thread owns E
// points in registers and runs the reference's Stockham DIT stages on them:
// a radix-8 first pass for odd P (src/common/zldsp_fft_common_radix.hpp:477-657),
// a radix-4 first pass for even P (radix.hpp:170-239), then radix-4 passes
// with twiddles W_{4L}^{q k} (radix.hpp:78-158, :391-465). Two consecutive
// radix-4 stages run in registers as one radix-16 group; groups exchange data
// through padded shared memory in the Stockham (autosort) order, so a
// transform costs one HBM read and one HBM write.
//
// The RFFT epilogue/prologue of the reference (execute.hpp:318-368 forward
// split, :481-536 squared magnitude, :399-451 backward pre-step) is fused: the
// complex result stays in shared memory and the split runs before the single
// HBM write (forward), or the pre-step writes shared memory before the first
// group (backward).
//
// Index algebra (Stockham): after the stages up to sub-length L, element k of
// sub-transform j sits at position j*L + k. A group of radix R = product of
// its stage radices starting at sub-length L is run by "butterfly" b (J = b/L,
// k = b%L, b < N/R): it reads positions b + rho*N/R and writes positions
// J*R*L + k + mu*L.
#pragma once

#include <utility>

#include "zlfft_device.cuh"

namespace zlfft {

enum Op : int { kC2CFwd = 0, kC2CBwd = 1, kR2CFwd = 2, kR2CSqrMag = 3, kC2RBwd = 4 };
enum Layout : int { kAoS = 0, kSoA = 1 };

struct Grp {
    int R;      // points per butterfly (product of the group's stage radices)
    int L;      // sub-transform length at group entry
    int first;  // contains the first (untwiddled) stage
    int nst;    // stages in the group (1 or 2)
};

// Stage structure of the reference for order P (src/common/zldsp_fft_common_init.hpp:193-206):
// odd P >= 3: radix-8 first pass, then (P-3)/2 radix-4 passes;
// even P >= 2: P/2 radix-4 passes (the first untwiddled); P == 1: one radix-2.
__host__ __device__ constexpr int tile_num_groups(int P) {
    if (P == 0) return 0;
    if (P == 1) return 1;
    const int rest = (P % 2) ? (P - 3) / 2 : (P / 2 >= 2 ? P / 2 - 2 : 0);
    return 1 + rest / 2 + rest % 2;
}

__host__ __device__ constexpr Grp tile_group(int P, int g) {
    if (P == 1) return Grp{2, 1, 1, 1};
    Grp g0{};
    int rest = 0, L = 1;
    if (P % 2) {
        g0 = Grp{8, 1, 1, 1};
        rest = (P - 3) / 2;
        L = 8;
    } else if (P / 2 >= 2) {
        g0 = Grp{16, 1, 1, 2};
        rest = P / 2 - 2;
        L = 16;
    } else {
        g0 = Grp{4, 1, 1, 1};
        rest = 0;
        L = 4;
    }
    if (g == 0) return g0;
    int idx = 1;
    while (rest >= 2) {
        if (idx == g) return Grp{16, L, 0, 2};
        L *= 16;
        rest -= 2;
        ++idx;
    }
    return Grp{4, L, 0, 1};
}

__host__ __device__ constexpr int tile_elems(int P) {
    int e = 1;
    for (int g = 0; g < tile_num_groups(P); ++g) {
        const int r = tile_group(P, g).R;
        e = r > e ? r : e;
    }
    return e;
}

__host__ __device__ constexpr int ilog2c(long long x) {
    int r = 0;
    while ((1LL << r) < x) ++r;
    return r;
}

struct TileArgs {
    const void* in0;
    const void* in1;
    void* out0;
    void* out1;
    long long batch;
    long long in_stride;   // in units of the loaded element (complex; R2C: complex pairs of reals)
    long long out_stride;  // in units of the stored element (complex, or real for sqr_mag)
    const void* tw;        // unified table, 3N/4 complex, N = 2^P
    const void* rwc;       // RFFT split twiddles 0.5*cos, k = 0..N/2
    const void* rws;       // RFFT split twiddles 0.5*sin + 0.5
};

template <typename F, int P>
struct TileCfg {
    using C = Cx<F>;
    static constexpr int N = 1 << P;
    static constexpr int E = tile_elems(P);
    static constexpr int T = N / E;  // threads per transform
    static constexpr int TPC = T >= 256 ? 1 : 256 / T;
    static constexpr int THREADS = T * TPC;
    static constexpr int NPAD = (int)SmemPad<C>::size(N);
    static constexpr size_t SMEM = (size_t)TPC * NPAD * sizeof(C);
    static constexpr int NG = tile_num_groups(P);
    // Register budget: enough resident CTAs for ~80 registers per thread.
    static constexpr int MINB = (65536 / (THREADS * 80)) > 0 ? (65536 / (THREADS * 80)) : 1;
};

// ---------------------------------------------------------------- global I/O
// A complex stream seen from one transform's base: AoS is one array of
// complex values, SoA two arrays of reals. Indices are 32-bit offsets from the
// base, so unrolled accesses become base + immediate addressing.
template <typename F, int LAYOUT>
struct CxIn {
    const void* p0;
    const void* p1;
    __device__ __forceinline__ CxIn(const void* a0, const void* a1, long long base) {
        if constexpr (LAYOUT == kAoS) {
            p0 = static_cast<const Cx<F>*>(a0) + base;
            p1 = nullptr;
        } else {
            p0 = static_cast<const F*>(a0) + base;
            p1 = static_cast<const F*>(a1) + base;
        }
    }
    __device__ __forceinline__ Cx<F> operator[](int i) const {
        if constexpr (LAYOUT == kAoS) {
            return __ldcs(static_cast<const Cx<F>*>(p0) + i);
        } else {
            return cx<Cx<F>>(__ldcs(static_cast<const F*>(p0) + i), __ldcs(static_cast<const F*>(p1) + i));
        }
    }
};

template <typename F, int LAYOUT>
struct CxOut {
    void* p0;
    void* p1;
    __device__ __forceinline__ CxOut(void* a0, void* a1, long long base) {
        if constexpr (LAYOUT == kAoS) {
            p0 = static_cast<Cx<F>*>(a0) + base;
            p1 = nullptr;
        } else {
            p0 = static_cast<F*>(a0) + base;
            p1 = static_cast<F*>(a1) + base;
        }
    }
    __device__ __forceinline__ void put(int i, Cx<F> v) const {
        if constexpr (LAYOUT == kAoS) {
            __stcs(static_cast<Cx<F>*>(p0) + i, v);
        } else {
            __stcs(static_cast<F*>(p0) + i, v.x);
            __stcs(static_cast<F*>(p1) + i, v.y);
        }
    }
};

// ---------------------------------------------------------------- group compute
// Runs the stages of a group (R points, entry sub-length L) on the R
// registers r[] of one butterfly with in-group index k (k < L).
// Output register s then holds output mu(s) (see group_mu).
template <int P, int R, int L, int FIRST, typename C>
__device__ __forceinline__ void group_compute(C* r, uint32_t k, const C* tw) {
    if constexpr (R == 2) {
        bfly2(r[0], r[1]);
    } else if constexpr (R == 8) {
        bfly8_first(r);
    } else if constexpr (R == 4) {
        if constexpr (FIRST) {
            bfly4_first(r[0], r[1], r[2], r[3]);
        } else {
            constexpr int s = P - ilog2c(4LL * L);
            const C w1 = tw_load(tw, (1u * k) << s), w2 = tw_load(tw, (2u * k) << s), w3 = tw_load(tw, (3u * k) << s);
            bfly4_tw(r[0], r[1], r[2], r[3], w1, w2, w3);
        }
    } else {  // R == 16: two radix-4 stages
        if constexpr (FIRST) {
#pragma unroll
            for (int a = 0; a < 4; ++a) bfly4_first(r[a], r[a + 4], r[a + 8], r[a + 12]);
        } else {
            constexpr int s = P - ilog2c(4LL * L);
            const C w1 = tw_load(tw, (1u * k) << s), w2 = tw_load(tw, (2u * k) << s), w3 = tw_load(tw, (3u * k) << s);
#pragma unroll
            for (int a = 0; a < 4; ++a) bfly4_tw(r[a], r[a + 4], r[a + 8], r[a + 12], w1, w2, w3);
        }
        constexpr int s2 = P - ilog2c(16LL * L);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const uint32_t kk = k + (uint32_t)(m * L);
            const C w1 = tw_load(tw, (1u * kk) << s2), w2 = tw_load(tw, (2u * kk) << s2),
                    w3 = tw_load(tw, (3u * kk) << s2);
            bfly4_tw(r[4 * m], r[4 * m + 1], r[4 * m + 2], r[4 * m + 3], w1, w2, w3);
        }
    }
}

// Output index mu of register slot s after a group.
__host__ __device__ constexpr int group_mu(const Grp G, int s) {
    return G.nst == 2 ? (s >> 2) + 4 * (s & 3) : s;
}

// ---------------------------------------------------------------- the kernel
template <typename F, int P, int OP, int IL, int OL>
__global__ void __launch_bounds__(TileCfg<F, P>::THREADS, TileCfg<F, P>::MINB) tile_kernel(const TileArgs a) {
    using Cfg = TileCfg<F, P>;
    using C = Cx<F>;
    using Pad = SmemPad<C>;
    constexpr int N = Cfg::N, E = Cfg::E, T = Cfg::T, TPC = Cfg::TPC, NG = Cfg::NG;
    constexpr bool kFwd = (OP == kC2CFwd || OP == kR2CFwd || OP == kR2CSqrMag);
    constexpr bool kR2C = (OP == kR2CFwd || OP == kR2CSqrMag);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lt = (int)threadIdx.x % T;
    const int slot = (int)threadIdx.x / T;
    C* sx = reinterpret_cast<C*>(smem_raw) + (size_t)slot * Cfg::NPAD;
    const C* tw = static_cast<const C*>(a.tw);

    for (long long tile = blockIdx.x; tile * TPC < a.batch; tile += gridDim.x) {
        const long long tr = tile * TPC + slot;
        const bool valid = tr < a.batch;
        const long long ibase = valid ? tr * a.in_stride : 0;
        const long long obase = valid ? tr * a.out_stride : 0;
        C v[E];

        // ------------------------------------------------ input
        if constexpr (OP == kC2RBwd) {
            // Backward RFFT pre-step into shared memory (execute.hpp:399-451).
            if (valid) {
                const F* rwc = static_cast<const F*>(a.rwc);
                const F* rws = static_cast<const F*>(a.rws);
                const CxIn<F, IL> in(a.in0, a.in1, ibase);
                for (int k = 1 + lt; k <= N / 2; k += T) {
                    const C x1 = in[k];
                    const C x2 = in[N - k];
                    const F c = rwc[k], s = rws[k];
                    const F si = x1.y + x2.y, dr = x1.x - x2.x;
                    const C zk = cx<C>(fma_rn(-dr, s, fma_rn(-si, c, x1.x)), fma_rn(dr, c, fma_rn(-si, s, x1.y)));
                    const C zm = cx<C>(fma_rn(dr, s, fma_rn(si, c, x2.x)), fma_rn(dr, c, fma_rn(-si, s, x2.y)));
                    if (k != N / 2) sx[Pad::idx(k)] = zk;
                    sx[Pad::idx(N - k)] = zm;
                }
                if (lt == 0) {
                    const C x0 = in[0];
                    const C xm = in[N];
                    sx[0] = cx<C>(mul_rn(x0.x + xm.x, (F)0.5), mul_rn(x0.x - xm.x, (F)0.5));
                }
            }
            __syncthreads();
            if constexpr (NG > 0) {
                constexpr Grp G0 = tile_group(P, 0);
#pragma unroll
                for (int u = 0; u < E / G0.R; ++u) {
                    const int b = lt + u * T;
#pragma unroll
                    for (int rho = 0; rho < G0.R; ++rho) v[u * G0.R + rho] = cswap(sx[Pad::idx(b + rho * (N / G0.R))]);
                }
            } else {
                v[0] = cswap(sx[0]);
            }
        } else {
            constexpr int IL2 = kR2C ? (int)kAoS : IL;
            const CxIn<F, IL2> in(a.in0, a.in1, ibase);
            if constexpr (NG > 0) {
                constexpr Grp G0 = tile_group(P, 0);
#pragma unroll
                for (int u = 0; u < E / G0.R; ++u) {
                    const int b = lt + u * T;
#pragma unroll
                    for (int rho = 0; rho < G0.R; ++rho) {
                        C x = valid ? in[b + rho * (N / G0.R)] : cx<C>((F)0, (F)0);
                        v[u * G0.R + rho] = kFwd ? x : cswap(x);
                    }
                }
            } else {
                C x = valid ? in[0] : cx<C>((F)0, (F)0);
                v[0] = kFwd ? x : cswap(x);
            }
        }

        // ------------------------------------------------ stage groups
        // Final complex results go to global memory (C2C, C2R) or, for the
        // forward RFFT, to shared memory for the split epilogue.
        constexpr int OL2 = (OP == kC2RBwd || OP == kR2CSqrMag) ? (int)kAoS : OL;
        const CxOut<F, OL2> out(a.out0, a.out1, obase);
        auto emit = [&](int pos, C val) {
            if constexpr (kR2C) {
                sx[Pad::idx(pos)] = val;
            } else {
                if (valid) out.put(pos, kFwd ? val : cswap(val));
            }
        };
        if constexpr (NG == 0) {
            emit(0, v[0]);
        } else {
            // Unrolled over groups through a constexpr index sequence.
            [&]<int... GI>(std::integer_sequence<int, GI...>) {
                (
                    [&] {
                        constexpr Grp G = tile_group(P, GI);
                        constexpr int NB = E / G.R;
                        if constexpr (GI > 0) {
                            // Read this group's inputs from the exchange buffer.
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = lt + u * T;
#pragma unroll
                                for (int rho = 0; rho < G.R; ++rho) v[u * G.R + rho] = sx[Pad::idx(b + rho * (N / G.R))];
                            }
                        }
#pragma unroll
                        for (int u = 0; u < NB; ++u) {
                            const int b = lt + u * T;
                            group_compute<P, G.R, G.L, G.first>(v + u * G.R, (uint32_t)(b % G.L), tw);
                        }
                        if constexpr (GI + 1 < NG) {
                            __syncthreads();
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = lt + u * T;
                                const int J = b / G.L, k = b % G.L;
#pragma unroll
                                for (int s = 0; s < G.R; ++s)
                                    sx[Pad::idx(J * G.R * G.L + k + group_mu(G, s) * G.L)] = v[u * G.R + s];
                            }
                            __syncthreads();
                        } else {
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = lt + u * T;  // J == 0 in the last group
#pragma unroll
                                for (int s = 0; s < G.R; ++s) emit(b + group_mu(G, s) * G.L, v[u * G.R + s]);
                            }
                        }
                    }(),
                    ...);
            }(std::make_integer_sequence<int, NG>{});
        }

        // ------------------------------------------------ RFFT forward split
        if constexpr (kR2C) {
            __syncthreads();
            if (valid) {
                const F* rwc = static_cast<const F*>(a.rwc);
                const F* rws = static_cast<const F*>(a.rws);
                for (int k = 1 + lt; k <= N / 2; k += T) {
                    const C z1 = sx[Pad::idx(k)], z2 = sx[Pad::idx(N - k)];
                    const F c = rwc[k], s = rws[k];
                    const F si = z1.y + z2.y, dr = z1.x - z2.x;
                    const F xr_k = fma_rn(-dr, s, fma_rn(si, c, z1.x));
                    const F xi_k = fma_rn(-dr, c, fma_rn(-si, s, z1.y));
                    const F xr_m = fma_rn(dr, s, fma_rn(-si, c, z2.x));
                    const F xi_m = fma_rn(-dr, c, fma_rn(-si, s, z2.y));
                    if constexpr (OP == kR2CFwd) {
                        if (k != N / 2) out.put(k, cx<C>(xr_k, xi_k));
                        out.put(N - k, cx<C>(xr_m, xi_m));
                    } else {
                        F* o = static_cast<F*>(a.out0) + obase;
                        if (k != N / 2) __stcs(o + k, fma_rn(xr_k, xr_k, mul_rn(xi_k, xi_k)));
                        __stcs(o + N - k, fma_rn(xr_m, xr_m, mul_rn(xi_m, xi_m)));
                    }
                }
                if (lt == 0) {
                    const C z0 = sx[0];
                    const F dc = z0.x + z0.y, ny = z0.x - z0.y;
                    if constexpr (OP == kR2CFwd) {
                        out.put(0, cx<C>(dc, (F)0));
                        out.put(N, cx<C>(ny, (F)0));
                    } else {
                        F* o = static_cast<F*>(a.out0) + obase;
                        __stcs(o, mul_rn(dc, dc));
                        __stcs(o + N, mul_rn(ny, ny));
                    }
                }
            }
        }
        __syncthreads();  // the exchange buffer is reused by the next tile
    }
}

}  // namespace zlfft
