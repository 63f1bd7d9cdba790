// G2: CTA-resident Stockham FFT ("tile" kernel), plain form, FP32 or FP64.
//
// One CTA holds TPC whole transforms of N = 2^P points. Each thread owns E
// points in registers and runs the reference's Stockham DIT stages on them:
// a radix-8 first pass for odd P (src/common/zldsp_fft_common_radix.hpp:477-657),
// a radix-4 first pass for even P (radix.hpp:170-239), then radix-4 passes
// with twiddles W_{4L}^{q k} (radix.hpp:78-158, :391-465). Consecutive
// radix-4 stages run in registers as radix-16 groups; groups exchange data
// through XOR-swizzled shared memory in the Stockham (autosort) order, so a
// transform costs one HBM read and one HBM write.
//
// Group order: the first (untwiddled) stage group, then a lone radix-4 stage
// when the count of remaining radix-4 stages is odd, then radix-16 groups.
// The last group is therefore radix-16 with one butterfly per thread, and
// its twiddles depend on the thread only: they are loaded into registers
// once per CTA and reused for every transform the CTA processes.
//
// The RFFT epilogue of the reference (execute.hpp:318-368 forward split,
// :481-536 squared magnitude) is fused after the last group without another
// shared-memory pass: bins k and N-k live in two adjacent lanes (a mirrored
// thread order), which exchange them with one warp shuffle. The backward
// pre-step (execute.hpp:399-451) writes shared memory before the first group.
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
    int rest;
    if (P % 2) {
        rest = (P - 3) / 2;
    } else {
        const int n4 = P / 2;
        rest = (n4 % 2 == 1) ? n4 - 1 : n4 - 2;
    }
    return 1 + rest % 2 + rest / 2;
}

__host__ __device__ constexpr Grp tile_group(int P, int g) {
    if (P == 1) return Grp{2, 1, 1, 1};
    Grp g0{};
    int rest = 0, L = 1;
    if (P % 2) {
        g0 = Grp{8, 1, 1, 1};
        rest = (P - 3) / 2;
        L = 8;
    } else if ((P / 2) % 2 == 1) {
        g0 = Grp{4, 1, 1, 1};
        rest = P / 2 - 1;
        L = 4;
    } else {
        g0 = Grp{16, 1, 1, 2};
        rest = P / 2 - 2;
        L = 16;
    }
    if (g == 0) return g0;
    int idx = 1;
    if (rest % 2 == 1) {
        if (g == 1) return Grp{4, L, 0, 1};
        L *= 4;
        rest -= 1;
        idx = 2;
    }
    while (idx < g) {
        L *= 16;
        ++idx;
    }
    return Grp{16, L, 0, 2};
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
    const void* tws;       // per-stage tables (see stage_tw_offset), same values as tw
    const void* rw;        // RFFT split twiddles (0.5*cos, 0.5*sin + 0.5) pairs, k = 0..N/2
    int* err;              // device error word (kDevErrWaitTimeout on a timed-out wait)
    int tma;               // inputs qualify for bulk copies (16-byte aligned bases and strides)
    // Gathered transforms (mixed batches): when gin0 is set, transform t reads
    // from gin0[t] (and gin1[t] for split SoA) and writes to gout0[t] (gout1[t]);
    // the strides are then unused.
    const void* const* gin0;
    const void* const* gin1;
    void* const* gout0;
    void* const* gout1;
    // Gathered multi-pass transforms: one input tensor map (CUtensorMap, in
    // device memory) per transform for the first pass's bulk copies, or null.
    const void* gmaps;
    // RFFT forward only: window multiplied into every frame as it is loaded
    // (the STFT front end); pairs (w[2i], w[2i+1]) per complex-pair input.
    const void* win;
};

// Output sink of the backward RFFT's last group. NoSink: the transform's
// samples go to the output array. A sink with kActive (the overlap-add of
// zlfft_istft.cuh) receives them instead, as add(pos, x) with x = real samples
// 2 pos and 2 pos + 1, and may carry a spectral filter h (N + 1 bins,
// multiplied into the bins as the pre-step reads them; null: none).
struct NoSink {
    static constexpr bool kActive = false;
    const void* h = nullptr;
};

// Complex product with each operation rounded on its own:
// (x.re h.re - x.im h.im, x.re h.im + x.im h.re).
template <typename C>
__device__ __forceinline__ C cmul_rn(const C x, const C h) {
    return cx<C>(sub_rn(mul_rn(x.x, h.x), mul_rn(x.y, h.y)), add_rn(mul_rn(x.x, h.y), mul_rn(x.y, h.x)));
}

template <typename F, int P, int OP = kC2CFwd, int BLOCK = 128, int EM = 0>
struct TileCfg {
    using C = Cx<F>;
    static constexpr int N = 1 << P;
    // points per thread: the largest group radix; order 14 takes two radix-16
    // butterflies per thread per group (512 threads for 16384 points); EM > 0
    // sets it (a multiple of the largest group radix)
    static constexpr int E = EM > 0 ? EM : (P == 14 ? 2 * tile_elems(P) : tile_elems(P));
    static_assert(E % tile_elems(P) == 0 || P == 0, "points per thread: a multiple of the largest group radix");
    static constexpr int T = N / E;  // threads per transform
    static constexpr int TPC = T >= BLOCK ? 1 : BLOCK / T;
    static constexpr int THREADS = T * TPC;
    static constexpr size_t XBYTES = (size_t)TPC * N * sizeof(C);  // exchange buffer
    // Register budget: enough resident CTAs for ~96 registers per thread in
    // FP32 (the last group's 15 complex twiddles stay in registers), ~128 in FP64.
    static constexpr int REGS = sizeof(F) == 4 ? (((OP == kC2CFwd || OP == kC2CBwd) && P >= 10) ? 128 : 96) : 128;
    // Staging buffer for the next tile's input, filled by TMA bulk copies
    // while the current tile computes (not for the RFFT backward, whose
    // pre-step reads the bins).
    static constexpr bool kTMA = P >= 4 && OP != kC2RBwd && 2 * XBYTES <= 200 * 1024;
    // Backward RFFT: the next tile's bins (TPC frames of N + 1 complex; SoA:
    // a re row then an im row per frame) are copied into the staging buffer
    // by cp.async while the current tile computes (dense bin arrays put odd
    // frames off the 16-byte alignment bulk copies need). Measured per order
    // (FP32, GB/s, AoS): complex order 9: 2848 -> 3210, 11: 2879 -> 3300,
    // 12: 2214 -> 2986, 13: 1848 -> 2346; but 8: 4533 -> 3770 and 10: 3910 ->
    // 3482, where the extra copy and shared-memory read outweigh the hidden
    // latency. FP64 keeps direct loads (its buffers would cost resident CTAs).
    static constexpr size_t BBYTES = ((size_t)TPC * (N + 1) * sizeof(C) + 15) / 16 * 16;
    static constexpr bool kStageBins = OP == kC2RBwd && sizeof(F) == 4 && (P == 9 || (P >= 11 && P <= 13)) &&
                                       XBYTES + BBYTES <= 200 * 1024;
    // 128 KB tiles (FP32 order 14, FP64 order 13: no room for a second
    // buffer): the next tile's input lands by TMA in the exchange buffer
    // itself, once the last group has read it, while the last group computes
    // and stores. For the forward RFFT only where the split runs in registers
    // (the shuffle epilogue of TileWorker: last group radix 16 = E), so the
    // buffer is free after the last group's reads.
    static constexpr int NG_ = tile_num_groups(P);
    static constexpr Grp GL_ = tile_group(P, NG_ > 0 ? NG_ - 1 : 0);
    static constexpr bool kShufSplit = (OP == kR2CFwd || OP == kR2CSqrMag) && NG_ >= 2 && GL_.R == E && !GL_.first &&
                                       GL_.R == 16 && T >= 2;
    static constexpr bool kTMA1 = !kTMA && (P == 14 || (sizeof(F) == 8 && P == 13)) &&
                                  (OP == kC2CFwd || OP == kC2CBwd || kShufSplit) && XBYTES + 16 <= 200 * 1024;
    static constexpr size_t SMEM = kTMA ? 2 * XBYTES + 16 : (kTMA1 ? XBYTES + 16 : XBYTES + (kStageBins ? BBYTES : 0));
    static constexpr int NG = tile_num_groups(P);
    static constexpr int MINB = (65536 / (THREADS * REGS)) > 0 ? (65536 / (THREADS * REGS)) : 1;
};

// XOR swizzle of a shared-memory slot index: keeps each 128-byte row, permutes
// the slots inside it so the strided Stockham writes and the unit-stride reads
// hit distinct banks (checked by simulation for every exchange of every order).
template <typename C>
__device__ __forceinline__ uint32_t swz(uint32_t p) {
    if constexpr (sizeof(C) == 8) {
        return p ^ (((p >> 4) ^ (p >> 7)) & 15u);
    } else {
        return p ^ (((p >> 3) + (p >> 6)) & 7u);
    }
}

// Swizzle of the exchange that feeds a mirrored last group (RFFT forward): its
// reads are two runs of 16 consecutive slots, one of them offset by one slot
// from a 128-byte row, so only the writer's run blocks (LW consecutive slots,
// LW rows apart) are separated, by XOR of whole LW-slot blocks. Checked by
// simulation to be conflict-free for the orders that use it (8, 10, 11, 12, 14).
template <typename C, int LW>
__device__ __forceinline__ uint32_t swz_mirror(uint32_t p) {
    if constexpr (sizeof(C) != 8 || LW >= 16) {
        return sizeof(C) == 8 ? p : swz<C>(p);
    } else {
        const uint32_t r = p >> 4;
        return p ^ (((r / LW) & (16u / LW - 1u)) * LW);
    }
}

// Per-stage twiddle tables: the radix-4 stage with sub-length L (twiddles
// W_{4L}^{qk}, q = 1..3, k < L) occupies 3L consecutive entries at offset
// L - L0, q-major, where L0 is the first twiddled stage's sub-length (4 for
// even orders, 8 for odd). Threads with consecutive k read consecutive
// entries. The values are copies of the unified table's entries.
__host__ __device__ constexpr int stage_l0(int P) { return (P % 2) ? 8 : 4; }

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
// Twiddles of a group for in-group index k: radix-4 non-first: w[0..2] =
// W_{4L}^{qk}; radix-16 non-first: w[0..2] (stage A) then w[3+3m+(q-1)] =
// W_{16L}^{q(k+mL)} (stage B, m = 0..3); radix-16 first: stage B only.
template <int P, int R, int L, int FIRST>
__host__ __device__ constexpr int group_tw_count() {
    return R == 4 ? (FIRST ? 0 : 3) : R == 16 ? (FIRST ? 12 : 15) : 0;
}

template <int P, int R, int L, int FIRST, typename C>
__device__ __forceinline__ void group_load_tw(const C* tw, uint32_t k, C* w) {
    if constexpr (R == 4 && !FIRST) {
        constexpr int s = P - ilog2c(4LL * L);
        w[0] = tw_load(tw, (1u * k) << s);
        w[1] = tw_load(tw, (2u * k) << s);
        w[2] = tw_load(tw, (3u * k) << s);
    } else if constexpr (R == 16) {
        constexpr int o = FIRST ? 0 : 3;
        if constexpr (!FIRST) {
            constexpr int s = P - ilog2c(4LL * L);
            w[0] = tw_load(tw, (1u * k) << s);
            w[1] = tw_load(tw, (2u * k) << s);
            w[2] = tw_load(tw, (3u * k) << s);
        }
        constexpr int s2 = P - ilog2c(16LL * L);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const uint32_t kk = k + (uint32_t)(m * L);
            w[o + 3 * m + 0] = tw_load(tw, (1u * kk) << s2);
            w[o + 3 * m + 1] = tw_load(tw, (2u * kk) << s2);
            w[o + 3 * m + 2] = tw_load(tw, (3u * kk) << s2);
        }
    }
}

// Runs the stages of a group on the R registers r[] of one butterfly.
// Output register s then holds output mu(s) (see group_mu).
template <int R, int FIRST, typename C>
__device__ __forceinline__ void group_compute(C* r, const C* w) {
    if constexpr (R == 2) {
        bfly2(r[0], r[1]);
    } else if constexpr (R == 8) {
        bfly8_first(r);
    } else if constexpr (R == 4) {
        if constexpr (FIRST) {
            bfly4_first(r[0], r[1], r[2], r[3]);
        } else {
            bfly4_tw(r[0], r[1], r[2], r[3], w[0], w[1], w[2]);
        }
    } else {  // R == 16: two radix-4 stages
        constexpr int o = FIRST ? 0 : 3;
        if constexpr (FIRST) {
#pragma unroll
            for (int a = 0; a < 4; ++a) bfly4_first(r[a], r[a + 4], r[a + 8], r[a + 12]);
        } else {
#pragma unroll
            for (int a = 0; a < 4; ++a) bfly4_tw(r[a], r[a + 4], r[a + 8], r[a + 12], w[0], w[1], w[2]);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m)
            bfly4_tw(r[4 * m], r[4 * m + 1], r[4 * m + 2], r[4 * m + 3], w[o + 3 * m], w[o + 3 * m + 1],
                     w[o + 3 * m + 2]);
    }
}

// As group_compute, loading each butterfly's twiddles from the table right
// before use (short live ranges; used where the twiddles are not held in
// registers across transforms).
template <int P, int R, int L, int FIRST, typename C>
__device__ __forceinline__ void group_compute_ld(C* r, uint32_t k, const C* tws) {
    constexpr int L0 = stage_l0(P);
    if constexpr (R == 4 && !FIRST) {
        const C* t = tws + (L - L0) + k;
        bfly4_tw(r[0], r[1], r[2], r[3], tw_load(t, 0), tw_load(t, L), tw_load(t, 2 * L));
    } else if constexpr (R == 16) {
        if constexpr (FIRST) {
#pragma unroll
            for (int a = 0; a < 4; ++a) bfly4_first(r[a], r[a + 4], r[a + 8], r[a + 12]);
        } else {
            const C* t = tws + (L - L0) + k;
            const C w1 = tw_load(t, 0), w2 = tw_load(t, L), w3 = tw_load(t, 2 * L);
#pragma unroll
            for (int a = 0; a < 4; ++a) bfly4_tw(r[a], r[a + 4], r[a + 8], r[a + 12], w1, w2, w3);
        }
        const C* t2 = tws + (4 * L - L0) + k;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            bfly4_tw(r[4 * m], r[4 * m + 1], r[4 * m + 2], r[4 * m + 3], tw_load(t2, m * L),
                     tw_load(t2, m * L + 4 * L), tw_load(t2, m * L + 8 * L));
        }
    } else {
        group_compute<R, FIRST>(r, (const C*)nullptr);
    }
}

// Output index mu of register slot s after a group.
__host__ __device__ constexpr int group_mu(const Grp G, int s) {
    return G.nst == 2 ? (s >> 2) + 4 * (s & 3) : s;
}

// Butterfly of thread lt in a last group with one butterfly per thread and
// L = T butterflies. With MIRROR, threads come in groups of 2H (H = half a
// warp, or T/2 when T < 32): the lower H threads hold b = j, the upper H hold
// b = L - j for the same j (b = L/2 for j = 0), so bins k and N - k sit in
// lanes that differ by H. Each half-warp still reads consecutive positions.
template <bool MIRROR, int T>
__device__ __forceinline__ int last_butterfly(int lt, int L) {
    if constexpr (!MIRROR) {
        return lt;
    } else {
        constexpr int H = (T < 32 ? T : 32) / 2;
        const int g = lt / (2 * H), l = lt % (2 * H);
        const int j = g * H + (l % H);
        return l < H ? j : (j == 0 ? L / 2 : L - j);
    }
}

// The RFFT forward split of one bin pair from z1 = Z[k], z2 = Z[N-k]
// (src/common/zldsp_fft_common_execute.hpp:347-358).
template <typename F>
struct SplitOut {
    F xr_k, xi_k, xr_m, xi_m;
};
template <typename F, typename C>
__device__ __forceinline__ SplitOut<F> rfft_split(C z1, C z2, F c, F s) {
    const F si = z1.y + z2.y, dr = z1.x - z2.x;
    SplitOut<F> o;
    o.xr_k = fma_rn(-dr, s, fma_rn(si, c, z1.x));
    o.xi_k = fma_rn(-dr, c, fma_rn(-si, s, z1.y));
    o.xr_m = fma_rn(dr, s, fma_rn(-si, c, z2.x));
    o.xi_m = fma_rn(-dr, c, fma_rn(-si, s, z2.y));
    return o;
}

// Radix-16 group (not the first) of the fast-twiddle form, sub-length L,
// in-group index k: the group equals a pre-twiddle of input register rho by
// W_{16L}^{rho k} followed by the untwiddled radix-16 (stage A plain
// radix-4s, stage B radix-4s with the constants W_16^{a m}), with the same
// output order as group_compute. The 15 twiddles come from two table values,
// W_{16L}^{k} and W_{16L}^{4k}, by products (at most four roundings), instead
// of 15 table loads: results stay within the FP bar, but are not the
// reference's bits.
//
// group16_fast_tw loads the two table values; group16_fast_w runs the group
// from them, so a caller can issue the loads early. Both come from the
// per-stage tables (stage_l0 layout), where they are contiguous in k:
// W_{16L}^k is stage 4L's q = 1 entry k and W_{16L}^{4k} = W_{4L}^k is stage
// L's q = 1 entry k, so consecutive k (lanes) read consecutive entries. (From
// the unified table they sit 2^s apart, one sector per lane.)
template <int P, int L, typename C>
__device__ __forceinline__ void group16_fast_tw(uint32_t k, const C* tws, C& w1, C& w4) {
    constexpr uint32_t L0 = (uint32_t)stage_l0(P);
    w1 = tw_load(tws, 4u * (uint32_t)L - L0 + k);
    w4 = tw_load(tws, (uint32_t)L - L0 + k);
}

template <typename C>
__device__ __forceinline__ void group16_fast_w(C* r, const C w1, const C w4) {
    using F = decltype(C::x);
    const C w2 = cmul_tw(w1, w1), w3 = cmul_tw(w1, w2);
    const C w8 = cmul_tw(w4, w4), w12 = cmul_tw(w4, w8);
    const C one = cx<C>((F)1, (F)0);
    const C lo[4] = {one, w1, w2, w3};
    const C hi[4] = {one, w4, w8, w12};
#pragma unroll
    for (int rho = 1; rho < 16; ++rho) {
        const C w = (rho & 3) == 0 ? hi[rho >> 2] : ((rho >> 2) == 0 ? lo[rho & 3] : cmul_tw(lo[rho & 3], hi[rho >> 2]));
        r[rho] = cmul_tw(r[rho], w);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) bfly4_first(r[a], r[a + 4], r[a + 8], r[a + 12]);
    // W_16^j = exp(-2 pi i j / 16) for j = a * m
    const C c1 = cx<C>((F)0.92387953251128674, (F)-0.38268343236508978);
    const C c2 = cx<C>((F)0.70710678118654752, (F)-0.70710678118654752);
    const C c3 = cx<C>((F)0.38268343236508978, (F)-0.92387953251128674);
    const C c4 = cx<C>((F)0, (F)-1);
    const C c6 = cx<C>((F)-0.70710678118654752, (F)-0.70710678118654752);
    const C c9 = cx<C>((F)-0.92387953251128674, (F)0.38268343236508978);
    bfly4_first(r[0], r[1], r[2], r[3]);
    bfly4_tw(r[4], r[5], r[6], r[7], c1, c2, c3);
    bfly4_tw(r[8], r[9], r[10], r[11], c2, c4, c6);
    bfly4_tw(r[12], r[13], r[14], r[15], c3, c6, c9);
}

template <int P, int L, typename C>
__device__ __forceinline__ void group16_fast(C* r, uint32_t k, const C* tws) {
    C w1, w4;
    group16_fast_tw<P, L>(k, tws, w1, w4);
    group16_fast_w(r, w1, w4);
}

// ---------------------------------------------------------------- the tile worker
// Per-thread state of one CTA working on tiles of TPC transforms of order P,
// and the processing of one tile. tile_kernel drives it over a contiguous
// batch with TMA prefetch; mixed_kernel (zlfft_mixed.cuh) drives it over a
// queue of tiles of many orders.
//
// KEEP (forward C2C only): the transform's output stays in the exchange
// buffer instead of going to global memory, slot-interleaved with an XOR
// swizzle (keep_idx), for a caller that stores the TPC transforms of a tile
// together (the transposed store of the macro path, zlfft_macro.cuh).
template <typename F, int P, int OP, int IL, int OL, int BLOCK = 128, bool GATHER = false, bool WIN = false,
          bool FAST = false, bool KEEP = false, int EM = 0>
struct TileWorker {
    using Cfg = TileCfg<F, P, OP, BLOCK, EM>;
    using C = Cx<F>;
    static constexpr int N = Cfg::N, E = Cfg::E, T = Cfg::T, TPC = Cfg::TPC, NG = Cfg::NG;
    static constexpr bool kFwd = (OP == kC2CFwd || OP == kR2CFwd || OP == kR2CSqrMag);
    static constexpr bool kR2C = (OP == kR2CFwd || OP == kR2CSqrMag);
    static constexpr Grp GL = tile_group(P, NG > 0 ? NG - 1 : 0);
    // last group: one butterfly per thread, twiddles held in registers (FP32;
    // FP64 twiddles would take twice the registers and are read from L1)
    static constexpr bool kLastReg = NG >= 2 && GL.R == E && !GL.first && sizeof(F) == 4;
    static constexpr bool kShufPost = kR2C && NG >= 2 && GL.R == E && !GL.first && GL.R == 16 && T >= 2;
    static constexpr int kLastTw = group_tw_count<P, GL.R, GL.L, GL.first>();
    static_assert(!Cfg::kTMA1 || !kR2C || kShufPost, "single-buffer staging needs the split in registers");
    static constexpr int H = (T < 32 ? T : 32) / 2;  // partner-lane distance of the shuffle split
    static constexpr bool kSoAIn = (IL == kSoA) && !kR2C;

    C* sm;
    int lt, slot;
    uint32_t sbase;
    const C* tw;
    const C* tws;
    int b_last;
    C wl[kLastTw > 0 ? kLastTw : 1];
    // fast form, complex orders 12 and up: the two table twiddles of each
    // radix-16 group that reads its twiddles (one butterfly per thread in such
    // a group, at a per-thread constant k), loaded once per CTA. (Measured:
    // +8-10% at orders 12-13; at order 11 the longer live ranges cost 3-5%.)
    static constexpr bool kHoistFast = FAST && P >= 12;
    C fw[NG > 0 ? NG : 1][2];

    __device__ __forceinline__ TileWorker(const TileArgs& a, unsigned char* smem_raw) {
        sm = reinterpret_cast<C*>(smem_raw);
        lt = (int)threadIdx.x % T;
        slot = (int)threadIdx.x / T;
        sbase = (uint32_t)slot * N;
        tw = static_cast<const C*>(a.tw);
        tws = static_cast<const C*>(a.tws);
        b_last = last_butterfly<kShufPost, T>(lt, GL.L);
        if constexpr (kLastReg) group_load_tw<P, GL.R, GL.L, GL.first>(tw, (uint32_t)(b_last % GL.L), wl);
        if constexpr (kHoistFast && NG > 0) {
            [&]<int... GI>(std::integer_sequence<int, GI...>) {
                (
                    [&] {
                        constexpr Grp G = tile_group(P, GI);
                        constexpr bool kLast = (GI + 1 == NG);
                        if constexpr (fast_group<G, kLast>()) {
                            const int b = kLast ? b_last : lt;
                            group16_fast_tw<P, G.L>((uint32_t)(b % G.L), tws, fw[GI][0], fw[GI][1]);
                        }
                    }(),
                    ...);
            }(std::make_integer_sequence<int, NG>{});
        }
    }

    // the radix-16 groups whose fast-form twiddles are hoisted
    template <Grp G, bool kLast>
    static constexpr bool fast_group() {
        return kHoistFast && G.R == 16 && !G.first && E == 16 && !(kLast && kLastReg);
    }

    __device__ __forceinline__ uint32_t sidx(int pos) const { return swz<C>(sbase + (uint32_t)pos); }

    // KEEP layout: output k of slot q at k * TPC + (q ^ ((k / KR) % TPC)), with
    // KR rows of TPC points per 128-byte line (1 when a row fills the line).
    // Consecutive k of one slot (a half-warp's writes) then take distinct
    // (row in line, slot) pairs, and whole rows (all slots of consecutive k, the
    // transposed store's reads) are permutations within each line: both touch
    // every bank once per line.
    static constexpr int KR = (int)(128 / sizeof(C)) > TPC ? (int)(128 / sizeof(C)) / TPC : 1;
    static __host__ __device__ __forceinline__ uint32_t keep_idx(int k, int q) {
        return (uint32_t)k * TPC + (uint32_t)(q ^ ((k / KR) & (TPC - 1)));
    }

    // Backward RFFT: issue the cp.async copies of tile t's bins into the
    // staging buffer (all threads share them) and commit them as one group.
    __device__ __forceinline__ void stage_bins(const TileArgs& a, long long t) const {
        if constexpr (Cfg::kStageBins) {
            F* st = reinterpret_cast<F*>(sm + (size_t)TPC * N);
            for (int q = 0; q < TPC; ++q) {
                const long long tr = t * TPC + q;
                if (tr >= a.batch) break;
                F* d = st + (size_t)q * 2 * (N + 1);
                const long long base = tr * a.in_stride;
                if constexpr (IL == kSoA) {
                    const F* re = static_cast<const F*>(a.in0) + base;
                    const F* im = static_cast<const F*>(a.in1) + base;
                    for (int i = (int)threadIdx.x; i <= N; i += Cfg::THREADS) {
                        cp_async<sizeof(F)>(d + i, re + i);
                        cp_async<sizeof(F)>(d + N + 1 + i, im + i);
                    }
                } else {
                    const C* src = static_cast<const C*>(a.in0) + base;
                    C* dc = reinterpret_cast<C*>(d);
                    for (int i = (int)threadIdx.x; i <= N; i += Cfg::THREADS) cp_async<sizeof(C)>(dc + i, src + i);
                }
            }
            cp_async_commit();
        }
    }

    // Process tile `tile`. With use_tma, group 0 reads this tile's input from
    // the staging buffer that follows the exchange buffer in shared memory
    // (placed there by TMA) and calls refill() once done; for a backward RFFT,
    // use_tma means the pre-step reads the bins staged by stage_bins (it
    // waits for them) and calls refill() once they are read. A backward RFFT
    // may hand its output samples to `sink` (see NoSink).
    template <class Refill, class Sink = NoSink>
    __device__ __forceinline__ void run(const TileArgs& a, long long tile, bool use_tma, Refill&& refill,
                                        const Sink& sink = Sink{}) {
        static_assert(!Sink::kActive || OP == kC2RBwd, "output sinks take backward RFFT samples");
        static_assert(!KEEP || (OP == kC2CFwd && (TPC & (TPC - 1)) == 0), "KEEP: forward C2C, power-of-two slots");
        const C* stage = Cfg::kTMA1 ? sm : sm + (size_t)TPC * N;
        const long long tr = tile * TPC + slot;
        const bool valid = tr < a.batch;
        // this slot's transform: contiguous (base + stride) or gathered pointers
        const void* ib0 = a.in0;
        const void* ib1 = a.in1;
        void* ob0 = a.out0;
        void* ob1 = a.out1;
        long long ibase = valid ? tr * a.in_stride : 0;
        long long obase = valid ? tr * a.out_stride : 0;
        if constexpr (GATHER) {
            const long long g = valid ? tr : 0;
            ib0 = a.gin0[g];
            ib1 = a.gin1 ? a.gin1[g] : nullptr;
            ob0 = a.gout0[g];
            ob1 = a.gout1 ? a.gout1[g] : nullptr;
            ibase = obase = 0;
        }
        C v[E];

        // ------------------------------------------------ input
        // Backward RFFT pre-step (execute.hpp:399-451): Z[p] from the bins at p
        // and N - p. Where the bins are staged in shared memory (and no sink is
        // attached), each thread computes the Z of its own group-0 positions in
        // registers (bin pair k, N - k is read by the two threads that need it),
        // so Z never goes through shared memory. Elsewhere Z is built in shared
        // memory first: reading each bin twice from global memory measured
        // 20-50% slower (FP32 orders 7-9 and 11, FP64, the inverse STFT), while
        // the staged orders gained 3-9% (RFFT<float> backward order 13: 3018 ->
        // 3301 GB/s, order 14: 2342 -> 2558).
        constexpr bool kDirectPre = OP == kC2RBwd && NG >= 2 && Cfg::kStageBins && !Sink::kActive;
        [[maybe_unused]] const C* rw = static_cast<const C*>(a.rw);
        [[maybe_unused]] const C* hf = static_cast<const C*>(sink.h);
        [[maybe_unused]] const F* sb = reinterpret_cast<const F*>(stage) + (size_t)slot * 2 * (N + 1);
        [[maybe_unused]] const CxIn<F, IL> bins(ib0, ib1, ibase);
        [[maybe_unused]] auto bin = [&](int k) -> C {  // bin k, times the filter's bin k
            C x;
            if constexpr (Cfg::kStageBins) {
                if (use_tma) {
                    if constexpr (IL == kSoA) {
                        x = cx<C>(sb[k], sb[N + 1 + k]);
                    } else {
                        x = reinterpret_cast<const C*>(sb)[k];
                    }
                } else {
                    x = bins[k];
                }
            } else {
                x = bins[k];
            }
            if constexpr (Sink::kActive) {
                if (hf) x = cmul_rn(x, hf[k]);
            }
            return x;
        };
        // Z[p]: p = 0 from bins 0 and N; 1 <= p < N/2 the first value of pair
        // k = p, N/2 <= p < N the second value of pair k = N - p
        [[maybe_unused]] auto prez = [&](int p) -> C {
            if (p == 0) {
                const C x0 = bin(0), xm = bin(N);
                return cx<C>(mul_rn(x0.x + xm.x, (F)0.5), mul_rn(x0.x - xm.x, (F)0.5));
            }
            const int k = p < N / 2 ? p : N - p;
            const C x1 = bin(k), x2 = bin(N - k);
            const C w = rw[k];
            const F c = w.x, s = w.y;
            const F si = x1.y + x2.y, dr = x1.x - x2.x;
            if (p < N / 2) return cx<C>(fma_rn(-dr, s, fma_rn(-si, c, x1.x)), fma_rn(dr, c, fma_rn(-si, s, x1.y)));
            return cx<C>(fma_rn(dr, s, fma_rn(si, c, x2.x)), fma_rn(dr, c, fma_rn(-si, s, x2.y)));
        };
        if constexpr (OP == kC2RBwd) {
            if constexpr (Cfg::kStageBins) {
                if (use_tma) {  // this tile's bins are in the staging buffer
                    cp_async_wait_all();
                    __syncthreads();
                }
            }
            if constexpr (!kDirectPre) {
                if (valid) {  // one thread per bin pair (k, N - k): both Z values from one read of the pair
                    for (int k = 1 + lt; k <= N / 2; k += T) {
                        const C x1 = bin(k), x2 = bin(N - k);
                        const C w = rw[k];
                        const F c = w.x, s = w.y;
                        const F si = x1.y + x2.y, dr = x1.x - x2.x;
                        const C zk = cx<C>(fma_rn(-dr, s, fma_rn(-si, c, x1.x)), fma_rn(dr, c, fma_rn(-si, s, x1.y)));
                        const C zm = cx<C>(fma_rn(dr, s, fma_rn(si, c, x2.x)), fma_rn(dr, c, fma_rn(-si, s, x2.y)));
                        if (k != N / 2) sm[sidx(k)] = zk;
                        sm[sidx(N - k)] = zm;
                    }
                    if (lt == 0) sm[sidx(0)] = prez(0);
                }
                __syncthreads();
                if constexpr (Cfg::kStageBins) {
                    if (use_tma) refill();  // the staged bins are read: the next tile's may come in
                }
            }
        }

        // ------------------------------------------------ stage groups
        constexpr int OL2 = (OP == kC2RBwd || OP == kR2CSqrMag) ? (int)kAoS : OL;
        const CxOut<F, OL2> out(ob0, ob1, obase);
        if constexpr (NG == 0) {
            C x;
            if constexpr (OP == kC2RBwd) {
                x = cswap(sm[sidx(0)]);
            } else {
                constexpr int IL2 = kR2C ? (int)kAoS : IL;
                const CxIn<F, IL2> in(ib0, ib1, ibase);
                x = valid ? in[0] : cx<C>((F)0, (F)0);
                if constexpr (!kFwd) x = cswap(x);
            }
            if constexpr (kR2C && WIN) {
                {
                    const C w = static_cast<const C*>(a.win)[0];
                    x = cx<C>(mul_rn(x.x, w.x), mul_rn(x.y, w.y));
                }
            }
            v[0] = x;
            if constexpr (kR2C) {
                sm[sidx(0)] = v[0];
            } else if (valid) {
                out.put(0, kFwd ? v[0] : cswap(v[0]));
            }
        } else {
            [&]<int... GI>(std::integer_sequence<int, GI...>) {
                (
                    [&] {
                        constexpr Grp G = tile_group(P, GI);
                        constexpr int NB = E / G.R;
                        constexpr bool kLast = (GI + 1 == NG);
                        // ---- inputs of this group
                        if constexpr (GI == 0 && kDirectPre) {
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = lt + u * T;
#pragma unroll
                                for (int rho = 0; rho < G.R; ++rho)
                                    v[u * G.R + rho] = valid ? cswap(prez(b + rho * (N / G.R))) : cx<C>((F)0, (F)0);
                            }
                        } else if constexpr (GI == 0 && OP != kC2RBwd) {
                            if (use_tma) {
                                const C* sc = stage + (size_t)slot * N;
                                const F* sf = reinterpret_cast<const F*>(sc);
#pragma unroll
                                for (int u = 0; u < NB; ++u) {
                                    const int b = (kLast ? b_last : lt) + u * T;
#pragma unroll
                                    for (int rho = 0; rho < G.R; ++rho) {
                                        const int pos = b + rho * (N / G.R);
                                        C x = kSoAIn ? cx<C>(sf[pos], sf[N + pos]) : sc[pos];
                                        v[u * G.R + rho] = kFwd ? x : cswap(x);
                                    }
                                }
                                if constexpr (!Cfg::kTMA1) refill();
                            } else {
                                constexpr int IL2 = kR2C ? (int)kAoS : IL;
                                const CxIn<F, IL2> in(ib0, ib1, ibase);
#pragma unroll
                                for (int u = 0; u < NB; ++u) {
                                    const int b = (kLast ? b_last : lt) + u * T;
#pragma unroll
                                    for (int rho = 0; rho < G.R; ++rho) {
                                        C x = valid ? in[b + rho * (N / G.R)] : cx<C>((F)0, (F)0);
                                        v[u * G.R + rho] = kFwd ? x : cswap(x);
                                    }
                                }
                            }
                            if constexpr (kR2C && WIN) {  // STFT: window the frame as it is loaded
                                {
                                    const C* wp = static_cast<const C*>(a.win);
#pragma unroll
                                    for (int u = 0; u < NB; ++u) {
                                        const int b = (kLast ? b_last : lt) + u * T;
#pragma unroll
                                        for (int rho = 0; rho < G.R; ++rho) {
                                            const C w = __ldg(wp + b + rho * (N / G.R));
                                            C& x = v[u * G.R + rho];
                                            x = cx<C>(mul_rn(x.x, w.x), mul_rn(x.y, w.y));
                                        }
                                    }
                                }
                            }
                        } else {
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = (kLast ? b_last : lt) + u * T;
#pragma unroll
                                for (int rho = 0; rho < G.R; ++rho) {
                                    const int pos = b + rho * (N / G.R);
                                    uint32_t ix;
                                    if constexpr (kShufPost && kLast) {
                                        ix = swz_mirror<C, tile_group(P, NG >= 2 ? NG - 2 : 0).L>(sbase + (uint32_t)pos);
                                    } else {
                                        ix = sidx(pos);
                                    }
                                    const C x = sm[ix];
                                    v[u * G.R + rho] = (GI == 0 && OP == kC2RBwd) ? cswap(x) : x;
                                }
                            }
                            if constexpr (kLast && Cfg::kTMA1) {
                                if (use_tma) refill();  // the buffer is read: the next tile's input may land
                            }
                        }
                        // ---- compute
                        if constexpr (kLast && kLastReg) {
                            group_compute<G.R, G.first>(v, wl);
                        } else {
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = (kLast ? b_last : lt) + u * T;
                                if constexpr (fast_group<G, kLast>()) {  // fast-twiddle form, hoisted twiddles
                                    group16_fast_w(v + u * G.R, fw[GI][0], fw[GI][1]);
                                } else if constexpr (FAST && G.R == 16 && !G.first) {
                                    group16_fast<P, G.L>(v + u * G.R, (uint32_t)(b % G.L), tws);
                                } else {
                                    group_compute_ld<P, G.R, G.L, G.first>(v + u * G.R, (uint32_t)(b % G.L), tws);
                                }
                            }
                        }
                        // ---- outputs
                        if constexpr (!kLast) {
                            __syncthreads();
                            if constexpr (GI == 0 && kDirectPre && Cfg::kStageBins) {
                                if (use_tma) refill();  // the staged bins are read: the next tile's may come in
                            }
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = lt + u * T;
                                const int J = b / G.L, k = b % G.L;
#pragma unroll
                                for (int s = 0; s < G.R; ++s) {
                                    const int pos = J * G.R * G.L + k + group_mu(G, s) * G.L;
                                    uint32_t ix;
                                    if constexpr (kShufPost && GI + 2 == NG) {
                                        ix = swz_mirror<C, G.L>(sbase + (uint32_t)pos);
                                    } else {
                                        ix = sidx(pos);
                                    }
                                    sm[ix] = v[u * G.R + s];
                                }
                            }
                            __syncthreads();
                        } else if constexpr (kShufPost) {
                            // RFFT split from registers: z[mu] = Z[b + mu*L]; the partner lane
                            // (lt ^ H) holds Z[N - b - mu*L] at slot 15 - mu (for the lanes
                            // holding b = 0 and b = L/2 the partner is the lane itself).
                            constexpr int L = G.L;
                            C z[16];
#pragma unroll
                            for (int s = 0; s < 16; ++s) z[group_mu(G, s)] = v[s];
                            const C* rw = static_cast<const C*>(a.rw);
                            [[maybe_unused]] F* osq = static_cast<F*>(ob0) + obase;
#pragma unroll
                            for (int m = 0; m < 8; ++m) {
                                C p;
                                p.x = __shfl_xor_sync(0xffffffffu, z[15 - m].x, H);
                                p.y = __shfl_xor_sync(0xffffffffu, z[15 - m].y, H);
                                C z2 = p;
                                const int k = b_last + m * L;
                                if (lt == 0) {  // b = 0: pairs (m, 16 - m); m = 0 is DC/Nyquist
                                    z2 = z[(16 - m) & 15];
                                } else if (lt == H) {  // b = L/2: pairs (m, 15 - m) in this lane
                                    z2 = z[15 - m];
                                }
                                if (valid && !(lt == 0 && m == 0)) {
                                    const C w = rw[k];
                                    const SplitOut<F> o = rfft_split<F>(z[m], z2, w.x, w.y);
                                    if constexpr (OP == kR2CFwd) {
                                        if (k != N / 2) out.put(k, cx<C>(o.xr_k, o.xi_k));
                                        out.put(N - k, cx<C>(o.xr_m, o.xi_m));
                                    } else {
                                        if (k != N / 2) __stcs(osq + k, fma_rn(o.xr_k, o.xr_k, mul_rn(o.xi_k, o.xi_k)));
                                        __stcs(osq + N - k, fma_rn(o.xr_m, o.xr_m, mul_rn(o.xi_m, o.xi_m)));
                                    }
                                }
                            }
                            if (valid && lt == 0) {  // b = 0 also owns k = N/2 (slot 8) and DC/Nyquist
                                const C w = rw[N / 2];
                                const SplitOut<F> o = rfft_split<F>(z[8], z[8], w.x, w.y);
                                const F dc = z[0].x + z[0].y, ny = z[0].x - z[0].y;
                                if constexpr (OP == kR2CFwd) {
                                    out.put(N / 2, cx<C>(o.xr_m, o.xi_m));
                                    out.put(0, cx<C>(dc, (F)0));
                                    out.put(N, cx<C>(ny, (F)0));
                                } else {
                                    __stcs(osq + N / 2, fma_rn(o.xr_m, o.xr_m, mul_rn(o.xi_m, o.xi_m)));
                                    __stcs(osq, mul_rn(dc, dc));
                                    __stcs(osq + N, mul_rn(ny, ny));
                                }
                            }
                        } else if constexpr (KEEP) {
                            __syncthreads();  // every input of the last group is read: the buffer is free
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = b_last + u * T;
#pragma unroll
                                for (int s = 0; s < G.R; ++s) sm[keep_idx(b + group_mu(G, s) * G.L, slot)] = v[u * G.R + s];
                            }
                        } else {
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
                                const int b = b_last + u * T;  // J == 0 in the last group
#pragma unroll
                                for (int s = 0; s < G.R; ++s) {
                                    const int pos = b + group_mu(G, s) * G.L;
                                    if constexpr (kR2C) {
                                        sm[sidx(pos)] = v[u * G.R + s];
                                    } else if (valid) {
                                        if constexpr (Sink::kActive) {
                                            sink.add(pos, cswap(v[u * G.R + s]));
                                        } else {
                                            out.put(pos, kFwd ? v[u * G.R + s] : cswap(v[u * G.R + s]));
                                        }
                                    }
                                }
                            }
                        }
                    }(),
                    ...);
            }(std::make_integer_sequence<int, NG>{});
        }

        // ------------------------------------------------ RFFT forward split through shared memory
        // (orders without a shuffle-friendly last group)
        if constexpr (kR2C && !kShufPost) {
            __syncthreads();
            if (valid) {
                const C* rw = static_cast<const C*>(a.rw);
                [[maybe_unused]] F* osq = static_cast<F*>(ob0) + obase;
                for (int k = 1 + lt; k <= N / 2; k += T) {
                    const C w = rw[k];
                    const SplitOut<F> o = rfft_split<F>(sm[sidx(k)], sm[sidx(N - k)], w.x, w.y);
                    if constexpr (OP == kR2CFwd) {
                        if (k != N / 2) out.put(k, cx<C>(o.xr_k, o.xi_k));
                        out.put(N - k, cx<C>(o.xr_m, o.xi_m));
                    } else {
                        if (k != N / 2) __stcs(osq + k, fma_rn(o.xr_k, o.xr_k, mul_rn(o.xi_k, o.xi_k)));
                        __stcs(osq + N - k, fma_rn(o.xr_m, o.xr_m, mul_rn(o.xi_m, o.xi_m)));
                    }
                }
                if (lt == 0) {
                    const C z0 = sm[sidx(0)];
                    const F dc = z0.x + z0.y, ny = z0.x - z0.y;
                    if constexpr (OP == kR2CFwd) {
                        out.put(0, cx<C>(dc, (F)0));
                        out.put(N, cx<C>(ny, (F)0));
                    } else {
                        __stcs(osq, mul_rn(dc, dc));
                        __stcs(osq + N, mul_rn(ny, ny));
                    }
                }
            }
        }
        // The next tile's first shared-memory write is preceded by a barrier in
        // every path except the backward RFFT pre-step and the single-point case.
        if constexpr (OP == kC2RBwd || NG == 0) __syncthreads();
    }
};

// ---------------------------------------------------------------- the kernel
template <typename F, int P, int OP, int IL, int OL, bool GATHER = false, bool WIN = false, bool FAST = false>
__global__ void __launch_bounds__(TileCfg<F, P, OP>::THREADS, TileCfg<F, P, OP>::MINB) tile_kernel(const TileArgs a) {
    using W = TileWorker<F, P, OP, IL, OL, 128, GATHER, WIN, FAST>;
    using Cfg = typename W::Cfg;
    using C = Cx<F>;
    constexpr int N = Cfg::N, TPC = Cfg::TPC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    W w(a, smem_raw);

    // ---- TMA staging of each tile's input (one tile ahead)
    constexpr bool kSoAIn = W::kSoAIn;
    C* stage = reinterpret_cast<C*>(smem_raw) + (Cfg::kTMA1 ? 0 : (size_t)TPC * N);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + Cfg::XBYTES * (Cfg::kTMA1 ? 1 : 2));
    // gathered transforms (AoS): one bulk copy from each transform's own pointer,
    // where the batch found every input 16-byte aligned (a.tma)
    const bool use_tma = (Cfg::kTMA || Cfg::kTMA1) && (!GATHER || !kSoAIn) && a.tma;
    auto issue = [&](long long t) {  // warp 0 issues the copies of tile t
        if (!use_tma || threadIdx.x >= 32 || t * TPC >= a.batch) return;
        const long long left = a.batch - t * TPC;
        const int nvalid = (int)(left < TPC ? left : TPC);
        constexpr uint32_t kSlot = (uint32_t)(N * sizeof(C));
        if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, kSlot * (uint32_t)nvalid);
        __syncwarp();
        for (int q = (int)threadIdx.x; q < nvalid; q += 32) {
            const long long base = (t * TPC + q) * a.in_stride;
            if constexpr (kSoAIn) {
                F* dst = reinterpret_cast<F*>(stage + (size_t)q * N);
                bulk_g2s(dst, static_cast<const F*>(a.in0) + base, kSlot / 2, bar);
                bulk_g2s(dst + N, static_cast<const F*>(a.in1) + base, kSlot / 2, bar);
            } else if constexpr (GATHER) {
                bulk_g2s(stage + (size_t)q * N, static_cast<const C*>(a.gin0[t * TPC + q]), kSlot, bar);
            } else {
                bulk_g2s(stage + (size_t)q * N, static_cast<const C*>(a.in0) + base, kSlot, bar);
            }
        }
    };
    if constexpr (Cfg::kTMA || Cfg::kTMA1) {
        if (use_tma) {
            if (threadIdx.x == 0) {
                mbar_init(bar, 1);
                fence_mbar_init();
            }
            __syncthreads();
            issue(blockIdx.x);
        }
    }
    uint32_t phase = 0;
    // backward RFFT: bins staged by cp.async, one tile ahead
    const bool use_stage = Cfg::kStageBins && !GATHER && a.tma;
    if (use_stage) w.stage_bins(a, blockIdx.x);

    for (long long tile = blockIdx.x; tile * TPC < a.batch; tile += gridDim.x) {
        if constexpr (Cfg::kTMA || Cfg::kTMA1) {
            if (use_tma) {
                const bool ok = mbar_wait(bar, phase);
                if (__syncthreads_or(!ok)) {  // bounded wait ran out: report and leave
                    if (threadIdx.x == 0) atomicOr(a.err, kDevErrWaitTimeout);
                    mbar_wait(bar, phase);  // give copies in flight a bounded chance to land
                    return;
                }
                phase ^= 1u;
            }
        }
        if constexpr (OP == kC2RBwd) {
            w.run(a, tile, use_stage, [&]() { w.stage_bins(a, tile + gridDim.x); });
        } else {
            w.run(a, tile, use_tma, [&]() {
                fence_proxy_async_smem();  // reads of the staging buffer before its TMA refill
                __syncthreads();           // staging fully read: refill it with the next tile
                issue(tile + gridDim.x);
            });
        }
    }
}

}  // namespace zlfft
