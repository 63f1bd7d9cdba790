// The reference's macro path ("hybrid" CFFT) on the GPU, plain form.
//
// On a host whose caches put a CFFT of order O at or above its switch order,
// the reference does not run its Stockham stages over the whole transform
// (src/common/zldsp_fft_common_init.hpp:305-339, system.hpp:132-157). It runs
//   1. nm Cooley-Tukey radix-4 DIF "macro" stages in place, the twiddle of
//      output m applied after the butterfly
//      (src/common/zldsp_fft_common_radix.hpp:670-843);
//   2. a forward Stockham FFT of order m (the micro order) on each of the
//      S = 4^nm contiguous segments (execute.hpp:198-245);
//   3. a transposed store: output k*S + c is output k of the segment at
//      position digit_rev4(c) (execute.hpp:246-271), through the store's
//      direction swap.
// Its output differs in its rounding from the micro-only path's, so a
// drop-in that must reproduce the reference's bits on such a host runs the
// same arithmetic. Two kernels do it here:
//
// dif_pass_kernel: DIF stages i0 .. i0+G-1 of a transform. Stage i has
// butterfly stride w_i = N / 4^(i+1); every stride of the pass is a multiple
// of the last one, W, so the pass works on "units" of R = 4^G points at
// stride W: unit U = blk * W + lo holds positions blk*R*W + lo + t*W, t < R,
// and stage i's butterflies combine the t that differ in one base-4 digit.
// A CTA takes UPC consecutive units (consecutive lo), so every global row it
// reads or writes is 128 contiguous bytes. Inside a unit the stages run as
// radix-16 register groups (two DIF stages) and a last radix-4 group when G
// is odd; groups exchange in shared memory in place ([t][unit], padded rows).
// The twiddle of stage i for j = position mod w_i is W_{4 w_i}^{m j}, read
// from the plan's per-stage table of sub-length L = w_i (the values of the
// reference's macro table, init.hpp:227-274). The last DIF pass writes
// segment sigma to position digit_rev4(sigma) * M of the scratch, so that
// the segment of output column c is the c-th contiguous block.
//
// macro_seg_kernel: the micro FFT of CB consecutive columns per tile (the
// tile kernel's TileWorker, forward, no swap), kept in shared memory
// (TileWorker KEEP), then stored transposed: column c's point k goes to
// k*S + c, so each output row of the tile is CB consecutive points (128 bytes
// in FP32 with CB = 16).
//
// Nothing here is approximate: with the reference's twiddle bits and the
// same operation order the output is the reference's macro-path output bit
// for bit (FP32; FP64 twiddles differ in ulps from the host's libm).
#pragma once

#include "zlfft_launch.cuh"
#include "zlfft_tile.cuh"

namespace zlfft {

// Radix-4 DIF butterfly in place, twiddles after the butterfly
// (src/common/zldsp_fft_common_radix.hpp:686-749 and :780-841):
// t0 = x0 + x2, t1 = x0 - x2, t2 = x1 + x3, t3 = x1 - x3;
// y0 = t0 + t2, y1 = (t1 - i t3) w1, y2 = (t0 - t2) w2, y3 = (t1 + i t3) w3.
template <typename C>
__device__ __forceinline__ void bfly4_dif(C& a0, C& a1, C& a2, C& a3, C w1, C w2, C w3) {
    const C t0 = cadd(a0, a2), t1 = csub(a0, a2);
    const C t2 = cadd(a1, a3), t3 = csub(a1, a3);
    const C y1 = csub_i(t1, t3);
    const C y2 = csub(t0, t2);
    const C y3 = cadd_i(t1, t3);
    a0 = cadd(t0, t2);
    a1 = cmul_tw(y1, w1);
    a2 = cmul_tw(y2, w2);
    a3 = cmul_tw(y3, w3);
}

// Base-4 digit reversal of x over nd digits (src/common/zldsp_fft_common_init.hpp:282-296):
// reversing 2*nd bits moves digit k to digit nd-1-k with its two bits
// swapped, which the pair swap undoes.
__device__ __forceinline__ uint32_t digit_rev4(uint32_t x, int nd) {
    if (nd == 0) return 0;
    const uint32_t y = __brev(x) >> (32 - 2 * nd);
    return ((y & 0x55555555u) << 1) | ((y >> 1) & 0x55555555u);
}

// ---------------------------------------------------------------- DIF passes
template <typename F, int G>
struct DifCfg {
    using C = Cx<F>;
    static constexpr int R = 1 << (2 * G);
    static constexpr int UMIN = 128 / (int)sizeof(C);  // units per 128-byte row
    static constexpr int E0 = R < 16 ? R : 16;
    static constexpr int UPC = (128 * E0 / R) > UMIN ? (128 * E0 / R) : UMIN;  // units per CTA
    // points per thread: one radix-16 butterfly per group, two where a CTA
    // would otherwise exceed 512 threads
    static constexpr int E = (UPC * R / E0 > 512) ? 2 * E0 : E0;
    static constexpr int T = R / E;  // threads per unit
    static constexpr int THREADS = UPC * T;
    static constexpr int ROW = UPC + 1;
    static constexpr int NG = G / 2 + G % 2;  // radix-16 groups, then one radix-4 group when G is odd
    static constexpr size_t SMEM = NG > 1 ? (size_t)R * ROW * sizeof(C) : 0;
    static_assert(SMEM <= 200 * 1024, "DIF pass tile too large");
};

struct DifArgs {
    const void* in0;  // first pass: the transform input (layout IL); else scratch (AoS)
    const void* in1;
    void* out;        // scratch (AoS)
    long long batch;
    long long in_stride;   // elements between transforms of the input
    long long out_stride;  // elements between transforms of the output
    const void* tws;       // per-stage tables of the order (stage_l0 layout of zlfft_tile.cuh)
    int order;             // log2 N
    int i0;                // global index of the pass's first DIF stage
    int wlog;              // log2 of W, the pass's smallest butterfly stride (unit stride)
    int nm;                // macro stages in all (digits of the segment reversal)
    int mlog;              // micro order (log2 of the segment length)
};

// Register slot r of butterfly b in DIF group g of a G-stage pass: the unit
// position t. A radix-16 group (local stages s = 2g, 2g+1) covers the points
// base + a*S1 + c*S2 (r = 4a + c, S1 = R / 4^(s+1), S2 = S1 / 4, base =
// hi * 4 S1 + lo_t with hi = b / S2, lo_t = b % S2); the radix-4 group (the
// last stage) covers 4b + r.
template <int G, int g>
struct DifGroup {
    static constexpr int R = 1 << (2 * G);
    static constexpr int s = 2 * g;
    static constexpr bool R16 = (2 * g + 1 < G);
    static constexpr int RG = R16 ? 16 : 4;
    static constexpr int S1 = R >> (2 * (s + 1));
    static constexpr int S2 = R16 ? S1 / 4 : 1;
    static __device__ __forceinline__ int t(int b, int r) {
        if constexpr (R16) {
            const int hi = b / S2, lt = b % S2;
            return hi * 4 * S1 + lt + (r >> 2) * S1 + (r & 3) * S2;
        } else {
            return 4 * b + r;
        }
    }
};

template <typename C>
__device__ __forceinline__ void dif_tw(const C* tws, uint32_t L, uint32_t L0, uint32_t j, C& w1, C& w2, C& w3) {
    const C* t = tws + (L - L0) + j;
    w1 = tw_load(t, 0);
    w2 = tw_load(t, L);
    w3 = tw_load(t, 2 * L);
}

// The stages of group g on one butterfly's registers r[0..RG), with the
// global twiddles: unit offset lo, unit stride W = 2^wlog.
template <int G, int g, typename C>
__device__ __forceinline__ void dif_group_compute(C* r, int b, uint32_t lo, int wlog, uint32_t L0, const C* tws) {
    using Gr = DifGroup<G, g>;
    const uint32_t W = 1u << wlog;
    if constexpr (Gr::R16) {
        const uint32_t lt = (uint32_t)(b % Gr::S2);
        // stage s: the four columns c, j = lo + (lo_t + c*S2) * W, sub-length L = W * S1
        const uint32_t L1 = W * (uint32_t)Gr::S1;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            C w1, w2, w3;
            dif_tw(tws, L1, L0, lo + (lt + (uint32_t)(c * Gr::S2)) * W, w1, w2, w3);
            bfly4_dif(r[c], r[4 + c], r[8 + c], r[12 + c], w1, w2, w3);
        }
        // stage s+1: the four rows a, j = lo + lo_t * W, L = W * S2
        C w1, w2, w3;
        dif_tw(tws, W * (uint32_t)Gr::S2, L0, lo + lt * W, w1, w2, w3);
#pragma unroll
        for (int a = 0; a < 4; ++a) bfly4_dif(r[4 * a], r[4 * a + 1], r[4 * a + 2], r[4 * a + 3], w1, w2, w3);
    } else {
        C w1, w2, w3;
        dif_tw(tws, W, L0, lo, w1, w2, w3);
        bfly4_dif(r[0], r[1], r[2], r[3], w1, w2, w3);
    }
}

// One DIF pass over `batch` transforms. FIRST: reads the transform input in
// layout IL, re/im swapped for the backward direction (FWD false), as the
// reference's first DIF stage loads it (structure.hpp:47-62). LAST: writes
// segment sigma to digit_rev4(sigma) * M.
template <typename F, int G, bool FIRST, bool FWD, int IL, bool LAST>
__global__ void __launch_bounds__(DifCfg<F, G>::THREADS, 1) dif_pass_kernel(const DifArgs a) {
    using Cfg = DifCfg<F, G>;
    using C = Cx<F>;
    constexpr int R = Cfg::R, E = Cfg::E, T = Cfg::T, UPC = Cfg::UPC, ROW = Cfg::ROW, NG = Cfg::NG;
    constexpr int IL2 = FIRST ? IL : (int)kAoS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    const int u = (int)threadIdx.x % UPC;
    const int tb = (int)threadIdx.x / UPC;
    const C* tws = static_cast<const C*>(a.tws);
    const uint32_t L0 = (uint32_t)((a.order & 1) ? 8 : 4);
    const uint32_t W = 1u << a.wlog;
    const long long ipt = (1LL << (a.order - 2 * G)) / UPC;  // items (CTA tiles) per transform
    const long long items = a.batch * ipt;

    for (long long item = blockIdx.x; item < items; item += gridDim.x) {
        const long long tr = item / ipt;
        const uint32_t U = (uint32_t)(item % ipt) * UPC + (uint32_t)u;
        const uint32_t blk = U >> a.wlog;
        const uint32_t lo = U & (W - 1);
        const uint32_t pbase = blk * (uint32_t)R * W + lo;  // position of t = 0
        C v[E];
        [&]<int... GI>(std::integer_sequence<int, GI...>) {
            (
                [&] {
                    using Gr = DifGroup<G, GI>;
                    constexpr int NB = E / Gr::RG;
                    constexpr bool kLastG = (GI + 1 == NG);
                    // ---- inputs
                    if constexpr (GI == 0) {
                        const CxIn<F, IL2> in(a.in0, a.in1, tr * a.in_stride);
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
#pragma unroll
                            for (int r = 0; r < Gr::RG; ++r) {
                                const C x = in[(int)(pbase + (uint32_t)Gr::t(tb + i * T, r) * W)];
                                v[i * Gr::RG + r] = (FIRST && !FWD) ? cswap(x) : x;
                            }
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
#pragma unroll
                            for (int r = 0; r < Gr::RG; ++r) v[i * Gr::RG + r] = sm[Gr::t(tb + i * T, r) * ROW + u];
                        }
                    }
                    // ---- compute
#pragma unroll
                    for (int i = 0; i < NB; ++i)
                        dif_group_compute<G, GI>(v + i * Gr::RG, tb + i * T, lo, a.wlog, L0, tws);
                    // ---- outputs: in place in shared memory, or to global memory
                    if constexpr (!kLastG) {
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
#pragma unroll
                            for (int r = 0; r < Gr::RG; ++r) sm[Gr::t(tb + i * T, r) * ROW + u] = v[i * Gr::RG + r];
                        }
                        __syncthreads();
                    } else {
                        const CxOut<F, kAoS> out(a.out, nullptr, tr * a.out_stride);
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
#pragma unroll
                            for (int r = 0; r < Gr::RG; ++r) {
                                const uint32_t t = (uint32_t)Gr::t(tb + i * T, r);
                                uint32_t dst;
                                if constexpr (LAST) {  // W == M: segment sigma = blk * R + t, offset lo
                                    dst = (digit_rev4(blk * (uint32_t)R + t, a.nm) << a.mlog) + lo;
                                } else {
                                    dst = pbase + t * W;
                                }
                                out.put((int)dst, v[i * Gr::RG + r]);
                            }
                        }
                    }
                }(),
                ...);
        }(std::make_integer_sequence<int, NG>{});
        // the next item's first exchange writes after every read of this one
        if constexpr (NG > 1) __syncthreads();
    }
}

// ---------------------------------------------------------------- segment FFTs + transposed store
// CB columns per tile: 128 bytes of points per output row, within 128 KB of
// exchange buffer (FP32: 16 up to micro order 10; FP64: 8 up to order 10).
template <typename F, int M>
struct SegCfg {
    using C = Cx<F>;
    static constexpr int CB0 = 4;  // 32- (FP32) / 64-byte (FP64) output rows, 2 CTAs per SM
    static constexpr int CBM = (128 * 1024) / ((1 << M) * (int)sizeof(C));
    static constexpr int CB = CB0 < CBM ? CB0 : CBM;
    static constexpr int EB = tile_elems(M);
    // points per thread: the largest group radix, doubled while the tile
    // would need more than 512 threads
    static constexpr int E = (CB * (1 << M) / EB > 512) ? ((CB * (1 << M) / (2 * EB) > 512) ? 4 * EB : 2 * EB) : EB;
    static constexpr int BLOCK = CB * ((1 << M) / E);
    using W = TileCfg<F, M, kC2CFwd, BLOCK, E>;
    static_assert(W::TPC == CB, "one column per slot");
};

struct SegArgs {
    TileArgs t;            // input: the DIF output, columns contiguous (in_stride = M), batch = transforms * S
    void* out0;            // the transform output (layout OL); SoA: out0 = re, out1 = im
    void* out1;
    long long out_stride;  // elements between transforms of the output
    int slog;              // log2 S (columns per transform)
};

template <typename F, int M, bool FWD, int OL>
__global__ void __launch_bounds__(SegCfg<F, M>::BLOCK, SegCfg<F, M>::W::MINB) macro_seg_kernel(const SegArgs sa) {
    using SC = SegCfg<F, M>;
    using Wk = TileWorker<F, M, kC2CFwd, kAoS, kAoS, SC::BLOCK, false, false, false, true, SC::E>;
    using Cfg = typename Wk::Cfg;
    using C = Cx<F>;
    constexpr int N = Cfg::N, TPC = Cfg::TPC;
    const TileArgs& a = sa.t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Wk w(a, smem_raw);
    C* sm = reinterpret_cast<C*>(smem_raw);

    // ---- TMA staging of each tile's columns (one tile ahead), where two buffers fit
    C* stage = sm + (size_t)TPC * N;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + Cfg::XBYTES * 2);
    const bool use_tma = Cfg::kTMA && a.tma;
    auto issue = [&](long long t) {
        if (!use_tma || threadIdx.x >= 32 || t * TPC >= a.batch) return;
        const long long left = a.batch - t * TPC;
        const int nvalid = (int)(left < TPC ? left : TPC);
        constexpr uint32_t kSlot = (uint32_t)(N * sizeof(C));
        if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, kSlot * (uint32_t)nvalid);
        __syncwarp();
        for (int q = (int)threadIdx.x; q < nvalid; q += 32)
            bulk_g2s(stage + (size_t)q * N, static_cast<const C*>(a.in0) + (t * TPC + q) * a.in_stride, kSlot, bar);
    };
    if constexpr (Cfg::kTMA) {
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
    const long long S = 1LL << sa.slog;
    for (long long tile = blockIdx.x; tile * TPC < a.batch; tile += gridDim.x) {
        if constexpr (Cfg::kTMA) {
            if (use_tma) {
                const bool ok = mbar_wait(bar, phase);
                if (__syncthreads_or(!ok)) {  // bounded wait ran out: report and leave
                    if (threadIdx.x == 0) atomicOr(a.err, kDevErrWaitTimeout);
                    mbar_wait(bar, phase);
                    return;
                }
                phase ^= 1u;
            }
        }
        w.run(a, tile, use_tma, [&]() {
            fence_proxy_async_smem();
            __syncthreads();
            issue(tile + gridDim.x);
        });
        __syncthreads();  // the tile's columns are in shared memory (KEEP layout)
        // transposed store: element e = k * TPC + q is point k of column tile*TPC + q
        const long long gc0 = tile * TPC;
        for (int e = (int)threadIdx.x; e < TPC * N; e += (int)blockDim.x) {
            const int q = e % TPC, k = e / TPC;
            const long long gc = gc0 + q;
            if (gc >= a.batch) continue;
            const long long b = gc >> sa.slog, c = gc & (S - 1);
            const C x = sm[Wk::keep_idx(k, q)];
            const long long o = b * sa.out_stride + (long long)k * S + c;
            const C y = FWD ? x : cswap(x);
            if constexpr (OL == kAoS) {
                __stcs(static_cast<C*>(sa.out0) + o, y);
            } else {
                __stcs(static_cast<F*>(sa.out0) + o, y.x);
                __stcs(static_cast<F*>(sa.out1) + o, y.y);
            }
        }
        __syncthreads();  // the store has read the buffer before the next tile writes it
    }
}

// ---------------------------------------------------------------- launch tables
constexpr int kMacroMaxG = 5;     // DIF stages per pass (1024-point units)
constexpr int kSegMinM = 8;       // micro orders with segment kernels
constexpr int kSegMaxM = 12;

using DifLaunchFn = cudaError_t (*)(const DifArgs&, cudaStream_t, const LaunchCtx&);
using SegLaunchFn = cudaError_t (*)(const SegArgs&, cudaStream_t, const LaunchCtx&);

struct MacroTable {
    DifLaunchFn first[kMacroMaxG][2][2][2];  // [G-1][fwd][input layout][last]
    DifLaunchFn mid[kMacroMaxG][2];          // [G-1][last]: later passes read scratch
    SegLaunchFn seg[kSegMaxM - kSegMinM + 1][2][2];  // [M - kSegMinM][fwd][output layout]
};

template <typename F, int G, bool FIRST, bool FWD, int IL, bool LAST>
cudaError_t launch_dif(const DifArgs& a, cudaStream_t stream, const LaunchCtx& ctx) {
    using Cfg = DifCfg<F, G>;
    auto kern = dif_pass_kernel<F, G, FIRST, FWD, IL, LAST>;
    static ResidentSlots slots;
    const int per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, Cfg::THREADS, Cfg::SMEM); });
    if (a.batch <= 0) return cudaSuccess;
    const long long items = a.batch * ((1LL << (a.order - 2 * G)) / Cfg::UPC);
    const long long cap = (long long)ctx.num_sms * per_sm;
    const unsigned grid = (unsigned)(items < cap ? items : cap);
    kern<<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(a);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

template <typename F, int M, bool FWD, int OL>
cudaError_t launch_seg(const SegArgs& a, cudaStream_t stream, const LaunchCtx& ctx) {
    using SC = SegCfg<F, M>;
    using Cfg = typename SC::W;
    auto kern = macro_seg_kernel<F, M, FWD, OL>;
    static ResidentSlots slots;
    const int per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, SC::BLOCK, Cfg::SMEM); });
    if (a.t.batch <= 0) return cudaSuccess;
    const long long tiles = (a.t.batch + Cfg::TPC - 1) / Cfg::TPC;
    const long long cap = (long long)ctx.num_sms * per_sm;
    const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    kern<<<grid, SC::BLOCK, Cfg::SMEM, stream>>>(a);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

template <typename F, int G>
void fill_macro_g(MacroTable& t) {
    auto& f = t.first[G - 1];
    f[1][kAoS][0] = launch_dif<F, G, true, true, kAoS, false>;
    f[1][kSoA][0] = launch_dif<F, G, true, true, kSoA, false>;
    f[0][kAoS][0] = launch_dif<F, G, true, false, kAoS, false>;
    f[0][kSoA][0] = launch_dif<F, G, true, false, kSoA, false>;
    f[1][kAoS][1] = launch_dif<F, G, true, true, kAoS, true>;
    f[1][kSoA][1] = launch_dif<F, G, true, true, kSoA, true>;
    f[0][kAoS][1] = launch_dif<F, G, true, false, kAoS, true>;
    f[0][kSoA][1] = launch_dif<F, G, true, false, kSoA, true>;
    t.mid[G - 1][0] = launch_dif<F, G, false, true, kAoS, false>;
    t.mid[G - 1][1] = launch_dif<F, G, false, true, kAoS, true>;
}

template <typename F, int M>
void fill_macro_seg(MacroTable& t) {
    auto& s = t.seg[M - kSegMinM];
    s[1][kAoS] = launch_seg<F, M, true, kAoS>;
    s[1][kSoA] = launch_seg<F, M, true, kSoA>;
    s[0][kAoS] = launch_seg<F, M, false, kAoS>;
    s[0][kSoA] = launch_seg<F, M, false, kSoA>;
}

template <typename F>
void fill_macro_dif(MacroTable& t) {
    fill_macro_g<F, 1>(t);
    fill_macro_g<F, 2>(t);
    fill_macro_g<F, 3>(t);
    fill_macro_g<F, 4>(t);
    fill_macro_g<F, 5>(t);
}

template <typename F>
void fill_macro_segs(MacroTable& t) {
    fill_macro_seg<F, 8>(t);
    fill_macro_seg<F, 9>(t);
    fill_macro_seg<F, 10>(t);
    fill_macro_seg<F, 11>(t);
    fill_macro_seg<F, 12>(t);
}

// Each translation unit fills its part of a precision's table.
void fill_macro_dif_f32(MacroTable& t);
void fill_macro_seg_f32(MacroTable& t);
void fill_macro_dif_f64(MacroTable& t);
void fill_macro_seg_f64(MacroTable& t);

}  // namespace zlfft
