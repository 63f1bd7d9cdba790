// G4: multi-pass Stockham FFT for transforms too large for one CTA.
//
// The reference's stage sequence for order P (radix-8 or radix-4 first pass,
// then radix-4 passes; src/common/zldsp_fft_common_init.hpp:193-206) is cut
// into 2 or 3 kernel passes over the same stage groups the tile kernel uses.
// A pass covering the stages from sub-length L_in to L_out = L_in * R works
// on "units" U = J * L_in + k (J < N / L_out, k < L_in): the R elements
// Y_{L_in}[J + rho * N / L_out][k] form a closed Stockham FFT of length R over
// rho whose twiddles are the global ones, W_{4L}^{q (k + L_in * k_local)}.
// Unit U reads positions U + pos * N / R and writes positions
// J * L_out + k + pos * L_in (pos < R), so the passes compose exactly to the
// reference's arithmetic: results are bit-identical to the single-CTA kernel.
//
// Layout in shared memory: element (pos, unit slot u) at pos * ROW + u with
// ROW = UPC + 1. Lanes run over units fastest, so every read, exchange write
// and global access of a half-warp touches 16 consecutive units (128 bytes
// of f32 complex) of one position, and the padded row also makes the
// column-wise copy-out of the first pass conflict-free. The 512- and
// 1024-point passes have fewer units per CTA; their rows share 128-byte lines
// and use an XOR-swizzled layout (pass_xidx).
//
// The first pass (sub-length 1 -> R) writes each unit's R results
// contiguously, so its CTA output is one contiguous block, copied out of
// shared memory with coalesced stores. Later passes store straight from
// registers (consecutive units are consecutive positions).
#pragma once

#include <cuda.h>

#include "zlfft_tile.cuh"

namespace zlfft {

// Pass schemes. Scheme 0 (every order): the tile kernel's stage groups
// (tile_group); from the end, pairs of radix-16 groups (256 points) form
// passes until the remaining leading groups fit 1024 points. Scheme 1 (orders
// 19 and 20, kPassSplitMinP..kPassSplitMaxP): the third group, radix 16 at
// sub-length L, runs as two radix-4 groups (stages L and 4L, the same
// butterflies and twiddles, so the same arithmetic), and the passes are
// groups [0, 3) and [3, 6): 512 | 1024 points for order 19, 1024 | 1024 for
// order 20, two passes over the data instead of three.
constexpr int kPassSplitMinP = 19;
constexpr int kPassSplitMaxP = 20;

__host__ __device__ constexpr int pass_num_groups(int P, int S) { return tile_num_groups(P) + (S == 1 ? 1 : 0); }

__host__ __device__ constexpr Grp pass_group(int P, int S, int g) {
    if (S == 0 || g < 2) return tile_group(P, g);
    if (g == 2) return Grp{4, tile_group(P, 2).L, 0, 1};
    if (g == 3) return Grp{4, 4 * tile_group(P, 2).L, 0, 1};
    return tile_group(P, g - 1);
}

__host__ __device__ constexpr int pass_count(int P, int S = 0) {
    if (S == 1) return 2;
    const int ng = tile_num_groups(P);
    int end = ng, n = 0;
    while (true) {
        int prod = 1;
        for (int g = 0; g < end; ++g) prod *= tile_group(P, g).R;
        if (prod <= 1024 || end <= 2) return n + 1;
        end -= 2;
        ++n;
    }
}

// First group index of pass i (0-based); pass i covers groups [pass_gb(i), pass_gb(i + 1)).
__host__ __device__ constexpr int pass_gb(int P, int i, int S = 0) {
    const int ng = pass_num_groups(P, S);
    const int np = pass_count(P, S);
    if (i >= np) return ng;
    if (i == 0) return 0;
    if (S == 1) return 3;
    // passes 1..np-1 are pairs of radix-16 groups at the end
    return ng - 2 * (np - i);
}

__host__ __device__ constexpr int pass_radix(int P, int i, int S = 0) {
    int r = 1;
    for (int g = pass_gb(P, i, S); g < pass_gb(P, i + 1, S); ++g) r *= pass_group(P, S, g).R;
    return r;
}

template <typename F, int P, int PI, int S = 0>
struct PassCfg {
    using C = Cx<F>;
    static_assert(S == 0 || (P >= kPassSplitMinP && P <= kPassSplitMaxP && tile_group(P, 2).R == 16),
                  "pass scheme 1: orders 19-20");
    static constexpr int N = 1 << P;
    static constexpr int GB = pass_gb(P, PI, S);
    static constexpr int GE = pass_gb(P, PI + 1, S);
    static constexpr int R = pass_radix(P, PI, S);
    static constexpr int L_IN = pass_group(P, S, GB).L;
    static constexpr int L_OUT = L_IN * R;
    static constexpr bool FIRST = (PI == 0);
    static constexpr bool LAST = (GE == pass_num_groups(P, S));
    static constexpr int E = [] {
        int e = 1;
        for (int g = GB; g < GE; ++g) e = pass_group(P, S, g).R > e ? pass_group(P, S, g).R : e;
        return e;
    }();
    static constexpr int T = R / E;  // threads per unit
    static constexpr int UMIN = 128 / (int)sizeof(C);  // units per 128-byte row
    // Units per CTA: whole 128-byte rows up to 256-point passes (256 threads);
    // the 512- and 1024-point passes keep 256 threads with 64- / 32-byte rows
    // (FP32), which leaves room for TMA staging and 2-3 resident CTAs. Measured
    // against 128-byte rows (CFFT<float> fast form, GB/s): order 17 (a 512-point
    // pass) 2571 -> 2942; order 18 (a 1024-point pass) 2117 -> 2670; FP64
    // order 18 2059 -> 2407.
    // (The passes below 256 points keep 128 threads: 256 measured 2-16% slower
    // at orders 19-21.)
    static constexpr int UPC = R >= 512 ? 256 * E / R : ((128 * E / R) > UMIN ? (128 * E / R) : UMIN);
    static constexpr int ROW = UPC + 1;
    static constexpr int THREADS = UPC * T;
    // Exchange layout. Rows of 128 bytes or more: [pos][unit] with one padding
    // element per row. Shorter rows (KROWS position rows per 128-byte line) are
    // unpadded and XOR-swizzled instead (pass_xidx).
    static constexpr int SLOTS = 128 / (int)sizeof(C);  // elements per 128-byte line
    static constexpr int KROWS = UPC >= SLOTS ? 1 : SLOTS / UPC;
    static constexpr size_t XBYTES = (size_t)R * (KROWS > 1 ? UPC : ROW) * sizeof(C);  // exchange buffer
    static constexpr size_t SOFF = (XBYTES + 127) / 128 * 128;     // staging offset (128-byte aligned)
    static constexpr size_t SBYTES = (size_t)R * UPC * sizeof(C);  // staging buffer
    // The next item's input (a box of UPC units x R positions) is prefetched
    // by one 3-D tensor copy per 256 positions while the current item computes.
    static constexpr int RB = R < 256 ? R : 256;  // positions per box
    static constexpr bool kTMA = SOFF + SBYTES + 16 + 1024 <= 200 * 1024;
    // (+1024: the buffers start at the first 1024-byte boundary of the dynamic
    // shared memory, as the swizzled output boxes of the first pass require)
    static constexpr size_t SMEM = (kTMA ? SOFF + SBYTES + 16 : XBYTES) + 1024;
    // Last pass with the RFFT split fused: the item's HALF low units (one box)
    // and a window of WIN = HALF + 2 units that holds their HALF mirrors
    // (split_unit; a mirror block starts at an odd unit, which no bulk copy
    // can, so the window starts at the even unit below it). With the 2 HALF
    // window of the first version the pass held two CTAs per SM instead of three.
    static constexpr int HALF = UPC / 2;
    static constexpr int WIN = HALF + 2;
    static constexpr size_t SBYTES_SPLIT = (size_t)(HALF + WIN) * R * sizeof(C);
    static constexpr bool kTMA_SPLIT = SOFF + SBYTES_SPLIT + 16 + 1024 <= 200 * 1024;
    static constexpr size_t SMEM_SPLIT = (kTMA_SPLIT ? SOFF + SBYTES_SPLIT + 16 : XBYTES) + 1024;
    // First pass: the CTA's output block (UPC units x R contiguous points) is
    // written by tensor stores of 128-byte-swizzled boxes, 128 bytes of points
    // x UPC units each, staged in the exchange buffer.
    static constexpr int CPB = 128 / (int)sizeof(C);  // points per box row
    static constexpr bool kStoreTMA = (L_IN == 1) && !LAST && (R % CPB == 0) && (UPC % 8 == 0) &&
                                      (size_t)UPC * R * sizeof(C) <= XBYTES;
    static constexpr int UNITS = N / R;            // units per transform
    static constexpr int CPT = UNITS / UPC;        // CTAs (work items) per transform
    // Resident CTAs per SM: as many as the shared memory allows, within a
    // budget of 80 registers per thread in FP32 and 96 in FP64 (a cap of ~100
    // made the FP64 plain form spill).
    static constexpr int SMEM_CTAS = (227 * 1024) / (int)(SMEM + 1024);
    static constexpr int REG_CTAS = 65536 / (THREADS * (sizeof(F) == 4 ? 80 : 96));
    static constexpr int MINB_ = SMEM_CTAS < REG_CTAS ? SMEM_CTAS : REG_CTAS;
    static constexpr int MINB = MINB_ > 0 ? MINB_ : 1;
    static_assert(UNITS % UPC == 0, "a transform must split into whole CTAs");
    static_assert(SMEM <= 200 * 1024, "pass tile too large");
};

struct PassArgs {
    const void* in0;  // first pass: user input (layout IL); else scratch (AoS complex)
    const void* in1;
    void* out0;       // last pass: user output (layout OL); else scratch (AoS complex)
    void* out1;
    long long batch;
    long long in_stride;   // elements between transforms of the input
    long long out_stride;  // elements between transforms of the output
    const void* tws;       // per-stage twiddle tables (stage_l0 layout)
    const void* tw;        // unified table T[t] = W_N^t, t < 3N/4 (tensor-core passes)
    const void* tctw;      // this pass's tensor-core twiddles when L_in > 1 (zlfft_tc_pass.cuh)
    const void* rw;        // RFFT split twiddle pairs (last pass with the split fused)
    int tma_out;           // first pass: the output map (PassMaps::mo) is valid, store by TMA
    int* err;              // device error word (kDevErrWaitTimeout on a timed-out wait)
    int tma;               // the tensor maps describe the input (else direct loads)
    int discard_in;        // the input is scratch that nothing reads after this pass: drop it from L2
    // Gathered transforms (mixed batches): the first pass reads transform t
    // at gin0[t] (gin1[t]) and the last pass writes it at gout0[t] (gout1[t]).
    const void* const* gin0;
    const void* const* gin1;
    void* const* gout0;
    void* const* gout1;
    // Gathered first pass (AoS): transform t's input tensor map is gmaps[t], in
    // device memory (a box of the same shape as PassMaps::m0 over that one
    // transform), so its items are prefetched by bulk copies as in the
    // contiguous case. Null: direct loads.
    const CUtensorMap* gmaps;
};

// Tensor maps of a pass input, encoded on the host (zlfft_launch.cuh): a 3-D
// view {units * comps, R positions, batch} of the AoS array (comps = 2
// interleaved re/im scalars) or of each SoA array (comps = 1).
struct PassMaps {
    CUtensorMap m0;
    CUtensorMap m1;
    CUtensorMap mo;  // first pass: the output, as rows of R points (one row per unit)
};

// XOR of the base-K digits of x (K = 2 or 4, x < 2^16). Linear over bits:
// the fold of a | b (disjoint bits) is fold(a) ^ fold(b).
template <int K>
__host__ __device__ constexpr int digit_fold(int x) {
    static_assert(K == 2 || K == 4, "two or four position rows per line");
    if constexpr (K == 4) {
        x ^= x >> 2;
        x ^= x >> 4;
        x ^= x >> 8;
        return x & 3;
    } else {
        x ^= x >> 1;
        x ^= x >> 2;
        x ^= x >> 4;
        x ^= x >> 8;
        return x & 1;
    }
}

// Exchange-buffer index of position pt | pc (disjoint bits: pt the thread's
// part, pc a part the compiler knows) and unit slot u.
// - 128-byte rows or more (KROWS == 1): [pos][u] with rows of UPC + 1.
// - Shorter rows: K = KROWS rows share a 128-byte line (line = pos / K). Row
//   pos takes row slot fold_K(pos) of its line, the XOR of pos's base-K
//   digits, and unit u takes slot u ^ (line mod UPC). The lanes of a half-warp
//   (a quarter-warp in FP64) then touch distinct banks for every access of the
//   kernel: K consecutive positions (group reads, position-major writes),
//   positions 2^j apart (a radix group's writes at sub-length ELL), and one
//   unit's consecutive positions (the first pass's copy-out). The padded
//   layout puts positions 16 apart on one bank; measured on the 1024-point
//   pass of CFFT<float> order 18, 40% of its shared-memory wavefronts were
//   conflicts.
template <class Cfg>
__host__ __device__ __forceinline__ int pass_xidx(int pt, int pc, int u) {
    if constexpr (Cfg::KROWS == 1) {
        return (pt + pc) * Cfg::ROW + u;
    } else {
        constexpr int K = Cfg::KROWS, LK = K == 4 ? 2 : 1;
        const int lt = pt >> LK, lc = pc >> LK;
        const int x = ((digit_fold<K>(pt) ^ digit_fold<K>(pc)) * Cfg::UPC) | ((u ^ lt ^ lc) & (Cfg::UPC - 1));
        return (lt + lc) * Cfg::SLOTS + x;
    }
}

// Unit of slot u in work item ib of a last pass with the RFFT split fused:
// the first half of the slots take units HALF*ib + u, the second half their
// mirrors L_in - (HALF*ib + u) (unit L_in/2 stands in for the mirror of unit
// 0), so every Z[k] of the item meets Z[M - k] in the same CTA: position
// p = k + pos * L_in of a low unit k >= 1 mirrors to unit L_in - k at
// position R - 1 - pos.
template <int L_IN, int UPC>
__device__ __forceinline__ int split_unit(int ib, int u) {
    constexpr int HALF = UPC / 2;
    if (u < HALF) return HALF * ib + u;
    const int v = HALF * ib + (u - HALF);
    return v == 0 ? L_IN / 2 : L_IN - v;
}

// One pass over `batch` transforms. FWD selects the direction swap on the
// first pass's loads and the last pass's stores (the reference's backward
// transform is swap(DFT(swap(x))), src/common/zldsp_fft_common_structure.hpp:47-95).
//
// SPLIT (kR2CFwd or kR2CSqrMag, last pass of an RFFT forward only) fuses the
// RFFT split: the item's spectrum values go to shared memory in [pos][slot]
// order, the slots hold mirror pairs of units (split_unit), and the epilogue
// writes bins k and M - k of every pair with the reference's arithmetic
// (src/common/zldsp_fft_common_execute.hpp:318-368, :481-536), as
// rfft_split_kernel does.
//
// FAST selects the fast-twiddle form of the radix-16 groups (group16_fast).
template <typename F, int P, int PI, bool FWD, int IL, int OL, int SPLIT = 0, bool FAST = false, int S = 0>
__global__ void __launch_bounds__(PassCfg<F, P, PI, S>::THREADS, PassCfg<F, P, PI, S>::MINB)
    pass_kernel(const PassArgs a, const __grid_constant__ PassMaps maps) {
    using Cfg = PassCfg<F, P, PI, S>;
    using C = Cx<F>;
    constexpr int N = Cfg::N, R = Cfg::R, E = Cfg::E, T = Cfg::T, UPC = Cfg::UPC, ROW = Cfg::ROW;
    constexpr int L_IN = Cfg::L_IN, L_OUT = Cfg::L_OUT, GB = Cfg::GB, GE = Cfg::GE;
    constexpr int IL2 = Cfg::FIRST ? IL : (int)kAoS;
    constexpr int OL2 = Cfg::LAST ? OL : (int)kAoS;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    // first 1024-byte boundary, as an offset into the shared array (keeps the
    // pointer in the shared address space for the compiler)
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    C* sm = reinterpret_cast<C*>(smem);
    const int u = (int)threadIdx.x % UPC;
    const int tb = (int)threadIdx.x / UPC;
    const C* tws = static_cast<const C*>(a.tws);
    const long long items = a.batch * Cfg::CPT;

    // ---- TMA staging: [pos][u] unpadded (SoA: a re plane then an im plane)
    constexpr bool kSoAIn = (IL2 == kSoA);
    constexpr int CMP = kSoAIn ? 1 : 2;  // scalars per unit in the map's innermost dimension
    C* stage = reinterpret_cast<C*>(smem + Cfg::SOFF);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + Cfg::SOFF + (SPLIT != 0 ? Cfg::SBYTES_SPLIT : Cfg::SBYTES));
    const bool store_tma = Cfg::kStoreTMA && a.tma_out;
    static_assert(SPLIT == 0 || (Cfg::LAST && FWD && L_IN > 1 && Cfg::UPC >= 2 && Cfg::KROWS == 1),
                  "split fusion: RFFT forward last pass (padded layout)");
    const bool use_tma = (SPLIT == 0 ? Cfg::kTMA : Cfg::kTMA_SPLIT) && a.tma;
    // split pass: the first unit of item ib's mirror window (item 0's window is
    // the last WIN units, which hold its mirrors L_IN - 1 .. L_IN - (HALF - 1);
    // its remaining slot, unit L_IN / 2, is read directly)
    auto split_ws = [](int ib) { return ib == 0 ? L_IN - Cfg::WIN : L_IN - Cfg::HALF * ib - Cfg::HALF; };
    auto issue = [&](long long it) {  // one thread issues the item's box copies
        if (!use_tma || threadIdx.x != 0 || it >= items) return;
        if constexpr (SPLIT != 0) {
            constexpr int H = Cfg::HALF;
            const int z = (int)(it / Cfg::CPT);
            const int ib = (int)(it % Cfg::CPT);
            mbar_arrive_expect_tx(bar, (uint32_t)Cfg::SBYTES_SPLIT);
            C* lo = stage;
            C* win = stage + (size_t)H * R;
#pragma unroll
            for (int y = 0; y < R; y += Cfg::RB) {
                tma_load_3d(lo + (size_t)y * H, &maps.m0, H * ib * 2, y, z, bar);
                tma_load_3d(win + (size_t)y * Cfg::WIN, &maps.m1, split_ws(ib) * 2, y, z, bar);
            }
            return;
        }
        int z = (int)(it / Cfg::CPT);
        const int x = (int)(it % Cfg::CPT) * UPC * CMP;  // x * sizeof(F) = 16-byte multiple
        const CUtensorMap* m0 = &maps.m0;
        if constexpr (Cfg::FIRST && !kSoAIn) {
            if (a.gmaps) {  // gathered: the transform's own map, batch coordinate 0
                m0 = a.gmaps + z;
                z = 0;
            }
        }
        mbar_arrive_expect_tx(bar, (uint32_t)Cfg::SBYTES);
        F* sf = reinterpret_cast<F*>(stage);
#pragma unroll
        for (int y = 0; y < R; y += Cfg::RB) {
            if constexpr (kSoAIn) {
                tma_load_3d(sf + (size_t)y * UPC, &maps.m0, x, y, z, bar);
                tma_load_3d(sf + (size_t)R * UPC + (size_t)y * UPC, &maps.m1, x, y, z, bar);
            } else {
                tma_load_3d(stage + (size_t)y * UPC, m0, x, y, z, bar);
            }
        }
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

    // Fast form: the two table twiddles of each radix-16 group (a thread runs
    // one butterfly per such group: E == 16), loaded at the item's start,
    // ahead of the input wait.
    [[maybe_unused]] C fw[GE - GB][2];
    auto load_fw = [&](int ku) {
        if constexpr (FAST) {
            [&]<int... GI>(std::integer_sequence<int, GI...>) {
                (
                    [&] {
                        constexpr Grp G = pass_group(P, S, GB + GI);
                        if constexpr (G.R == 16 && !G.first) {
                            static_assert(G.R == E, "one radix-16 butterfly per thread");
                            constexpr int ELL = G.L / L_IN;
                            const uint32_t kk = (uint32_t)(ku + L_IN * (tb % ELL));
                            group16_fast_tw<P, G.L>(kk, tws, fw[GI][0], fw[GI][1]);
                        }
                    }(),
                    ...);
            }(std::make_integer_sequence<int, GE - GB>{});
        }
    };

    for (long long item = blockIdx.x; item < items; item += gridDim.x) {
        // the previous item's output stores have read the exchange buffer before
        // anyone writes it again (the first write follows a barrier)
        if (store_tma && threadIdx.x == 0) bulk_wait_read0();
        const long long tr = item / Cfg::CPT;
        const int ib = (int)(item % Cfg::CPT);
        const int U = SPLIT ? split_unit<L_IN, UPC>(ib, u) : ib * UPC + u;
        const int ku = U % L_IN;  // k of the unit
        const int J = U / L_IN;
        load_fw(ku);
        C v[E];
        if constexpr (Cfg::kTMA) {
            if (use_tma) {
                const bool ok = mbar_wait(bar, phase);
                if (__syncthreads_or(!ok)) {  // bounded wait ran out: report and leave
                    if (threadIdx.x == 0) atomicOr(a.err, kDevErrWaitTimeout);
                    mbar_wait(bar, phase);
                    if (store_tma && threadIdx.x == 0) bulk_wait0();
                    return;
                }
                phase ^= 1u;
            }
        }

        [&]<int... GI>(std::integer_sequence<int, GI...>) {
            (
                [&] {
                    constexpr int g = GB + GI;
                    constexpr Grp G = pass_group(P, S, g);
                    constexpr int NB = E / G.R;
                    constexpr int ELL = G.L / L_IN;  // local sub-length at group entry
                    constexpr bool kLastG = (g + 1 == GE);
                    // ---- inputs
                    if constexpr (GI == 0) {
                        if (use_tma && SPLIT != 0) {
                            // low slots from the low box; mirror slots from the window
                            // (slot H + j holds unit L_IN - (H ib + j)), except item 0's
                            // slot H, unit L_IN / 2, read directly
                            constexpr int H = Cfg::HALF;
                            const C* lo = stage;
                            const C* win = stage + (size_t)H * R;
                            const bool direct = (ib == 0 && u == H);
                            const int off = u < H ? u : (L_IN - (H * ib + (u - H))) - split_ws(ib);
                            const C* src = static_cast<const C*>(a.in0) + tr * a.in_stride + U;
#pragma unroll
                            for (int i = 0; i < NB; ++i) {
                                const int b = tb + i * T;
#pragma unroll
                                for (int rho = 0; rho < G.R; ++rho) {
                                    const int pos = b + rho * (R / G.R);
                                    v[i * G.R + rho] = direct ? src[(size_t)pos * (N / R)]
                                                       : (u < H ? lo[pos * H + off] : win[pos * Cfg::WIN + off]);
                                }
                            }
                            fence_proxy_async_smem();  // reads of the staging buffer before its TMA refill
                            __syncthreads();           // staging fully read: refill it with the next item
                            issue(item + gridDim.x);
                        } else if (use_tma) {
                            const F* sf = reinterpret_cast<const F*>(stage);
#pragma unroll
                            for (int i = 0; i < NB; ++i) {
                                const int b = tb + i * T;
#pragma unroll
                                for (int rho = 0; rho < G.R; ++rho) {
                                    const int pos = b + rho * (R / G.R);
                                    C x = kSoAIn ? cx<C>(sf[pos * UPC + u], sf[R * UPC + pos * UPC + u])
                                                 : stage[pos * UPC + u];
                                    v[i * G.R + rho] = (Cfg::FIRST && !FWD) ? cswap(x) : x;
                                }
                            }
                            fence_proxy_async_smem();  // reads of the staging buffer before its TMA refill
                            __syncthreads();           // staging fully read: refill it with the next item
                            issue(item + gridDim.x);
                        } else {
                            const bool g = Cfg::FIRST && a.gin0 != nullptr;
                            const CxIn<F, IL2> in(g ? a.gin0[tr] : a.in0, g ? (a.gin1 ? a.gin1[tr] : nullptr) : a.in1,
                                                  g ? 0 : tr * a.in_stride);
#pragma unroll
                            for (int i = 0; i < NB; ++i) {
                                const int b = tb + i * T;
#pragma unroll
                                for (int rho = 0; rho < G.R; ++rho) {
                                    const int pos = b + rho * (R / G.R);
                                    C x = in[U + pos * (N / R)];
                                    v[i * G.R + rho] = (Cfg::FIRST && !FWD) ? cswap(x) : x;
                                }
                            }
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
                            const int b = tb + i * T;
#pragma unroll
                            for (int rho = 0; rho < G.R; ++rho)
                                v[i * G.R + rho] = sm[pass_xidx<Cfg>(tb, b - tb + rho * (R / G.R), u)];
                        }
                    }
                    // ---- compute (global twiddles: kk = ku + L_IN * k_local)
#pragma unroll
                    for (int i = 0; i < NB; ++i) {
                        const int b = tb + i * T;
                        const uint32_t kk = (uint32_t)(ku + L_IN * (b % ELL));
                        if constexpr (FAST && G.R == 16 && !G.first) {
                            group16_fast_w(v + i * G.R, fw[GI][0], fw[GI][1]);
                        } else {
                            group_compute_ld<P, G.R, G.L, G.first>(v + i * G.R, kk, tws);
                        }
                    }
                    // ---- outputs
                    if constexpr (!kLastG) {
                        __syncthreads();
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
                            // position Jl * R_g * ELL + kl + mu * ELL of butterfly b = tb + i * T
                            // (Jl = b / ELL, kl = b % ELL), split into the parts of tb and i * T
                            const int pt = (tb / ELL) * G.R * ELL + tb % ELL;
                            const int pi = ((i * T) / ELL) * G.R * ELL + (i * T) % ELL;
#pragma unroll
                            for (int s = 0; s < G.R; ++s)
                                sm[pass_xidx<Cfg>(pt, pi + group_mu(G, s) * ELL, u)] = v[i * G.R + s];
                        }
                        __syncthreads();
                    } else if constexpr (L_IN == 1) {
                        if constexpr (Cfg::kStoreTMA) {
                            if (store_tma) {
                                // first pass: the CTA's output block (UPC units x R contiguous
                                // points) as R / CPB boxes [unit][CPB points], 128-byte swizzled
                                // (16-byte chunk c of unit row u at chunk c ^ (u & 7)), written by
                                // tensor stores while the next item computes
                                constexpr int CPB = Cfg::CPB;
                                __syncthreads();
#pragma unroll
                                for (int i = 0; i < NB; ++i) {
                                    const int b = tb + i * T;
#pragma unroll
                                    for (int s = 0; s < G.R; ++s) {
                                        const int pos = b + group_mu(G, s) * ELL;
                                        const uint32_t cb = (uint32_t)((pos % CPB) * (int)sizeof(C));
                                        const uint32_t off = (uint32_t)(pos / CPB) * (uint32_t)(UPC * 128) +
                                                             (uint32_t)u * 128u + ((((cb >> 4) ^ (uint32_t)(u & 7))) << 4) +
                                                             (cb & 15u);
                                        *reinterpret_cast<C*>(smem + off) = v[i * G.R + s];
                                    }
                                }
                                fence_proxy_async_smem();  // generic writes before the async-proxy reads
                                __syncthreads();
                                if (threadIdx.x == 0) {
                                    const int y = (int)(tr * Cfg::UNITS + (U - u));
                                    const uint64_t pol = l2_policy_evict_last();  // the next pass reads it from L2
#pragma unroll 1
                                    for (int bx = 0; bx < R / CPB; ++bx)
                                        tma_store_2d_hint(&maps.mo, bx * CPB * 2, y, smem + (size_t)bx * UPC * 128, pol);
                                    bulk_commit();
                                }
                                return;
                            }
                        }
                        // first pass: each unit's outputs are contiguous; stage them and copy
                        // the CTA's block (UPC units x R) out with consecutive threads on
                        // consecutive elements.
                        __syncthreads();
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
                            const int b = tb + i * T;  // J_local == 0 in the last group
#pragma unroll
                            for (int s = 0; s < G.R; ++s)
                                sm[pass_xidx<Cfg>(tb, b - tb + group_mu(G, s) * ELL, u)] = v[i * G.R + s];
                        }
                        __syncthreads();
                        const bool g = Cfg::LAST && a.gout0 != nullptr;
                        const CxOut<F, OL2> out(g ? a.gout0[tr] : a.out0, g ? (a.gout1 ? a.gout1[tr] : nullptr) : a.out1,
                                                (g ? 0 : tr * a.out_stride) + (long long)(U - u) * R);
                        if constexpr (Cfg::KROWS == 1) {
#pragma unroll 4
                            for (int e = (int)threadIdx.x; e < UPC * R; e += Cfg::THREADS) {
                                const int uu = e / R, pos = e % R;
                                const C x = sm[pos * ROW + uu];
                                out.put(e, (Cfg::LAST && !FWD) ? cswap(x) : x);
                            }
                        } else {
                            // element e = t + k * THREADS: unit e / R = k * THREADS / R, position
                            // t + (k * THREADS) % R (THREADS divides R here)
                            static_assert(R % Cfg::THREADS == 0, "swizzled copy-out: whole passes over R");
                            const int t = (int)threadIdx.x;
#pragma unroll
                            for (int k = 0; k < UPC * R / Cfg::THREADS; ++k) {
                                const int e = t + k * Cfg::THREADS;
                                const C x = sm[pass_xidx<Cfg>(t, (k * Cfg::THREADS) % R, (k * Cfg::THREADS) / R)];
                                out.put(e, (Cfg::LAST && !FWD) ? cswap(x) : x);
                            }
                        }
                        __syncthreads();
                    } else if constexpr (SPLIT != 0) {
                        // spectrum values of the item to shared memory, [pos][slot]
                        __syncthreads();
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
                            const int b = tb + i * T;
#pragma unroll
                            for (int s = 0; s < G.R; ++s)
                                sm[pass_xidx<Cfg>(tb, b - tb + group_mu(G, s) * ELL, u)] = v[i * G.R + s];
                        }
                    } else {
                        const bool g = Cfg::LAST && a.gout0 != nullptr;
                        const CxOut<F, OL2> out(g ? a.gout0[tr] : a.out0, g ? (a.gout1 ? a.gout1[tr] : nullptr) : a.out1,
                                                (g ? 0 : tr * a.out_stride) + (long long)J * L_OUT + ku);
#pragma unroll
                        for (int i = 0; i < NB; ++i) {
                            const int b = tb + i * T;
#pragma unroll
                            for (int s = 0; s < G.R; ++s) {
                                const int pos = b + group_mu(G, s) * ELL;
                                const C x = v[i * G.R + s];
                                out.put(pos * L_IN, (Cfg::LAST && !FWD) ? cswap(x) : x);
                            }
                        }
                    }
                }(),
                ...);
        }(std::make_integer_sequence<int, GE - GB>{});
        // The item's input rows (UPC consecutive units x R positions of AoS
        // scratch: each position's units are one run of UPC * sizeof(C) bytes)
        // are dead when nothing reads them after this pass: drop them from L2
        // rather than let L2 write them back to DRAM. Every thread's loaded
        // values have fed its stores of this item, so after the barrier no load
        // of the item is outstanding. (Rows under 128 bytes share their lines
        // with items that other CTAs may still be reading, so those passes keep
        // their input. Running a line's items one after another on one CTA, to
        // drop the line after the last, measured 10% slower on the 1024-point
        // passes: neighbouring CTAs no longer read the same lines together.)
        if constexpr (IL2 == kAoS && SPLIT == 0 && (UPC * sizeof(C)) % 128 == 0) {
            if (a.discard_in) {
                __syncthreads();
                constexpr int LPR = (int)(UPC * sizeof(C)) / 128;  // lines per position row
                const char* ib =
                    reinterpret_cast<const char*>(static_cast<const C*>(a.in0) + tr * a.in_stride + (U - u));
                for (int l = (int)threadIdx.x; l < R * LPR; l += Cfg::THREADS) {
                    const int pos = l / LPR, sub = l % LPR;
                    discard_l2_line(ib + (size_t)pos * (N / R) * sizeof(C) + (size_t)sub * 128);
                }
            }
        }
        if constexpr (SPLIT != 0) {
            // ---- fused RFFT split over the item's mirror pairs (M = N complex points)
            __syncthreads();
            constexpr int HALF = UPC / 2;
            const bool first_item = (ib == 0);
            const int tasks = HALF * R + (first_item ? 1 : 0);
            const C* rw = static_cast<const C*>(a.rw);
            const bool g = a.gout0 != nullptr;
            void* o0 = g ? a.gout0[tr] : a.out0;
            void* o1 = g ? (a.gout1 ? a.gout1[tr] : nullptr) : a.out1;
            const long long ob = g ? 0 : tr * a.out_stride;
            constexpr int OLS = (SPLIT == kR2CSqrMag) ? (int)kAoS : OL;
            const CxOut<F, OLS> out(o0, o1, ob);
            F* osq = static_cast<F*>(o0) + ob;
            // task t: the bin pair of slot pair (s1, s2) at positions (p1, p2)
            auto pair_of = [&](int t, int& s1, int& p1, int& s2, int& p2) {
                const int pos = t / HALF, us = t % HALF;
                if (first_item && us == 0) {
                    if (pos <= R / 2) {  // unit 0 pairs with itself
                        s1 = 0;
                        p1 = pos;
                        s2 = 0;
                        p2 = (R - pos) & (R - 1);
                    } else {  // unit L_in/2 pairs with itself
                        const int ph = pos - R / 2 - 1;
                        s1 = HALF;
                        p1 = ph;
                        s2 = HALF;
                        p2 = R - 1 - ph;
                    }
                } else {
                    s1 = us;
                    p1 = pos;
                    s2 = us + HALF;
                    p2 = R - 1 - pos;
                }
            };
            auto task = [&](int t, const C w) {
                int s1, p1, s2, p2;
                pair_of(t, s1, p1, s2, p2);
                const int g1 = split_unit<L_IN, UPC>(ib, s1) + p1 * L_IN;
                if (g1 == 0) {  // DC and Nyquist from Z[0]
                    const C z0 = sm[p1 * ROW + s1];
                    const F dc = z0.x + z0.y, ny = z0.x - z0.y;
                    if constexpr (SPLIT == kR2CFwd) {
                        out.put(0, cx<C>(dc, (F)0));
                        out.put(N, cx<C>(ny, (F)0));
                    } else {
                        osq[0] = mul_rn(dc, dc);
                        osq[N] = mul_rn(ny, ny);
                    }
                    return;
                }
                const C za = sm[p1 * ROW + s1], zb = sm[p2 * ROW + s2];
                const bool low = g1 <= N / 2;  // k = min(g1, N - g1)
                const int k = low ? g1 : N - g1;
                const SplitOut<F> o = rfft_split<F>(low ? za : zb, low ? zb : za, w.x, w.y);
                if constexpr (SPLIT == kR2CFwd) {
                    if (k != N / 2) out.put(k, cx<C>(o.xr_k, o.xi_k));
                    out.put(N - k, cx<C>(o.xr_m, o.xi_m));
                } else {
                    if (k != N / 2) osq[k] = fma_rn(o.xr_k, o.xr_k, mul_rn(o.xi_k, o.xi_k));
                    osq[N - k] = fma_rn(o.xr_m, o.xr_m, mul_rn(o.xi_m, o.xi_m));
                }
            };
            auto twiddle = [&](int t) -> C {  // the pair's split twiddle (unused for DC / Nyquist)
                int s1, p1, s2, p2;
                pair_of(t, s1, p1, s2, p2);
                const int g1 = split_unit<L_IN, UPC>(ib, s1) + p1 * L_IN;
                return g1 == 0 ? cx<C>((F)0, (F)0) : rw[g1 <= N / 2 ? g1 : N - g1];
            };
            // The HALF * R regular tasks, NT per thread: every twiddle is loaded
            // before the first is used (looped one task at a time, each task's
            // L2 round trip stalled the CTA: 8 per item).
            constexpr int NT = HALF * R / Cfg::THREADS;
            static_assert(HALF * R % Cfg::THREADS == 0, "split tasks: whole rounds of the CTA");
            C wv[NT];
#pragma unroll
            for (int j = 0; j < NT; ++j) wv[j] = twiddle((int)threadIdx.x + j * Cfg::THREADS);
#pragma unroll
            for (int j = 0; j < NT; ++j) task((int)threadIdx.x + j * Cfg::THREADS, wv[j]);
            if (tasks > HALF * R && threadIdx.x == 0) task(HALF * R, twiddle(HALF * R));  // item 0's last pair
        }
        // shared memory is rewritten by the next item's first exchange only after a barrier
    }
    if (store_tma && threadIdx.x == 0) bulk_wait0();  // stores done before the CTA's shared memory goes
}

// ---------------------------------------------------------------- RFFT split / pre-step
// Stand-alone forms for the multi-pass orders: the forward split reads the
// N/2-point spectrum Z (AoS, natural order) and writes bins (or squared
// magnitudes); the backward pre-step writes Z from bins
// (src/common/zldsp_fft_common_execute.hpp:318-368, :481-536, :399-451).
// One thread per bin pair (k, M - k), k = 0 .. M/2 (k = 0 is DC/Nyquist):
// grid x covers the pairs of a transform, grid y strides over the transforms
// (no 64-bit division per element).
template <typename F, int OP, int LAYOUT>
__global__ void rfft_split_kernel(const Cx<F>* z, void* out0, void* out1, const Cx<F>* rw, int M, long long batch,
                                  long long z_stride, long long out_stride, void* const* gout0, void* const* gout1) {
    using C = Cx<F>;
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k > M / 2) return;
    const C w = k > 0 ? rw[k] : cx<C>((F)0, (F)0);  // the pair's twiddles, for every transform
    for (long long tr = blockIdx.y; tr < batch; tr += gridDim.y) {
        const C* zt = z + tr * z_stride;
        constexpr int OL2 = (OP == kR2CSqrMag) ? (int)kAoS : LAYOUT;
        void* o0 = gout0 ? gout0[tr] : out0;
        void* o1 = gout0 ? (gout1 ? gout1[tr] : nullptr) : out1;
        const long long ob = gout0 ? 0 : tr * out_stride;
        const CxOut<F, OL2> out(o0, o1, ob);
        F* osq = static_cast<F*>(o0) + ob;
        if (k == 0) {
            const C z0 = zt[0];
            const F dc = z0.x + z0.y, ny = z0.x - z0.y;
            if constexpr (OP == kR2CFwd) {
                out.put(0, cx<C>(dc, (F)0));
                out.put(M, cx<C>(ny, (F)0));
            } else {
                osq[0] = mul_rn(dc, dc);
                osq[M] = mul_rn(ny, ny);
            }
            continue;
        }
        const SplitOut<F> o = rfft_split<F>(zt[k], zt[M - k], w.x, w.y);
        if constexpr (OP == kR2CFwd) {
            if (k != M / 2) out.put(k, cx<C>(o.xr_k, o.xi_k));
            out.put(M - k, cx<C>(o.xr_m, o.xi_m));
        } else {
            if (k != M / 2) osq[k] = fma_rn(o.xr_k, o.xr_k, mul_rn(o.xi_k, o.xi_k));
            osq[M - k] = fma_rn(o.xr_m, o.xr_m, mul_rn(o.xi_m, o.xi_m));
        }
    }
}

template <typename F, int LAYOUT>
__global__ void rfft_pre_kernel(const void* in0, const void* in1, Cx<F>* z, const Cx<F>* rw, int M, long long batch,
                                long long in_stride, long long z_stride, const void* const* gin0,
                                const void* const* gin1) {
    using C = Cx<F>;
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k > M / 2) return;
    const C w = k > 0 ? rw[k] : cx<C>((F)0, (F)0);  // the pair's twiddles, for every transform
    for (long long tr = blockIdx.y; tr < batch; tr += gridDim.y) {
        const CxIn<F, LAYOUT> in(gin0 ? gin0[tr] : in0, gin0 ? (gin1 ? gin1[tr] : nullptr) : in1,
                                 gin0 ? 0 : tr * in_stride);
        C* zt = z + tr * z_stride;
        if (k == 0) {
            const C x0 = in[0], xm = in[M];
            zt[0] = cx<C>(mul_rn(x0.x + xm.x, (F)0.5), mul_rn(x0.x - xm.x, (F)0.5));
            continue;
        }
        const C x1 = in[k], x2 = in[M - k];
        const F c = w.x, s = w.y;
        const F si = x1.y + x2.y, dr = x1.x - x2.x;
        const C zk = cx<C>(fma_rn(-dr, s, fma_rn(-si, c, x1.x)), fma_rn(dr, c, fma_rn(-si, s, x1.y)));
        const C zm = cx<C>(fma_rn(dr, s, fma_rn(si, c, x2.x)), fma_rn(dr, c, fma_rn(-si, s, x2.y)));
        if (k != M / 2) zt[k] = zk;
        zt[M - k] = zm;
    }
}

}  // namespace zlfft
