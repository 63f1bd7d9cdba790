// Launch tables: every (precision, order, operation, layout) kernel variant is
// instantiated once at build time and reached through a table of launch
// functions, so the C ABI dispatches with one indexed load.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <stdlib.h>
#include <string.h>

#include <atomic>

#include "zlfft_pass.cuh"
#include "zlfft_resident.cuh"
#include "zlfft_tc_pass.cuh"
#include "zlfft_tc_pipe.cuh"
#include "zlfft_tile.cuh"

namespace zlfft {

constexpr int kTileMaxP_f32 = 14;  // tile kernel: whole transform in one CTA
constexpr int kTileMaxP_f64 = 13;
constexpr int kTileMaxP = 13;      // orders every path treats as single-CTA
// FP32 order 14 (128 KB, one CTA per SM) has tile kernels too: the CFFT of
// order 14 and the RFFT of real order 15 run on them from the batched and
// mixed entry points (one pass over HBM; the other paths keep the multi-pass
// form).
constexpr int kTileTableP = 14;

struct LaunchCtx {
    int num_sms;
    std::atomic<size_t>* launches;  // incremented per kernel launch
};

using TileLaunchFn = cudaError_t (*)(const TileArgs&, cudaStream_t, const LaunchCtx&);

struct TileTable {
    // [order][op][in_layout][out_layout]
    TileLaunchFn fn[kTileTableP + 1][5][2][2];
    // STFT front end: RFFT forward with the window multiplied in at load,
    // [order][0: forward, 1: forward_sqr_mag][out_layout]
    TileLaunchFn stft[kTileTableP + 1][2][2];
    // fast-twiddle form of the orders with middle radix-16 groups (11..13),
    // AoS input: [order][op][out_layout]
    TileLaunchFn fast[kTileTableP + 1][5][2];
};

template <typename F, int P, int OP, int IL, int OL, bool WIN = false, bool FAST = false>
cudaError_t launch_tile(const TileArgs& a, cudaStream_t stream, const LaunchCtx& ctx) {
    using Cfg = TileCfg<F, P, OP>;
    auto kern = tile_kernel<F, P, OP, IL, OL, false, WIN, FAST>;
    static ResidentSlots slots;
    const int blocks_per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, Cfg::THREADS, Cfg::SMEM); });
    if (a.batch <= 0) return cudaSuccess;
    const long long tiles = (a.batch + Cfg::TPC - 1) / Cfg::TPC;
    const long long cap = (long long)ctx.num_sms * blocks_per_sm;
    const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    kern<<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(a);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

// ------------------------------------------------------------------ gathered tile launches
// Tile kernels reading/writing per-transform pointers (mixed batches), for
// the AoS <-> AoS operations: [order][op].
struct GatherTable {
    TileLaunchFn fn[kTileTableP + 1][5];
    TileLaunchFn fast[kTileTableP + 1][5];  // the fast-twiddle form, orders 11 and up (not C2R)
};

template <typename F, int P, int OP, bool FAST = false>
cudaError_t launch_tile_gather(const TileArgs& a, cudaStream_t stream, const LaunchCtx& ctx) {
    using Cfg = TileCfg<F, P, OP>;
    auto kern = tile_kernel<F, P, OP, kAoS, kAoS, true, false, FAST>;
    static ResidentSlots slots;
    const int blocks_per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, Cfg::THREADS, Cfg::SMEM); });
    if (a.batch <= 0) return cudaSuccess;
    const long long tiles = (a.batch + Cfg::TPC - 1) / Cfg::TPC;
    const long long cap = (long long)ctx.num_sms * blocks_per_sm;
    const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    kern<<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(a);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

template <typename F, int P>
void fill_gather_fast(GatherTable& t) {
    if constexpr (P >= 11) {
        t.fast[P][kC2CFwd] = launch_tile_gather<F, P, kC2CFwd, true>;
        t.fast[P][kC2CBwd] = launch_tile_gather<F, P, kC2CBwd, true>;
        t.fast[P][kR2CFwd] = launch_tile_gather<F, P, kR2CFwd, true>;
        t.fast[P][kR2CSqrMag] = launch_tile_gather<F, P, kR2CSqrMag, true>;
    }
}

template <typename F, int... Ps>
void fill_gather_orders(GatherTable& t, std::integer_sequence<int, Ps...>) {
    ((t.fn[Ps][kC2CFwd] = launch_tile_gather<F, Ps, kC2CFwd>, t.fn[Ps][kC2CBwd] = launch_tile_gather<F, Ps, kC2CBwd>,
      t.fn[Ps][kR2CFwd] = launch_tile_gather<F, Ps, kR2CFwd>, t.fn[Ps][kR2CSqrMag] = launch_tile_gather<F, Ps, kR2CSqrMag>,
      t.fn[Ps][kC2RBwd] = launch_tile_gather<F, Ps, kC2RBwd>, fill_gather_fast<F, Ps>(t)),
     ...);
}
void fill_gather_f32(GatherTable& t);
void fill_gather_f64(GatherTable& t);

// ------------------------------------------------------------------ multi-pass
constexpr int kPassMinP = 14;
constexpr int kPassMaxP = 26;  // three passes reach order 26
constexpr int kMaxPasses = 3;

using PassLaunchFn = cudaError_t (*)(const PassArgs&, cudaStream_t, const LaunchCtx&);

struct PassTable {
    // [order - kPassMinP][pass][fwd][in_layout][out_layout]; the layouts only
    // matter on the first (input) and last (output) pass.
    PassLaunchFn fn[kPassMaxP - kPassMinP + 1][kMaxPasses][2][2][2];
    // [order - kPassMinP][0: RFFT forward, 1: forward_sqr_mag][output layout]: the
    // last pass with the RFFT split fused (the N/2-point spectrum never leaves the CTA)
    PassLaunchFn split[kPassMaxP - kPassMinP + 1][2][2];
    // [order - kPassMinP][pass][fwd]: the fast-twiddle form, AoS in and out
    PassLaunchFn fast[kPassMaxP - kPassMinP + 1][kMaxPasses][2];
    // [order - kPassMinP]: the first pass's points per unit (R), units per CTA,
    // positions per input box and whether it stages its input (gathered maps)
    int first_geom[kPassMaxP - kPassMinP + 1][4];
};

// cuTensorMapEncodeTiled, reached through the runtime's driver entry point
// (no link-time dependency on libcuda).
inline PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled fn = []() -> PFN_cuTensorMapEncodeTiled {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    }();
    return fn;
}

// Encode the input maps of a pass: {units * comps, R, batch} with strides
// {N/R * comps, transform stride} scalars; box {UPC * comps, RB, 1}.
// Returns false (direct loads) when the source does not meet TMA rules.
template <typename F, int P, int PI, int IL2, int S = 0>
bool encode_pass_maps(const PassArgs& a, PassMaps& m) {
    using Cfg = PassCfg<F, P, PI, S>;
    if (!Cfg::kTMA) return false;
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    constexpr int CMP = IL2 == kSoA ? 1 : 2;
    const CUtensorMapDataType dt = sizeof(F) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t row_bytes = (cuuint64_t)(Cfg::N / Cfg::R) * CMP * sizeof(F);
    cuuint64_t tr_bytes = (cuuint64_t)a.in_stride * CMP * sizeof(F);
    if (a.batch == 1) tr_bytes = (cuuint64_t)Cfg::N * CMP * sizeof(F);
    if (tr_bytes % 16 != 0 || row_bytes % 16 != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)(Cfg::N / Cfg::R) * CMP, (cuuint64_t)Cfg::R, (cuuint64_t)a.batch};
    const cuuint64_t strides[2] = {row_bytes, tr_bytes};
    const cuuint32_t box[3] = {(cuuint32_t)(Cfg::UPC * CMP), (cuuint32_t)Cfg::RB, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const void* bases[2] = {a.in0, IL2 == kSoA ? a.in1 : nullptr};
    CUtensorMap* maps[2] = {&m.m0, &m.m1};
    for (int i = 0; i < (IL2 == kSoA ? 2 : 1); ++i) {
        if (reinterpret_cast<uintptr_t>(bases[i]) % 16 != 0) return false;
        if (enc(maps[i], dt, 3, const_cast<void*>(bases[i]), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

// One transform's input map for a gathered first pass of geometry (R, UPC, RB):
// the box of encode_pass_maps for AoS input, over a batch of one at `base`.
inline bool encode_first_map_one(CUtensorMap* m, const void* base, bool f64, int N, int R, int UPC, int RB) {
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc || reinterpret_cast<uintptr_t>(base) % 16 != 0) return false;
    const size_t es = f64 ? 8 : 4;
    const cuuint64_t row_bytes = (cuuint64_t)(N / R) * 2 * es;
    const cuuint64_t tr_bytes = (cuuint64_t)N * 2 * es;
    const cuuint64_t dims[3] = {(cuuint64_t)(N / R) * 2, (cuuint64_t)R, 1};
    const cuuint64_t strides[2] = {row_bytes, tr_bytes};
    const cuuint32_t box[3] = {(cuuint32_t)(UPC * 2), (cuuint32_t)RB, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base),
               dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Maps of the split-fused last pass (AoS scratch input): m0 boxes the item's
// HALF low units, m1 the window of HALF + 2 units that holds their mirrors.
template <typename F, int P, int PI, int S = 0>
bool encode_split_maps(const PassArgs& a, PassMaps& m) {
    using Cfg = PassCfg<F, P, PI, S>;
    if (!Cfg::kTMA_SPLIT) return false;
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc || reinterpret_cast<uintptr_t>(a.in0) % 16 != 0) return false;
    const CUtensorMapDataType dt = sizeof(F) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t row_bytes = (cuuint64_t)(Cfg::N / Cfg::R) * 2 * sizeof(F);
    cuuint64_t tr_bytes = (cuuint64_t)a.in_stride * 2 * sizeof(F);
    if (a.batch == 1) tr_bytes = (cuuint64_t)Cfg::N * 2 * sizeof(F);
    if (tr_bytes % 16 != 0 || row_bytes % 16 != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)(Cfg::N / Cfg::R) * 2, (cuuint64_t)Cfg::R, (cuuint64_t)a.batch};
    const cuuint64_t strides[2] = {row_bytes, tr_bytes};
    const cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t box_lo[3] = {(cuuint32_t)(Cfg::HALF * 2), (cuuint32_t)Cfg::RB, 1};
    const cuuint32_t box_win[3] = {(cuuint32_t)(Cfg::WIN * 2), (cuuint32_t)Cfg::RB, 1};
    void* base = const_cast<void*>(a.in0);
    return enc(&m.m0, dt, 3, base, dims, strides, box_lo, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
           enc(&m.m1, dt, 3, base, dims, strides, box_win, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename F, int P, int PI, bool FWD, int IL, int OL, int SPLIT = 0, bool FAST = false, int S = 0>
cudaError_t launch_pass(const PassArgs& a_in, cudaStream_t stream, const LaunchCtx& ctx) {
    using Cfg = PassCfg<F, P, PI, S>;
    auto kern = pass_kernel<F, P, PI, FWD, IL, OL, SPLIT, FAST, S>;
    constexpr int IL2 = Cfg::FIRST ? IL : (int)kAoS;
    PassArgs a = a_in;
    PassMaps maps;
    memset(&maps, 0, sizeof(maps));
    // ZLFFT_PASS_TMA=0 selects direct loads (diagnostics and comparison).
    static const bool tma_enabled = [] {
        const char* e = getenv("ZLFFT_PASS_TMA");
        return !(e && e[0] == '0');
    }();
    // (the split-fused last pass reads mirror-paired units directly)
    if constexpr (SPLIT != 0) {  // split-fused last pass: a low box and a mirror window per item
        a.tma = (tma_enabled && a.tma && encode_split_maps<F, P, PI, S>(a, maps)) ? 1 : 0;
    } else if (Cfg::FIRST && a.gin0) {  // gathered: per-transform maps made with the batch (PassArgs::gmaps)
        a.tma = (tma_enabled && a.tma && a.gmaps && Cfg::kTMA && IL2 == kAoS) ? 1 : 0;
    } else {
        a.tma = (tma_enabled && a.tma && encode_pass_maps<F, P, PI, IL2, S>(a, maps)) ? 1 : 0;
    }
    // a.tma_out on entry: the plan asks for tensor stores of the first pass's output
    const bool want_store = a.tma_out != 0;
    a.tma_out = 0;
    if constexpr (Cfg::kStoreTMA) {
        // first pass into dense scratch: rows of R points, one per unit of every transform
        PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
        if (want_store && tma_enabled && enc && a.out_stride == Cfg::N &&
            reinterpret_cast<uintptr_t>(a.out0) % 1024 == 0) {
            const CUtensorMapDataType dt =
                sizeof(F) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
            const cuuint64_t dims[2] = {(cuuint64_t)Cfg::R * 2, (cuuint64_t)a.batch * Cfg::UNITS};
            const cuuint64_t strides[1] = {(cuuint64_t)Cfg::R * 2 * sizeof(F)};
            const cuuint32_t box[2] = {(cuuint32_t)(Cfg::CPB * 2), (cuuint32_t)Cfg::UPC};
            const cuuint32_t estr[2] = {1, 1};
            if (enc(&maps.mo, dt, 2, a.out0, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
                a.tma_out = 1;
        }
    }
    static ResidentSlots slots;
    constexpr size_t kSmem = SPLIT != 0 ? Cfg::SMEM_SPLIT : Cfg::SMEM;
    const int blocks_per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, Cfg::THREADS, kSmem); });
    if (a.batch <= 0) return cudaSuccess;
    const long long items = a.batch * Cfg::CPT;
    const long long cap = (long long)ctx.num_sms * blocks_per_sm;
    const unsigned grid = (unsigned)(items < cap ? items : cap);
    kern<<<grid, Cfg::THREADS, kSmem, stream>>>(a, maps);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

template <typename F, int P, int PI, int S = 0>
void fill_pass_one(PassTable& t) {
    constexpr int np = pass_count(P, S);
    constexpr bool first = PI == 0, last = PI + 1 == np;
    for (int f = 0; f < 2; ++f)
        for (int il = 0; il < 2; ++il)
            for (int ol = 0; ol < 2; ++ol) t.fn[P - kPassMinP][PI][f][il][ol] = nullptr;
    // direction only matters on the first (load swap) and last (store swap) pass
    auto& e = t.fn[P - kPassMinP][PI];
    if constexpr (first) {
        e[1][kAoS][kAoS] = launch_pass<F, P, PI, true, kAoS, kAoS, 0, false, S>;
        e[1][kSoA][kAoS] = launch_pass<F, P, PI, true, kSoA, kAoS, 0, false, S>;
        e[0][kAoS][kAoS] = launch_pass<F, P, PI, false, kAoS, kAoS, 0, false, S>;
        e[0][kSoA][kAoS] = launch_pass<F, P, PI, false, kSoA, kAoS, 0, false, S>;
        e[1][kAoS][kSoA] = e[1][kAoS][kAoS];
        e[1][kSoA][kSoA] = e[1][kSoA][kAoS];
        e[0][kAoS][kSoA] = e[0][kAoS][kAoS];
        e[0][kSoA][kSoA] = e[0][kSoA][kAoS];
    } else if constexpr (last) {
        e[1][kAoS][kAoS] = launch_pass<F, P, PI, true, kAoS, kAoS, 0, false, S>;
        e[1][kAoS][kSoA] = launch_pass<F, P, PI, true, kAoS, kSoA, 0, false, S>;
        e[0][kAoS][kAoS] = launch_pass<F, P, PI, false, kAoS, kAoS, 0, false, S>;
        e[0][kAoS][kSoA] = launch_pass<F, P, PI, false, kAoS, kSoA, 0, false, S>;
        e[1][kSoA][kAoS] = e[1][kAoS][kAoS];
        e[1][kSoA][kSoA] = e[1][kAoS][kSoA];
        e[0][kSoA][kAoS] = e[0][kAoS][kAoS];
        e[0][kSoA][kSoA] = e[0][kAoS][kSoA];
    } else {
        for (int f = 0; f < 2; ++f)
            for (int il = 0; il < 2; ++il)
                for (int ol = 0; ol < 2; ++ol) e[f][il][ol] = launch_pass<F, P, PI, true, kAoS, kAoS, 0, false, S>;
    }
}

template <typename F, int P, int S = 0>
void fill_pass_order(PassTable& t) {
    {
        using C0 = PassCfg<F, P, 0, S>;
        int* g = t.first_geom[P - kPassMinP];
        g[0] = C0::R;
        g[1] = C0::UPC;
        g[2] = C0::RB;
        g[3] = C0::kTMA ? 1 : 0;
    }
    fill_pass_one<F, P, 0, S>(t);
    fill_pass_one<F, P, 1, S>(t);
    if constexpr (pass_count(P, S) > 2) fill_pass_one<F, P, 2, S>(t);
    else
        for (int f = 0; f < 2; ++f)
            for (int il = 0; il < 2; ++il)
                for (int ol = 0; ol < 2; ++ol) t.fn[P - kPassMinP][2][f][il][ol] = nullptr;
    // fast-twiddle form (AoS): the direction only matters on the first and last pass
    constexpr int NP = pass_count(P, S);
    [&]<int... PIs>(std::integer_sequence<int, PIs...>) {
        (
            [&] {
                auto& fe = t.fast[P - kPassMinP][PIs];
                if constexpr (PIs == 0 || PIs + 1 == NP) {
                    fe[1] = launch_pass<F, P, PIs, true, kAoS, kAoS, 0, true, S>;
                    fe[0] = launch_pass<F, P, PIs, false, kAoS, kAoS, 0, true, S>;
                } else {
                    fe[0] = fe[1] = launch_pass<F, P, PIs, true, kAoS, kAoS, 0, true, S>;
                }
            }(),
            ...);
    }(std::make_integer_sequence<int, NP>{});
    // last pass with the RFFT split fused: [forward | sqr_mag][output layout]
    // (scheme 0: its last pass has 128-byte unit rows, which the split's mirror pairs need)
    auto& sp = t.split[P - kPassMinP];
    if constexpr (S == 0) {
        constexpr int PL = pass_count(P) - 1;
        sp[0][kAoS] = launch_pass<F, P, PL, true, kAoS, kAoS, kR2CFwd>;
        sp[0][kSoA] = launch_pass<F, P, PL, true, kAoS, kSoA, kR2CFwd>;
        sp[1][kAoS] = sp[1][kSoA] = launch_pass<F, P, PL, true, kAoS, kAoS, kR2CSqrMag>;
    } else {
        sp[0][kAoS] = sp[0][kSoA] = sp[1][kAoS] = sp[1][kSoA] = nullptr;
    }
}

template <typename F, int... Ps>
void fill_pass_orders(PassTable& t, std::integer_sequence<int, Ps...>) {
    (fill_pass_order<F, kPassMinP + Ps>(t), ...);
}

// ranges split over translation units for parallel builds
void fill_pass_f32_a(PassTable& t);  // orders 14..18
void fill_pass_f32_b(PassTable& t);  // orders 19..24
void fill_pass_f32_c(PassTable& t);  // orders 25..26
void fill_pass_f64_a(PassTable& t);
void fill_pass_f64_b(PassTable& t);
void fill_pass_f64_c(PassTable& t);
// scheme 1 (two passes for orders 19-20), entries at the same order index
void fill_pass_split_f32(PassTable& t);
void fill_pass_split_f64(PassTable& t);

template <typename F, int Lo, int Hi, int... Ps>
void fill_pass_range_impl(PassTable& t, std::integer_sequence<int, Ps...>) {
    (fill_pass_order<F, Lo + Ps>(t), ...);
}
template <typename F, int Lo, int Hi>
void fill_pass_range(PassTable& t) {
    fill_pass_range_impl<F, Lo, Hi>(t, std::make_integer_sequence<int, Hi - Lo + 1>{});
}


// ------------------------------------------------------------------ tensor-core passes
// [order - kPassMinP][pass][fwd]: the split-precision kernel for the 256-point
// passes of FP32 complex AoS data (null where a pass is not 256 points).
struct TcPassTable {
    PassLaunchFn fn[kPassMaxP - kPassMinP + 1][kMaxPasses][2];
    PassLaunchFn pipe[kPassMaxP - kPassMinP + 1][kMaxPasses][2];  // the pipelined kernel (zlfft_tc_pipe.cuh)
    int l_in[kPassMaxP - kPassMinP + 1][kMaxPasses];  // sub-length at the pass's entry
};

template <int P, int PI, bool FWD>
cudaError_t launch_tc_pass(const PassArgs& a_in, cudaStream_t stream, const LaunchCtx& ctx) {
    using Cfg = TcPassCfg<P, PI>;
    auto kern = tc_pass_kernel<P, PI, FWD>;
    PassArgs a = a_in;
    PassMaps maps;
    memset(&maps, 0, sizeof(maps));
    static const bool tma_enabled = [] {
        const char* e = getenv("ZLFFT_PASS_TMA");
        return !(e && e[0] == '0');
    }();
    a.tma = (tma_enabled && a.tma && !(Cfg::FIRST && a.gin0) && encode_pass_maps<float, P, PI, kAoS>(a, maps)) ? 1
                                                                                                                 : 0;
    // Resident CTAs per SM from the kernel's own resources: registers and
    // shared memory per CTA (1 KB of it reserved by the driver), with the
    // shared-memory carve-out at its maximum. (The occupancy query answers 1
    // for this kernel, which would leave two thirds of each SM idle.)
    static ResidentSlots slots;
    const int blocks_per_sm = resident_ctas(slots, [kern] {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncAttributes fa{};
        int dev = 0, regs_sm = 65536, smem_sm = 228 * 1024;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        int b = 1;
        if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess && fa.numRegs > 0) {
            const int by_regs = regs_sm / (fa.numRegs * Cfg::THREADS);
            const int by_smem = smem_sm / (int)(Cfg::SMEM + 1024);
            b = by_regs < by_smem ? by_regs : by_smem;
            if (b < 1) b = 1;
        }
        return b;
    });
    if (a.batch <= 0) return cudaSuccess;
    const long long items = a.batch * Cfg::CPT;
    const long long cap = (long long)ctx.num_sms * blocks_per_sm;
    const unsigned grid = (unsigned)(items < cap ? items : cap);
    kern<<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(a, maps);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

// The pipelined tensor-core pass: one CTA per SM, items streamed through it.
template <int P, int PI, bool FWD>
cudaError_t launch_tc_pipe(const PassArgs& a_in, cudaStream_t stream, const LaunchCtx& ctx) {
    using Cfg = TcPipeCfg<P, PI>;
    auto kern = tc_pipe_kernel<P, PI, FWD>;
    PassArgs a = a_in;
    PassMaps maps;
    memset(&maps, 0, sizeof(maps));
    static const bool tma_enabled = [] {
        const char* e = getenv("ZLFFT_PASS_TMA");
        return !(e && e[0] == '0');
    }();
    a.tma = (tma_enabled && a.tma && !(Cfg::FIRST && a.gin0) && encode_pass_maps<float, P, PI, kAoS>(a, maps)) ? 1
                                                                                                                 : 0;
    static ResidentSlots slots;
    (void)resident_ctas(slots, [kern] {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM);
        return 1;
    });
    if (a.batch <= 0) return cudaSuccess;
    const long long items = a.batch * Cfg::CPT;
    const unsigned grid = (unsigned)(items < ctx.num_sms ? items : ctx.num_sms);
    kern<<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(a, maps);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

template <int P, int PI>
void fill_tc_pass_one(TcPassTable& t) {
    t.l_in[P - kPassMinP][PI] = PassCfg<float, P, PI>::L_IN;
    if constexpr (pass_radix(P, PI) == 256 && PassCfg<float, P, PI>::UPC == 16) {
        t.fn[P - kPassMinP][PI][1] = launch_tc_pass<P, PI, true>;
        t.fn[P - kPassMinP][PI][0] = launch_tc_pass<P, PI, false>;
        t.pipe[P - kPassMinP][PI][1] = launch_tc_pipe<P, PI, true>;
        t.pipe[P - kPassMinP][PI][0] = launch_tc_pipe<P, PI, false>;
    } else {
        t.fn[P - kPassMinP][PI][0] = t.fn[P - kPassMinP][PI][1] = nullptr;
        t.pipe[P - kPassMinP][PI][0] = t.pipe[P - kPassMinP][PI][1] = nullptr;
    }
}

template <int P>
void fill_tc_pass_order(TcPassTable& t) {
    fill_tc_pass_one<P, 0>(t);
    fill_tc_pass_one<P, 1>(t);
    if constexpr (pass_count(P) > 2) fill_tc_pass_one<P, 2>(t);
}

template <int Lo, int... Ps>
void fill_tc_pass_range_impl(TcPassTable& t, std::integer_sequence<int, Ps...>) {
    (fill_tc_pass_order<Lo + Ps>(t), ...);
}
void fill_tc_pass_a(TcPassTable& t);  // orders 14..18
void fill_tc_pass_b(TcPassTable& t);  // orders 19..24
void fill_tc_pass_c(TcPassTable& t);  // orders 25..26

// Each translation unit fills its part of a precision's table.
void fill_tile_c2c_f32(TileTable& t);
void fill_tile_r2c_f32(TileTable& t);
void fill_tile_c2c_f64(TileTable& t);
void fill_tile_r2c_f64(TileTable& t);

template <typename F, int P>
void fill_tile_c2c_order(TileTable& t) {
    t.fn[P][kC2CFwd][kAoS][kAoS] = launch_tile<F, P, kC2CFwd, kAoS, kAoS>;
    t.fn[P][kC2CFwd][kAoS][kSoA] = launch_tile<F, P, kC2CFwd, kAoS, kSoA>;
    t.fn[P][kC2CFwd][kSoA][kAoS] = launch_tile<F, P, kC2CFwd, kSoA, kAoS>;
    t.fn[P][kC2CFwd][kSoA][kSoA] = launch_tile<F, P, kC2CFwd, kSoA, kSoA>;
    t.fn[P][kC2CBwd][kAoS][kAoS] = launch_tile<F, P, kC2CBwd, kAoS, kAoS>;
    t.fn[P][kC2CBwd][kAoS][kSoA] = launch_tile<F, P, kC2CBwd, kAoS, kSoA>;
    t.fn[P][kC2CBwd][kSoA][kAoS] = launch_tile<F, P, kC2CBwd, kSoA, kAoS>;
    t.fn[P][kC2CBwd][kSoA][kSoA] = launch_tile<F, P, kC2CBwd, kSoA, kSoA>;
    if constexpr (P >= 11) {
        t.fast[P][kC2CFwd][kAoS] = launch_tile<F, P, kC2CFwd, kAoS, kAoS, false, true>;
        t.fast[P][kC2CBwd][kAoS] = launch_tile<F, P, kC2CBwd, kAoS, kAoS, false, true>;
    }
}

// R2C/C2R: P is the inner CFFT order (real length 2^(P+1)). The real side has
// no layout; both layout slots of that side point at the same kernel.
template <typename F, int P>
void fill_tile_r2c_order(TileTable& t) {
    for (int il = 0; il < 2; ++il) {
        t.fn[P][kR2CFwd][il][kAoS] = launch_tile<F, P, kR2CFwd, kAoS, kAoS>;
        t.fn[P][kR2CFwd][il][kSoA] = launch_tile<F, P, kR2CFwd, kAoS, kSoA>;
        for (int ol = 0; ol < 2; ++ol) t.fn[P][kR2CSqrMag][il][ol] = launch_tile<F, P, kR2CSqrMag, kAoS, kAoS>;
    }
    for (int ol = 0; ol < 2; ++ol) {
        t.fn[P][kC2RBwd][kAoS][ol] = launch_tile<F, P, kC2RBwd, kAoS, kAoS>;
        t.fn[P][kC2RBwd][kSoA][ol] = launch_tile<F, P, kC2RBwd, kSoA, kAoS>;
    }
    t.stft[P][0][kAoS] = launch_tile<F, P, kR2CFwd, kAoS, kAoS, true>;
    t.stft[P][0][kSoA] = launch_tile<F, P, kR2CFwd, kAoS, kSoA, true>;
    t.stft[P][1][kAoS] = t.stft[P][1][kSoA] = launch_tile<F, P, kR2CSqrMag, kAoS, kAoS, true>;
    if constexpr (P >= 11) {
        t.fast[P][kR2CFwd][kAoS] = launch_tile<F, P, kR2CFwd, kAoS, kAoS, false, true>;
        t.fast[P][kR2CFwd][kSoA] = launch_tile<F, P, kR2CFwd, kAoS, kSoA, false, true>;
        t.fast[P][kR2CSqrMag][kAoS] = t.fast[P][kR2CSqrMag][kSoA] = launch_tile<F, P, kR2CSqrMag, kAoS, kAoS, false, true>;
    }
}

template <typename F, int... Ps>
void fill_c2c_orders(TileTable& t, std::integer_sequence<int, Ps...>) {
    (fill_tile_c2c_order<F, Ps>(t), ...);
}
template <typename F, int... Ps>
void fill_r2c_orders(TileTable& t, std::integer_sequence<int, Ps...>) {
    (fill_tile_r2c_order<F, Ps>(t), ...);
}

}  // namespace zlfft
