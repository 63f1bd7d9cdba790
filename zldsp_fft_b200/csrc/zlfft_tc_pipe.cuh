// G6, pipelined: the tensor-core split-precision 256-point pass with its
// phases in separate warps and two items in flight.
//
// Same arithmetic as tc_pass_kernel (zlfft_tc_pass.cuh): per unit, stage A
// (twiddle W_{16 L_in}^{m k}, split hi/lo, DFT-16 contraction on the tensor
// cores), stage B (twiddle W_{256 L_in}, split, contraction), with exact
// power-of-two scaling around each split. What changes is the schedule. The
// serial kernel runs load -> operand build -> MMA -> epilogue -> MMA ->
// epilogue per item with full-CTA barriers, so each phase waits on the one
// before. Here one CTA per SM runs a pipeline over its items, each phase in
// its own warps, handing buffers on through mbarriers:
//
//   warp 14        TMA loads of the items' inputs          -> staging[s]
//   warps 0-3      stage-A operand build (twiddle, scale, split) -> aop[s]
//   warp 12        stage-A MMAs (one thread)              -> tensor memory DA[s]
//   warps 4-7      stage-A epilogue: DA -> twiddle, scale, split -> bop[s]
//   warp 13        stage-B MMAs (one thread)              -> tensor memory DB[s]
//   warps 8-11     stage-B epilogue: DB -> unscale -> global memory
//
// s = item parity: every buffer has two slots, so while one item's stage-B
// epilogue stores, the next item's operands are being built and multiplied.
// Barriers per slot: full_stage (TMA bytes), empty_stage (builders read the
// staging), full_a (operand A and its row exponents written), full_da (MMA-A
// done; tcgen05.commit), empty_da (epilogue A read DA and the exponents),
// full_b (operand B and unit exponents written), full_db (MMA-B done),
// empty_db (epilogue B read DB). A producer of slot s for item k + 2 waits
// for the consumer's release of item k; in particular the builders wait for
// epilogue A (which implies MMA A) and epilogue A waits for epilogue B, so no
// barrier ever runs a phase ahead of a consumer that still has to observe it.
//
// Every wait is bounded and also gives up when another warp has given up
// (a shared abort word); the kernel then records kDevErrWaitTimeout, waits
// (bounded) for the copies and MMAs it issued, frees its tensor memory and
// returns.
#pragma once

#include "zlfft_tc_pass.cuh"

namespace zlfft {

template <int P, int PI>
struct TcPipeCfg {
    using Base = PassCfg<float, P, PI>;
    static constexpr int N = Base::N, R = Base::R, UPC = Base::UPC;
    static constexpr int L_IN = Base::L_IN, L_OUT = Base::L_OUT, CPT = Base::CPT;
    static constexpr bool FIRST = Base::FIRST, LAST = Base::LAST;
    static_assert(R == 256 && UPC == 16, "tensor-core passes are 256-point passes of 16 units");
    static constexpr int W_BUILD = 0, W_EPIA = 4, W_EPIB = 8, W_MMAA = 12, W_MMAB = 13, W_TMA = 14;
    static constexpr int THREADS = 15 * 32;
    static constexpr size_t TILE = (size_t)R * UPC * sizeof(float2);  // 32 KB: one item's points
    static constexpr size_t STAGE_OFF = 0;                            // 2 x staging
    static constexpr size_t AOP_OFF = STAGE_OFF + 2 * TILE;           // 2 x 256 rows x 128 B
    static constexpr size_t BOP_OFF = AOP_OFF + 2 * TILE;
    static constexpr size_t BDFT_OFF = BOP_OFF + 2 * TILE;            // 32 rows x 128 B
    static constexpr size_t TW256_OFF = BDFT_OFF + 32 * 128;          // 256 float2, [q][j]
    static constexpr size_t TW16_OFF = TW256_OFF + 256 * 8;           // 16 float2
    static constexpr size_t EXPA_OFF = TW16_OFF + 16 * 8;             // 2 x 256 int
    static constexpr size_t EXPB_OFF = EXPA_OFF + 2 * 256 * 4;        // 2 x 16 int
    static constexpr size_t BAR_OFF = EXPB_OFF + 2 * 16 * 4;          // 16 barriers
    static constexpr size_t MISC_OFF = BAR_OFF + 16 * 8;              // TMEM slot, abort word
    static constexpr size_t SMEM = MISC_OFF + 16 + 1024;              // + alignment slack
    static constexpr uint32_t TMEM_COLS = 256;  // DA[2] (64 columns each), DB[2]
    static constexpr bool kUnitMajorB = (L_IN == 1);
    static_assert(SMEM <= 227 * 1024, "pipelined tensor-core pass: shared memory");
};

// Bounded wait that also ends when another warp has given up.
__device__ __forceinline__ bool pipe_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255u) == 255u && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int P, int PI, bool FWD>
__global__ void __launch_bounds__(TcPipeCfg<P, PI>::THREADS, 1)
    tc_pipe_kernel(const PassArgs a, const __grid_constant__ PassMaps maps) {
    using Cfg = TcPipeCfg<P, PI>;
    using C = float2;
    constexpr int N = Cfg::N, R = Cfg::R, UPC = Cfg::UPC, L_IN = Cfg::L_IN, L_OUT = Cfg::L_OUT, CPT = Cfg::CPT;
    constexpr bool UMAJ = Cfg::kUnitMajorB;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    C* stage = reinterpret_cast<C*>(smem + Cfg::STAGE_OFF);
    unsigned char* aop = smem + Cfg::AOP_OFF;
    unsigned char* bop = smem + Cfg::BOP_OFF;
    unsigned char* bdft = smem + Cfg::BDFT_OFF;
    C* tw256 = reinterpret_cast<C*>(smem + Cfg::TW256_OFF);
    C* tw16 = reinterpret_cast<C*>(smem + Cfg::TW16_OFF);
    int* expA = reinterpret_cast<int*>(smem + Cfg::EXPA_OFF);
    int* expB = reinterpret_cast<int*>(smem + Cfg::EXPB_OFF);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::BAR_OFF);
    uint64_t* full_stage = bars + 0;
    uint64_t* empty_stage = bars + 2;
    uint64_t* full_a = bars + 4;
    uint64_t* full_da = bars + 6;
    uint64_t* empty_da = bars + 8;
    uint64_t* full_b = bars + 10;
    uint64_t* full_db = bars + 12;
    uint64_t* empty_db = bars + 14;
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + Cfg::MISC_OFF);
    volatile int* abort = reinterpret_cast<volatile int*>(smem + Cfg::MISC_OFF + 4);

    const int t = (int)threadIdx.x, warp = t >> 5, lane = t & 31;
    const C* T = static_cast<const C*>(a.tw);
    const long long items = a.batch * CPT;
    const bool use_tma = a.tma != 0;

    // ---- set-up: tensor memory, barriers, DFT-16 operand, twiddle tables
    if (warp == 0) {
        tc::tmem_alloc(slot, Cfg::TMEM_COLS);
        tc::tmem_relinquish();
    }
    if (t == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(full_stage + s, 1);
            mbar_init(empty_stage + s, 128);
            mbar_init(full_a + s, 128);
            mbar_init(full_da + s, 1);
            mbar_init(empty_da + s, 128);
            mbar_init(full_b + s, 128);
            mbar_init(full_db + s, 1);
            mbar_init(empty_db + s, 128);
        }
        *abort = 0;
        fence_mbar_init();
    }
    if (t < 16) tw16[t] = tw_any(T, (uint32_t)t * (N / 16), N);
    if (t < 256) tw256[t] = tw_any(T, (uint32_t)((t & 15) * (t >> 4)) * (N / 256), N);  // [q = t >> 4][j = t & 15]
    __syncthreads();
    tc::build_dft16_b(bdft, tw16);
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    bool failed = false;

    auto give_up = [&]() {
        failed = true;
        *abort = 1;
    };
    // waits of the epilogue warps, whose tensor-memory loads are warp-collective:
    // the whole warp goes on, or the whole warp gives up
    auto warp_wait = [&](uint64_t* bar, uint32_t parity) {
        return __all_sync(0xffffffffu, pipe_wait(bar, parity, abort)) != 0;
    };

    if (warp == Cfg::W_TMA) {
        // ------------------------------------------------ TMA producer
        long long k = 0;
        if (use_tma && lane == 0) {
            for (long long item = blockIdx.x; item < items; item += gridDim.x, ++k) {
                const int s = (int)(k & 1);
                const uint32_t ph = (uint32_t)((k >> 1) & 1);
                if (k >= 2 && !pipe_wait(empty_stage + s, ph ^ 1u, abort)) {
                    give_up();
                    break;
                }
                const int z = (int)(item / CPT);
                const int x = (int)(item % CPT) * UPC * 2;  // x * 4 bytes: a multiple of 128
                mbar_arrive_expect_tx(full_stage + s, (uint32_t)Cfg::TILE);
                tma_load_3d(stage + (size_t)s * (Cfg::TILE / sizeof(C)), &maps.m0, x, 0, z, full_stage + s);
            }
            // the copies this thread issued land before the CTA's shared memory goes
            if (k > 0) {
                const long long kl = k - 1;
                mbar_wait(full_stage + (int)(kl & 1), (uint32_t)((kl >> 1) & 1));
            }
        }
    } else if (warp < Cfg::W_EPIA) {
        // ------------------------------------------------ stage-A operand builders (128 threads)
        const int tb = t;  // 0..127
        long long k = 0;
        for (long long item = blockIdx.x; item < items; item += gridDim.x, ++k) {
            const int s = (int)(k & 1);
            const uint32_t ph = (uint32_t)((k >> 1) & 1);
            const long long tr = item / CPT;
            const int ublk = (int)(item % CPT) * UPC;
            if (use_tma && !pipe_wait(full_stage + s, ph, abort)) {
                give_up();
                break;
            }
            if (k >= 2 && !pipe_wait(empty_da + s, ph ^ 1u, abort)) {  // epilogue A of item k - 2 is done
                give_up();
                break;
            }
            const C* stg = stage + (size_t)s * (Cfg::TILE / sizeof(C));
            unsigned char* at = aop + (size_t)s * Cfg::TILE;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int rr = tb + 128 * h;
                const int bu = rr & 15, bj = rr >> 4;
                const int rowA = tc_rowA(bu, bj);
                const int U = ublk + bu;
                const int ku = U % L_IN;
                C v[16];
                if (use_tma) {
#pragma unroll
                    for (int m = 0; m < 16; ++m) v[m] = stg[(bj + 16 * m) * UPC + bu];
                } else {
                    const C* src = (Cfg::FIRST && a.gin0) ? static_cast<const C*>(a.gin0[tr])
                                                          : static_cast<const C*>(a.in0) + tr * a.in_stride;
#pragma unroll
                    for (int m = 0; m < 16; ++m) v[m] = __ldcs(src + U + (bj + 16 * m) * (N / R));
                }
                if constexpr (Cfg::FIRST && !FWD) {
#pragma unroll
                    for (int m = 0; m < 16; ++m) v[m] = cswap(v[m]);
                }
                if constexpr (L_IN > 1) {
                    const float4* ta = static_cast<const float4*>(a.tctw) + 2 * ku;
                    const float4 t01 = __ldg(ta), t23 = __ldg(ta + 1);
                    const C w1 = make_float2(t01.x, t01.y), w2 = make_float2(t01.z, t01.w);
                    const C w4 = make_float2(t23.x, t23.y), w8 = make_float2(t23.z, t23.w);
                    const C w3 = cmul_tw(w1, w2), w12 = cmul_tw(w4, w8);
                    const C lo4[4] = {make_float2(1.f, 0.f), w1, w2, w3};
                    const C hi4[4] = {make_float2(1.f, 0.f), w4, w8, w12};
#pragma unroll
                    for (int m = 1; m < 16; ++m) {
                        const C w = (m & 3) == 0 ? hi4[m >> 2]
                                                 : ((m >> 2) == 0 ? lo4[m & 3] : cmul_tw(lo4[m & 3], hi4[m >> 2]));
                        v[m] = cmul_tw(v[m], w);
                    }
                }
                float mx = 0.f;
#pragma unroll
                for (int m = 0; m < 16; ++m) mx = fmaxf(mx, fmaxf(fabsf(v[m].x), fabsf(v[m].y)));
                const int e = tc_scale_exp(mx);
                const float sc = tc_pow2(-e);
                expA[s * 256 + rowA] = e;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const tc::HL2 p0 = tc::split_pair(tc_scale(v[4 * c], sc), tc_scale(v[4 * c + 1], sc));
                    const tc::HL2 p1 = tc::split_pair(tc_scale(v[4 * c + 2], sc), tc_scale(v[4 * c + 3], sc));
                    *reinterpret_cast<uint4*>(at + tc::sw128_off((uint32_t)rowA, (uint32_t)c)) =
                        make_uint4(p0.hi.x, p0.hi.y, p1.hi.x, p1.hi.y);
                    *reinterpret_cast<uint4*>(at + tc::sw128_off((uint32_t)rowA, (uint32_t)(4 + c))) =
                        make_uint4(p0.lo.x, p0.lo.y, p1.lo.x, p1.lo.y);
                }
            }
            fence_proxy_async_smem();  // staging reads and operand writes, before the async proxy's use
            if (use_tma) mbar_arrive(empty_stage + s);
            mbar_arrive(full_a + s);
        }
    } else if (warp == Cfg::W_MMAA || warp == Cfg::W_MMAB) {
        // ------------------------------------------------ MMA issuers (one thread each)
        const bool stA = (warp == Cfg::W_MMAA);
        uint64_t* fullin = stA ? full_a : full_b;
        uint64_t* emptyd = stA ? empty_da : empty_db;
        uint64_t* fulld = stA ? full_da : full_db;
        const uint32_t dbase = tmem + (stA ? 0u : 128u);
        const uint32_t opbase = smem_u32(stA ? aop : bop);
        const uint32_t b_addr = smem_u32(bdft);
        long long k = 0;
        if (lane == 0) {
            for (long long item = blockIdx.x; item < items; item += gridDim.x, ++k) {
                const int s = (int)(k & 1);
                const uint32_t ph = (uint32_t)((k >> 1) & 1);
                if (!pipe_wait(fullin + s, ph, abort)) {
                    give_up();
                    break;
                }
                if (k >= 2 && !pipe_wait(emptyd + s, ph ^ 1u, abort)) {
                    give_up();
                    break;
                }
                tc::fence_after_sync();
                const uint32_t d = dbase + 64u * (uint32_t)s;
                const uint32_t op = opbase + (uint32_t)(s * Cfg::TILE);
                tc::issue_split_dft16(d, op, b_addr);
                tc::issue_split_dft16(d + 32, op + 128 * 128, b_addr);
                tc::mma_commit(fulld + s);
            }
            if (k > 0) {  // the MMAs this thread issued complete before tensor memory is freed
                const long long kl = k - 1;
                mbar_wait(fulld + (int)(kl & 1), (uint32_t)((kl >> 1) & 1));
            }
        }
    } else if (warp < Cfg::W_EPIB) {
        // ------------------------------------------------ stage-A epilogue -> stage-B operand (128 threads)
        const int r = warp - Cfg::W_EPIA;
        long long k = 0;
        for (long long item = blockIdx.x; item < items; item += gridDim.x, ++k) {
            const int s = (int)(k & 1);
            const uint32_t ph = (uint32_t)((k >> 1) & 1);
            const int ublk = (int)(item % CPT) * UPC;
            // full_a: the builders' row exponents (it cannot run a phase ahead: the
            // builders of item k + 2 wait for this epilogue's release of item k)
            if (!warp_wait(full_a + s, ph) || !warp_wait(full_da + s, ph)) {
                give_up();
                break;
            }
            if (k >= 2 && !warp_wait(empty_db + s, ph ^ 1u)) {  // epilogue B of item k - 2 is done
                give_up();
                break;
            }
            tc::fence_after_sync();
            unsigned char* bt = bop + (size_t)s * Cfg::TILE;
#pragma unroll 1
            for (int blk = 0; blk < 2; ++blk) {
                const int ow = r + 4 * blk;  // the row group of the serial kernel's warp ow
                const int eA_s = (lane >> 4) & 1;
                const int eA_u = (ow & 3) + 8 * (ow >> 2) + 4 * eA_s;
                const int eA_j = (lane & 15) ^ (eA_u & 7);
                const int row = 32 * ow + lane;
                float d[32];
                tc::tmem_ld32(tmem + 64u * (uint32_t)s + ((uint32_t)(32 * r) << 16) + (uint32_t)(32 * blk), d);
                const float un = tc_pow2(expA[s * 256 + row]);
                C y[16];
                if constexpr (L_IN > 1) {
                    const int ku = (ublk + eA_u) % L_IN;
                    const C wb = __ldg(static_cast<const C*>(a.tctw) + 4 * L_IN + 16 * ku + eA_j);
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        y[q] = cmul_tw(make_float2(d[2 * q] * un, d[2 * q + 1] * un),
                                       cmul_tw(tw256[q * 16 + eA_j], wb));
                } else {
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        y[q] = cmul_tw(make_float2(d[2 * q] * un, d[2 * q + 1] * un), tw256[q * 16 + eA_j]);
                }
                float mx = 0.f;
#pragma unroll
                for (int q = 0; q < 16; ++q) mx = fmaxf(mx, fmaxf(fabsf(y[q].x), fabsf(y[q].y)));
#pragma unroll
                for (int o = 1; o < 16; o <<= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                const int e = tc_scale_exp(mx);
                const float sc = tc_pow2(-e);
                if ((lane & 15) == 0) expB[s * 16 + eA_u] = e;
                const uint32_t jc = (uint32_t)(eA_j >> 2), jo = (uint32_t)(eA_j & 3) * 4u;
                auto put = [&](int q, const C yq) {
                    const uint32_t rB = UMAJ ? (uint32_t)(16 * eA_u + q) : (uint32_t)(16 * q + eA_u);
                    __half hr, lr, hi_, li_;
                    tc::split_hl(yq.x * sc, hr, lr);
                    tc::split_hl(yq.y * sc, hi_, li_);
                    *reinterpret_cast<uint32_t*>(bt + tc::sw128_off(rB, jc) + jo) =
                        (uint32_t)__half_as_ushort(hr) | ((uint32_t)__half_as_ushort(hi_) << 16);
                    *reinterpret_cast<uint32_t*>(bt + tc::sw128_off(rB, 4u + jc) + jo) =
                        (uint32_t)__half_as_ushort(lr) | ((uint32_t)__half_as_ushort(li_) << 16);
                };
                if (!UMAJ || eA_s == 0) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) put(i, y[i]);
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) put(i ^ 4, y[i ^ 4]);
                }
            }
            tc::fence_before_sync();  // tensor-memory reads of DA[s] complete before the release
            mbar_arrive(empty_da + s);
            fence_proxy_async_smem();  // operand writes before the async proxy reads them
            mbar_arrive(full_b + s);
        }
    } else if (warp < Cfg::W_MMAA) {
        // ------------------------------------------------ stage-B epilogue -> pass output (128 threads)
        const int r = warp - Cfg::W_EPIB;
        long long k = 0;
        for (long long item = blockIdx.x; item < items; item += gridDim.x, ++k) {
            const int s = (int)(k & 1);
            const uint32_t ph = (uint32_t)((k >> 1) & 1);
            const long long tr = item / CPT;
            const int ublk = (int)(item % CPT) * UPC;
            if (!warp_wait(full_b + s, ph) || !warp_wait(full_db + s, ph)) {
                give_up();
                break;
            }
            tc::fence_after_sync();
            C* base = (Cfg::LAST && a.gout0) ? static_cast<C*>(a.gout0[tr]) : static_cast<C*>(a.out0) + tr * a.out_stride;
#pragma unroll 1
            for (int blk = 0; blk < 2; ++blk) {
                const int row = 128 * blk + 32 * r + lane;
                const int eB_u = UMAJ ? (row >> 4) : (row & 15);
                const int eB_b = UMAJ ? (row & 15) : (row >> 4);
                float d[32];
                tc::tmem_ld32(tmem + 128u + 64u * (uint32_t)s + ((uint32_t)(32 * r) << 16) + (uint32_t)(32 * blk), d);
                const float un = tc_pow2(expB[s * 16 + eB_u]);
                const int U = ublk + eB_u;
                const int ku = U % L_IN, J = U / L_IN;
                C* dst = base + (long long)J * L_OUT + ku;
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    C z = make_float2(d[2 * q] * un, d[2 * q + 1] * un);
                    if constexpr (Cfg::LAST && !FWD) z = cswap(z);
                    __stcs(dst + (long long)(eB_b + 16 * q) * L_IN, z);
                }
            }
            tc::fence_before_sync();
            mbar_arrive(empty_db + s);
        }
    }

    if (failed && (lane == 0)) atomicOr(a.err, kDevErrWaitTimeout);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, Cfg::TMEM_COLS);
}

}  // namespace zlfft
