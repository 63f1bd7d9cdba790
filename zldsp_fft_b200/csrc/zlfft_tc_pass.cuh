// G6: tensor-core split-precision form of the 256-point multi-pass passes.
//
// A pass with R = 256 (two radix-16 groups, see zlfft_pass.cuh) computes, per
// unit U = J * L_in + k, a 256-point DIT FFT over the positions
// pos = 0..255 (element U + pos * N / 256), as two radix-16 stages:
//   stage A  butterfly j < 16:  w[16 j + q] = sum_m W_16^{mq} W_{16 L_in}^{m k} x[j + 16 m]
//   stage B  butterfly b < 16:  z[b + 16 q] = sum_m W_16^{mq} W_{256 L_in}^{m (k + L_in b)} w[b + 16 m]
// and writes z[pos] to J * L_out + k + pos * L_in (the same positions as the
// plain pass; the mixed-radix DIT identity makes both compute the same DFT, with
// different rounding). Each stage is one dense product on the tensor cores
// (zlfft_tc.cuh): 16 units x 16 butterflies = 256 rows, two 128-row MMA blocks,
// D in tensor memory. The twiddles are applied in FP32 on the CUDA cores
// before each stage, so the MMAs only ever multiply by the DFT-16 matrix.
//
// Range: before the hi/lo split every value is scaled by an exact power of two
// so that the largest magnitude of its group lies in [0.5, 1): per A row in
// stage A (the building thread holds the whole row), per unit in stage B (the
// 16 writers of a unit's rows form a half-warp and agree on the exponent by
// shuffles); the epilogues multiply the exponents back out, exactly. FP16 then
// never overflows, and the FP16 low parts keep ~22 significant bits for the
// values that carry the norm.
//
// Shared-memory traffic per element: the staging read, one 16-byte-vector write
// of the stage-A operand, one 4-byte write per half of the stage-B operand, a
// twiddle read and the global store; the operand reads of both stages are done
// by the tensor core, not by the load/store pipe. Row orders are chosen so every
// operand write is bank-conflict-free (see the index functions below).
#pragma once

#include "zlfft_pass.cuh"
#include "zlfft_tc.cuh"

namespace zlfft {

// W_N^t for any t (mod N), from the unified table T[t] = W_N^t, t < 3N/4.
__device__ __forceinline__ float2 tw_any(const float2* T, uint32_t t, uint32_t n) {
    t &= n - 1;
    if (t < 3 * (n >> 2)) return T[t];
    const float2 w = T[n - t];
    return make_float2(w.x, -w.y);
}

// Exponent e such that m * 2^-e lies in [0.5, 1) (clamped; 0 maps to -100).
__device__ __forceinline__ int tc_scale_exp(float m) {
    const int e = ((__float_as_int(m) >> 23) & 255) - 126;
    return e < -100 ? -100 : (e > 100 ? 100 : e);
}
__device__ __forceinline__ float tc_pow2(int e) { return __int_as_float((127 + e) << 23); }

__device__ __forceinline__ float2 tc_scale(float2 v, float s) { return make_float2(v.x * s, v.y * s); }

// Per-pass twiddles of a tensor-core pass with L_in > 1 (PassArgs::tctw), the
// values of the unified table laid out for coalesced vector loads:
//   [4 k + 0..3]          = W_{16 L_in}^{k}, ^{2k}, ^{4k}, ^{8k}  (stage A; products give ^{mk})
//   [4 L_in + 16 k + j]   = W_{256 L_in}^{j k}                     (stage B; times W_256^{jq})

template <int P, int PI>
struct TcPassCfg {
    using Base = PassCfg<float, P, PI>;
    static constexpr int N = Base::N, R = Base::R, UPC = Base::UPC;
    static constexpr int L_IN = Base::L_IN, L_OUT = Base::L_OUT, CPT = Base::CPT;
    static constexpr bool FIRST = Base::FIRST, LAST = Base::LAST;
    static_assert(R == 256 && UPC == 16, "tensor-core passes are 256-point passes of 16 units");
    static constexpr int THREADS = 256;
    static constexpr size_t STAGE_OFF = 0;
    static constexpr size_t STAGE_BYTES = (size_t)R * UPC * sizeof(float2);  // 32 KB, TMA box [pos][unit]
    static constexpr size_t A_OFF = STAGE_OFF + STAGE_BYTES;                 // 256 rows x 128 bytes
    static constexpr size_t B_OFF = A_OFF + 256 * 128;                        // 32 rows x 128 bytes
    static constexpr size_t MISC_OFF = B_OFF + 32 * 128;
    // barriers (2 x 8 B), TMEM slot, 16 DFT-16 twiddles, 256 + 16 exponents,
    // then the 256 stage-B twiddles W_256^{jq} stored [q][j]
    static constexpr size_t TW256_OFF = MISC_OFF + 16 + 16 + 16 * 8 + 272 * 4;
    static constexpr size_t SMEM = TW256_OFF + 256 * 8 + 1024;  // + alignment slack
    // first pass: stage-B rows unit-major so each unit's 256 outputs leave as
    // contiguous 128-byte runs; later passes: butterfly-major (consecutive
    // units are consecutive output positions)
    static constexpr bool kUnitMajorB = (L_IN == 1);
};

// Row of the stage-A operand that holds butterfly j of unit u. Stage-A
// epilogue warp w owns units u1 = (w & 3) + 8 (w >> 2) and u1 + 4 (lanes
// 0-15 and 16-31, butterflies permuted by j ^ (u & 7)): its stage-B operand
// writes then cover all 32 banks, and the building threads (16 consecutive
// units per row group) write 8 distinct swizzle rows per quarter-warp.
__device__ __forceinline__ int tc_rowA(int u, int j) {
    return 32 * ((u & 3) + 4 * (u >> 3)) + 16 * ((u >> 2) & 1) + (j ^ (u & 7));
}

template <int P, int PI, bool FWD>
__global__ void __launch_bounds__(256, 3) tc_pass_kernel(const PassArgs a, const __grid_constant__ PassMaps maps) {
    using Cfg = TcPassCfg<P, PI>;
    using C = float2;
    constexpr int N = Cfg::N, R = Cfg::R, UPC = Cfg::UPC, L_IN = Cfg::L_IN, L_OUT = Cfg::L_OUT, CPT = Cfg::CPT;
    constexpr bool UMAJ = Cfg::kUnitMajorB;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    // first 1024-byte boundary, as an offset into the shared array (keeps the
    // pointer in the shared address space for the compiler)
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    C* stage = reinterpret_cast<C*>(smem + Cfg::STAGE_OFF);
    unsigned char* a_tile = smem + Cfg::A_OFF;
    unsigned char* b_tile = smem + Cfg::B_OFF;
    uint64_t* tma_bar = reinterpret_cast<uint64_t*>(smem + Cfg::MISC_OFF);
    uint64_t* mma_bar = tma_bar + 1;
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + Cfg::MISC_OFF + 16);
    C* tw16 = reinterpret_cast<C*>(smem + Cfg::MISC_OFF + 32);
    int* expA = reinterpret_cast<int*>(smem + Cfg::MISC_OFF + 32 + 16 * 8);
    int* expB = expA + 256;
    C* tw256 = reinterpret_cast<C*>(smem + Cfg::TW256_OFF);

    const int t = (int)threadIdx.x, warp = t >> 5, lane = t & 31;
    const C* T = static_cast<const C*>(a.tw);
    const long long items = a.batch * CPT;

    // ---- set-up: tensor memory (64 columns: two 128 x 32 accumulators), barriers, DFT-16 operand
    if (warp == 0) {
        tc::tmem_alloc(slot, 64);
        tc::tmem_relinquish();
    }
    if (t == 0) {
        mbar_init(tma_bar, 1);
        mbar_init(mma_bar, 1);
        fence_mbar_init();
    }
    if (t < 16) tw16[t] = tw_any(T, (uint32_t)t * (N / 16), N);
    tw256[t] = tw_any(T, (uint32_t)((t & 15) * (t >> 4)) * (N / 256), N);  // [q = t >> 4][j = t & 15]
    __syncthreads();
    tc::build_dft16_b(b_tile, tw16);

    // identities of this thread in the three phases
    const int bu = t & 15, bj = t >> 4;  // building thread: unit, butterfly (stage A)
    const int rowA = tc_rowA(bu, bj);
    const int eA_s = (lane >> 4) & 1;  // stage-A epilogue: row t
    const int eA_u = (warp & 3) + 8 * (warp >> 2) + 4 * eA_s;
    const int eA_j = (lane & 15) ^ (eA_u & 7);
    const int eB_u = UMAJ ? (t >> 4) : (t & 15);  // stage-B epilogue: row t
    const int eB_b = UMAJ ? (t & 15) : (t >> 4);

    fence_proxy_async_smem();  // the DFT-16 operand, written by generic stores, is read by the tensor core
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t a_addr = smem_u32(a_tile), b_addr = smem_u32(b_tile);
    const uint32_t t_row = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(32 * (warp >> 2));

    const bool use_tma = a.tma != 0;
    auto issue = [&](long long it) {  // one box of UPC units x 256 positions per item
        if (!use_tma || t != 0 || it >= items) return;
        const int z = (int)(it / CPT);
        const int x = (int)(it % CPT) * UPC * 2;  // x * 4 bytes: a multiple of 128
        mbar_arrive_expect_tx(tma_bar, (uint32_t)Cfg::STAGE_BYTES);
        tma_load_3d(stage, &maps.m0, x, 0, z, tma_bar);
    };
    if (use_tma) issue(blockIdx.x);
    uint32_t tma_phase = 0, mma_phase = 0;
    bool failed = false;

    for (long long item = blockIdx.x; item < items; item += gridDim.x) {
        const long long tr = item / CPT;
        const int ublk = (int)(item % CPT) * UPC;

        // ------------------------------------------------ stage A operand
        {
            const int U = ublk + bu;
            const int ku = U % L_IN;
            C v[16];
            if (use_tma) {
                const bool ok = mbar_wait(tma_bar, tma_phase);
                if (__syncthreads_or(!ok)) {
                    failed = true;
                    break;
                }
                tma_phase ^= 1u;
#pragma unroll
                for (int m = 0; m < 16; ++m) v[m] = stage[(bj + 16 * m) * UPC + bu];
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
            if constexpr (L_IN > 1) {  // W_{16 L_in}^{m k} = product of W^{k}, W^{2k}, W^{4k}, W^{8k} over m's bits
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
            expA[rowA] = e;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const tc::HL2 p0 = tc::split_pair(tc_scale(v[4 * c], sc), tc_scale(v[4 * c + 1], sc));
                const tc::HL2 p1 = tc::split_pair(tc_scale(v[4 * c + 2], sc), tc_scale(v[4 * c + 3], sc));
                *reinterpret_cast<uint4*>(a_tile + tc::sw128_off((uint32_t)rowA, (uint32_t)c)) =
                    make_uint4(p0.hi.x, p0.hi.y, p1.hi.x, p1.hi.y);
                *reinterpret_cast<uint4*>(a_tile + tc::sw128_off((uint32_t)rowA, (uint32_t)(4 + c))) =
                    make_uint4(p0.lo.x, p0.lo.y, p1.lo.x, p1.lo.y);
            }
        }
        fence_proxy_async_smem();  // staging reads and operand writes before the async proxy uses them
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) {
            issue(item + gridDim.x);  // the staging buffer is free: prefetch the next item
            tc::issue_split_dft16(tmem, a_addr, b_addr);
            tc::issue_split_dft16(tmem + 32, a_addr + 128 * 128, b_addr);
            tc::mma_commit(mma_bar);
        }
        {
            const bool ok = mbar_wait(mma_bar, mma_phase);
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            mma_phase ^= 1u;
        }
        tc::fence_after_sync();

        // ------------------------------------------------ stage A epilogue -> stage B operand
        {
            float d[32];
            tc::tmem_ld32(t_row, d);
            const float un = tc_pow2(expA[t]);
            C y[16];
            if constexpr (L_IN > 1) {
                const int ku = (ublk + eA_u) % L_IN;
                const C wb = __ldg(static_cast<const C*>(a.tctw) + 4 * L_IN + 16 * ku + eA_j);
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    y[q] = cmul_tw(make_float2(d[2 * q] * un, d[2 * q + 1] * un), cmul_tw(tw256[q * 16 + eA_j], wb));
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
            if ((lane & 15) == 0) expB[eA_u] = e;
            const uint32_t jc = (uint32_t)(eA_j >> 2), jo = (uint32_t)(eA_j & 3) * 4u;
            // output q goes to row (unit, butterfly q), column j; in the unit-major
            // order the half-warp of unit u1 + 4 writes q ^ 4 in the same step, so
            // that the two halves land in opposite halves of the swizzled row
            auto put = [&](int q, const C yq) {
                const uint32_t rB = UMAJ ? (uint32_t)(16 * eA_u + q) : (uint32_t)(16 * q + eA_u);
                __half hr, lr, hi_, li_;
                tc::split_hl(yq.x * sc, hr, lr);
                tc::split_hl(yq.y * sc, hi_, li_);
                *reinterpret_cast<uint32_t*>(a_tile + tc::sw128_off(rB, jc) + jo) =
                    (uint32_t)__half_as_ushort(hr) | ((uint32_t)__half_as_ushort(hi_) << 16);
                *reinterpret_cast<uint32_t*>(a_tile + tc::sw128_off(rB, 4u + jc) + jo) =
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
        fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) {
            tc::issue_split_dft16(tmem, a_addr, b_addr);
            tc::issue_split_dft16(tmem + 32, a_addr + 128 * 128, b_addr);
            tc::mma_commit(mma_bar);
        }
        {
            const bool ok = mbar_wait(mma_bar, mma_phase);
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            mma_phase ^= 1u;
        }
        tc::fence_after_sync();

        // ------------------------------------------------ stage B epilogue -> pass output
        {
            float d[32];
            tc::tmem_ld32(t_row, d);
            const float un = tc_pow2(expB[eB_u]);
            const int U = ublk + eB_u;
            const int ku = U % L_IN, J = U / L_IN;
            C* dst = (Cfg::LAST && a.gout0) ? static_cast<C*>(a.gout0[tr]) : static_cast<C*>(a.out0) + tr * a.out_stride;
            dst += (long long)J * L_OUT + ku;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                C z = make_float2(d[2 * q] * un, d[2 * q + 1] * un);
                if constexpr (Cfg::LAST && !FWD) z = cswap(z);
                __stcs(dst + (long long)(eB_b + 16 * q) * L_IN, z);
            }
        }
        tc::fence_before_sync();  // tensor-memory reads complete before the next item's MMAs
    }

    if (failed) {  // a bounded wait ran out: report, let pending copies and MMAs land (bounded), free TMEM
        if (t == 0) atomicOr(a.err, kDevErrWaitTimeout);
        mbar_wait(tma_bar, tma_phase);
        mbar_wait(mma_bar, mma_phase);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

}  // namespace zlfft
