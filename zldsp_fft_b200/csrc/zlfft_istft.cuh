// G9: inverse STFT with overlap-add, the backward-side counterpart of the STFT
// front end. Per frame f (bins X_f, N_c + 1 of them, N_c = 2^P):
//
//     x_f = RFFT::backward(H * X_f)                      (2 N_c reals)
//     y[f hop + n] += w[n] x_f[n],   f = 0, 1, ... in order
//
// with an optional spectral filter H (N_c + 1 bins, each complex product
// rounded operation by operation) and an optional synthesis window w. The
// inverse transform is the tile kernel's backward RFFT
// (src/common/zldsp_fft_common_execute.hpp:399-451 pre-step, then the
// swap-based backward CFFT), so x_f carries the reference's bits. With H
// the identity, the spectrum of a fast convolution, or an STFT's bins, the
// launch is inverse-STFT synthesis or overlap-add convolution.
//
// Determinism: the output is cut into blocks of `hop` reals; block m takes
// frames m - K + 1 .. m (K = 2 N_c / hop). Each CTA owns a run of consecutive
// blocks and transforms its frames in ascending order into a ring of K blocks
// in shared memory, beginning K - 1 frames before its first block (those
// frames' contributions to earlier blocks are dropped). After frame f, block
// f holds its final sum, is written once, and its ring slots are cleared for
// block f + K. Every output real is thus the sum of its frames' terms in
// ascending frame order, from zero, one rounding per term, whatever the grid:
// the same value as a sequential loop over frames, with no atomics.
#pragma once

#include "zlfft_launch.cuh"

namespace zlfft {

struct IstftArgs {
    const void* filt;    // H: N_c + 1 complex bins (null: none)
    const void* win;     // w: 2 N_c reals (null: none)
    void* sig;           // y: (n_frames - 1) * hop + 2 N_c reals
    long long n_frames;
    long long hop;       // reals: even, divides 2 N_c
    long long blocks;    // output blocks of hop reals: n_frames + K - 1
    long long run;       // blocks per CTA (set by the launch)
    int k;               // K: frames that overlap one block
};

// Last-group sink of the backward RFFT (TileWorker::run): adds the windowed
// sample pair (2 pos, 2 pos + 1) of frame f to the ring, whose slot for real
// sample j of the output is (j / 2) mod N_c.
template <typename F>
struct OlaSink {
    using C = Cx<F>;
    static constexpr bool kActive = true;
    const void* h;   // spectral filter (read by the pre-step) or null
    C* ring;         // shared memory, N_c pairs
    const C* w;      // synthesis window pairs or null
    uint32_t base;   // (f * hop / 2) mod N_c
    uint32_t mask;   // N_c - 1
    __device__ __forceinline__ void add(int pos, C x) const {
        if (w) {
            const C ww = w[pos];
            x = cx<C>(mul_rn(x.x, ww.x), mul_rn(x.y, ww.y));
        }
        C& r = ring[(base + (uint32_t)pos) & mask];
        r = cx<C>(add_rn(r.x, x.x), add_rn(r.y, x.y));
    }
};

template <typename F, int P>
struct IstftCfg {
    using C = Cx<F>;
    static constexpr int N = 1 << P;                  // complex points (frame length / 2)
    static constexpr int T = N / tile_elems(P);       // one transform per CTA
    using Tile = TileCfg<F, P, kC2RBwd, (T > 0 ? T : 1)>;
    // exchange, then the ring. The bins are read directly: staging them costs
    // a resident CTA here and measured no faster (the frame rate of the
    // transform bounds this kernel).
    static constexpr size_t RING = Tile::XBYTES;
    static constexpr size_t SMEM = RING + (size_t)N * sizeof(C);
    // whole warps, and the exchange and ring in shared memory
    static constexpr bool kOK = T >= 32 && Tile::TPC == 1 && SMEM <= 200 * 1024;
    static_assert(!kOK || Tile::THREADS == T, "one transform per CTA of T threads");
    static constexpr int MINB = Tile::MINB;
};

template <typename F, int P, int IL>
__global__ void __launch_bounds__(IstftCfg<F, P>::T, IstftCfg<F, P>::MINB)
    istft_kernel(const TileArgs a, const IstftArgs o) {
    using Cfg = IstftCfg<F, P>;
    using C = Cx<F>;
    using W = TileWorker<F, P, kC2RBwd, IL, kAoS, Cfg::T>;
    constexpr int N = Cfg::N, T = Cfg::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    W wk(a, smem_raw);
    C* ring = reinterpret_cast<C*>(smem_raw + Cfg::RING);
    C* sig = static_cast<C*>(o.sig);
    const long long hp = o.hop / 2;  // hop in sample pairs
    const long long m0 = (long long)blockIdx.x * o.run;
    const long long m1 = (m0 + o.run < o.blocks) ? m0 + o.run : o.blocks;
    const C zero = cx<C>((F)0, (F)0);
    for (int i = (int)threadIdx.x; i < N; i += T) ring[i] = zero;
    __syncthreads();
    const long long f0 = (m0 - o.k + 1 > 0) ? m0 - o.k + 1 : 0;
    const long long f1 = (m1 - 1 < o.n_frames - 1) ? m1 - 1 : o.n_frames - 1;
    OlaSink<F> sink{o.filt, ring, static_cast<const C*>(o.win), 0u, (uint32_t)(N - 1)};
    for (long long f = f0; f <= f1; ++f) {
        sink.base = (uint32_t)((f * hp) & (N - 1));
        wk.run(a, f, false, [] {}, sink);  // ends with a barrier: the frame is in the ring
        // block f is final: write it when this CTA owns it, clear its slots
        for (long long i = threadIdx.x; i < hp; i += T) {
            const uint32_t r = (uint32_t)((f * hp + i) & (N - 1));
            if (f >= m0) sig[f * hp + i] = ring[r];
            ring[r] = zero;
        }
        __syncthreads();
    }
    // blocks after the last frame are final once every frame is in
    for (long long m = (f1 + 1 > m0 ? f1 + 1 : m0); m < m1; ++m)
        for (long long i = threadIdx.x; i < hp; i += T) sig[m * hp + i] = ring[(uint32_t)((m * hp + i) & (N - 1))];
}

using IstftLaunchFn = cudaError_t (*)(const TileArgs&, const IstftArgs&, cudaStream_t, const LaunchCtx&);

// One CTA per run of blocks. A run spans ~one wave of resident CTAs over the
// output, and at least 4 (K - 1) blocks, so that the K - 1 frames each CTA
// transforms ahead of its run add at most a quarter to the work.
template <typename F, int P, int IL>
cudaError_t launch_istft(const TileArgs& a, const IstftArgs& o, cudaStream_t stream, const LaunchCtx& ctx) {
    using Cfg = IstftCfg<F, P>;
    auto kern = istft_kernel<F, P, IL>;
    static ResidentSlots slots;
    const int blocks_per_sm = resident_ctas(slots, [kern] { return occupancy_setup(kern, Cfg::T, Cfg::SMEM); });
    if (o.n_frames <= 0 || o.blocks <= 0) return cudaSuccess;
    IstftArgs oo = o;
    const long long cap = (long long)ctx.num_sms * blocks_per_sm;
    long long run = (o.blocks + cap - 1) / cap;
    if (run < 4LL * (o.k - 1)) run = 4LL * (o.k - 1);
    if (run < 1) run = 1;
    oo.run = run;
    const long long grid = (o.blocks + run - 1) / run;
    kern<<<(unsigned)grid, Cfg::T, Cfg::SMEM, stream>>>(a, oo);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

// [complex order][input layout]; null where the order has no ISTFT kernel
struct IstftTable {
    IstftLaunchFn fn[kTileMaxP + 1][2];
};

template <typename F, int... Ps>
void fill_istft_orders(IstftTable& t, std::integer_sequence<int, Ps...>) {
    (
        [&] {
            if constexpr (IstftCfg<F, Ps>::kOK) {
                t.fn[Ps][kAoS] = launch_istft<F, Ps, kAoS>;
                t.fn[Ps][kSoA] = launch_istft<F, Ps, kSoA>;
            }
        }(),
        ...);
}
void fill_istft_f32(IstftTable& t);
void fill_istft_f64(IstftTable& t);

}  // namespace zlfft
