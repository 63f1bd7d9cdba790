// TEST INFRASTRUCTURE ONLY — a C entry layer over the UNMODIFIED reference
// headers (zldsp::fft::CFFT<F> / RFFT<F>, src/zldsp_fft_cfft.hpp:11-118 and
// src/zldsp_fft_rfft.hpp:11-139), compiled against the project's Highway-API
// shim (oracle/hwy_shim). The build recipe (oracle/Makefile) points -I at the
// reference's own src/ directory; no reference source is copied.
//
// Used by the tests to check parity and by bench.py as the timed CPU
// baseline. Never linked into the product library.
//
// Batch conventions (all pointers host memory):
//   AoS complex:  transform b starts at base + b * 2 * n_complex scalars
//   SoA complex:  transform b's real part at re + b * n_complex, imag at im + b * n_complex
//   real:         transform b starts at base + b * n_real
// A plan holds one reference object per worker thread; a call splits the
// batch evenly over those threads (the reference itself is single-threaded).
#include <algorithm>
#include <array>
#include <complex>
#include <cstddef>
#include <memory>
#include <thread>
#include <utility>
#include <vector>

#include "zldsp_fft_cfft.hpp"
#include "zldsp_fft_rfft.hpp"

namespace {

enum Layout { kAoS = 0, kSoA = 1 };

template <typename F>
struct RefPlan {
    int kind = 0;  // 0 complex, 1 real
    size_t order = 0;
    std::vector<std::unique_ptr<zldsp::fft::CFFT<F>>> cfft;
    std::vector<std::unique_ptr<zldsp::fft::RFFT<F>>> rfft;
};

template <typename Fn>
void run_split(size_t batch, size_t nthreads, Fn&& fn) {
    nthreads = std::max<size_t>(1, std::min(nthreads, batch));
    if (nthreads == 1) {
        fn(0, 0, batch);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(nthreads);
    const size_t per = batch / nthreads, rem = batch % nthreads;
    size_t start = 0;
    for (size_t t = 0; t < nthreads; ++t) {
        const size_t count = per + (t < rem ? 1 : 0);
        pool.emplace_back([&fn, t, start, count]() { fn(t, start, start + count); });
        start += count;
    }
    for (auto& th : pool) th.join();
}

template <typename F>
void* plan_create(int kind, size_t order, size_t nthreads) {
    auto* p = new RefPlan<F>();
    p->kind = kind;
    p->order = order;
    nthreads = std::max<size_t>(1, nthreads);
    for (size_t t = 0; t < nthreads; ++t) {
        if (kind == 0) {
            p->cfft.emplace_back(std::make_unique<zldsp::fft::CFFT<F>>(order));
        } else {
            p->rfft.emplace_back(std::make_unique<zldsp::fft::RFFT<F>>(order));
        }
    }
    return p;
}

template <typename F>
void cfft_exec(void* plan_v, int forward, int in_layout, const void* in_re, const void* in_im, int out_layout,
               void* out_re, void* out_im, size_t batch) {
    auto* plan = static_cast<RefPlan<F>*>(plan_v);
    using C = std::complex<F>;
    const size_t n = size_t{1} << plan->order;
    run_split(batch, plan->cfft.size(), [&](size_t t, size_t b0, size_t b1) {
        auto& fft = *plan->cfft[t];
        for (size_t b = b0; b < b1; ++b) {
            C* ia = const_cast<C*>(static_cast<const C*>(in_re)) + b * n;
            std::array<F*, 2> is{const_cast<F*>(static_cast<const F*>(in_re)) + b * n,
                                 const_cast<F*>(static_cast<const F*>(in_im)) + b * n};
            C* oa = static_cast<C*>(out_re) + b * n;
            std::array<F*, 2> os{static_cast<F*>(out_re) + b * n, static_cast<F*>(out_im) + b * n};
            if (forward) {
                if (in_layout == kAoS && out_layout == kAoS) fft.forward(ia, oa);
                else if (in_layout == kAoS) fft.forward(ia, os);
                else if (out_layout == kAoS) fft.forward(is, oa);
                else fft.forward(is, os);
            } else {
                if (in_layout == kAoS && out_layout == kAoS) fft.backward(ia, oa);
                else if (in_layout == kAoS) fft.backward(ia, os);
                else if (out_layout == kAoS) fft.backward(is, oa);
                else fft.backward(is, os);
            }
        }
    });
}

// mode: 0 forward (to AoS/SoA), 1 forward_sqr_mag, 2 backward (from AoS/SoA)
template <typename F>
void rfft_exec(void* plan_v, int mode, int layout, const void* a_re, const void* a_im, void* b_re, void* b_im,
               size_t batch) {
    auto* plan = static_cast<RefPlan<F>*>(plan_v);
    using C = std::complex<F>;
    const size_t n = size_t{1} << plan->order;
    const size_t nb = n / 2 + 1;
    run_split(batch, plan->rfft.size(), [&](size_t t, size_t b0, size_t b1) {
        auto& fft = *plan->rfft[t];
        for (size_t b = b0; b < b1; ++b) {
            if (mode == 0) {
                F* real_in = const_cast<F*>(static_cast<const F*>(a_re)) + b * n;
                if (layout == kAoS) {
                    fft.forward(real_in, static_cast<C*>(b_re) + b * nb);
                } else {
                    fft.forward(real_in, std::array<F*, 2>{static_cast<F*>(b_re) + b * nb,
                                                           static_cast<F*>(b_im) + b * nb});
                }
            } else if (mode == 1) {
                F* real_in = const_cast<F*>(static_cast<const F*>(a_re)) + b * n;
                fft.forward_sqr_mag(real_in, static_cast<F*>(b_re) + b * nb);
            } else {
                F* real_out = static_cast<F*>(b_re) + b * n;
                if (layout == kAoS) {
                    fft.backward(const_cast<C*>(static_cast<const C*>(a_re)) + b * nb, real_out);
                } else {
                    fft.backward(std::array<F*, 2>{const_cast<F*>(static_cast<const F*>(a_re)) + b * nb,
                                                   const_cast<F*>(static_cast<const F*>(a_im)) + b * nb},
                                 real_out);
                }
            }
        }
    });
}

// Latency loop: forward(in -> mid) then backward(mid -> out) of one AoS
// transform, `reps` times, on the calling thread (the reference's own
// single-transform use, without a foreign-call round trip per transform).
template <typename F>
void cfft_roundtrip_repeat(void* plan_v, const void* in, void* mid, void* out, size_t reps) {
    auto* plan = static_cast<RefPlan<F>*>(plan_v);
    using C = std::complex<F>;
    auto& fft = *plan->cfft[0];
    for (size_t r = 0; r < reps; ++r) {
        fft.forward(const_cast<C*>(static_cast<const C*>(in)), static_cast<C*>(mid));
        fft.backward(static_cast<C*>(mid), static_cast<C*>(out));
    }
}

}  // namespace

extern "C" {

// prec: 0 float, 1 double. kind: 0 CFFT, 1 RFFT.
void* zlref_plan_create(int prec, int kind, size_t order, size_t nthreads) {
    return prec == 0 ? plan_create<float>(kind, order, nthreads) : plan_create<double>(kind, order, nthreads);
}

void zlref_plan_destroy(int prec, void* plan) {
    if (prec == 0) delete static_cast<RefPlan<float>*>(plan);
    else delete static_cast<RefPlan<double>*>(plan);
}

void zlref_cfft_exec(int prec, void* plan, int forward, int in_layout, const void* in_re, const void* in_im,
                     int out_layout, void* out_re, void* out_im, size_t batch) {
    if (prec == 0) cfft_exec<float>(plan, forward, in_layout, in_re, in_im, out_layout, out_re, out_im, batch);
    else cfft_exec<double>(plan, forward, in_layout, in_re, in_im, out_layout, out_re, out_im, batch);
}

void zlref_rfft_exec(int prec, void* plan, int mode, int layout, const void* a_re, const void* a_im, void* b_re,
                     void* b_im, size_t batch) {
    if (prec == 0) rfft_exec<float>(plan, mode, layout, a_re, a_im, b_re, b_im, batch);
    else rfft_exec<double>(plan, mode, layout, a_re, a_im, b_re, b_im, batch);
}

void zlref_cfft_roundtrip_repeat(int prec, void* plan, const void* in, void* mid, void* out, size_t reps) {
    if (prec == 0) cfft_roundtrip_repeat<float>(plan, in, mid, out, reps);
    else cfft_roundtrip_repeat<double>(plan, in, mid, out, reps);
}

// The reference's algorithm switch on this host (src/common/zldsp_fft_common_system.hpp:132-157).
void zlref_switch_order(int prec, size_t* max_l1_order, size_t* switch_order) {
    auto r = prec == 0 ? zldsp::fft::common::get_switch_order<float>()
                       : zldsp::fft::common::get_switch_order<double>();
    *max_l1_order = r.first;
    *switch_order = r.second;
}

}  // extern "C"
