// Latency of the C++ drop-in classes called the way the reference's users
// call zldsp::fft::CFFT<float>: one transform per call on host buffers,
// forward then backward, synchronous. bench.py compiles and runs it for the
// single-transform workload; it prints one JSON line.
//
//   dropin_latency [order=10] [pairs=2000] [rounds=7]
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "zldsp_fft_cuda/zldsp_fft_cfft.hpp"

int main(int argc, char** argv) {
    const size_t order = argc > 1 ? std::strtoul(argv[1], nullptr, 10) : 10;
    const int pairs = argc > 2 ? std::atoi(argv[2]) : 2000;
    const int rounds = argc > 3 ? std::atoi(argv[3]) : 7;
    const size_t n = size_t{1} << order;
    zldsp::fft::CFFT<float> cfft(order);
    std::vector<std::complex<float>> x(n), y(n), z(n);
    for (size_t i = 0; i < n; ++i) x[i] = {std::sin(0.37f * i), std::cos(0.11f * i)};
    for (int i = 0; i < 200; ++i) {  // warm-up: plan buffers, driver paths
        cfft.forward(x.data(), y.data());
        cfft.backward(y.data(), z.data());
    }
    std::vector<double> us;
    for (int r = 0; r < rounds; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < pairs; ++i) {
            cfft.forward(x.data(), y.data());
            cfft.backward(y.data(), z.data());
        }
        const auto t1 = std::chrono::steady_clock::now();
        us.push_back(std::chrono::duration<double, std::micro>(t1 - t0).count() / pairs);
    }
    std::sort(us.begin(), us.end());
    float err = 0.f;
    for (size_t i = 0; i < n; ++i) err = std::fmax(err, std::abs(z[i] / float(n) - x[i]));
    std::printf("{\"order\": %zu, \"pairs_per_round\": %d, \"rounds\": %d, \"us_per_pair_median\": %.3f, "
                "\"us_per_pair_min\": %.3f, \"roundtrip_max_abs_err\": %.3g}\n",
                order, pairs, rounds, us[us.size() / 2], us.front(), err);
    return err < 1e-3f ? 0 : 1;
}
