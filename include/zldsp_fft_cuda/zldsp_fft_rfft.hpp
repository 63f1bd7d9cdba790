// Drop-in replacement for zldsp::fft::RFFT<F> (reference: src/zldsp_fft_rfft.hpp:11-139)
// running on the GPU through libzlfft_cuda: constructor, getters, forward to
// AoS/SoA bins, backward from AoS/SoA bins, and forward_sqr_mag, on host
// buffers, synchronous. Link with -lzlfft_cuda.
#pragma once

#include <array>
#include <complex>

#include "zldsp_fft_common.hpp"

namespace zldsp::fft {

template <typename F>
class RFFT {
    using C = std::complex<F>;

public:
    // reference: src/zldsp_fft_rfft.hpp:24-53 (order >= 1; the reference's
    // RFFT(0) underflows, this one throws)
    explicit RFFT(const size_t rfft_order) : plan_(ZLFFT_R2C, cuda_detail::precision<F>(), rfft_order) {}

    // reference: src/zldsp_fft_rfft.hpp:55-61
    [[nodiscard]] size_t get_size() const { return plan_.size(); }
    [[nodiscard]] size_t get_order() const { return plan_.order(); }

    // real -> AoS bins (reference :68)
    void forward(F* in_buffer, C* out_buffer) { run(ZLFFT_FORWARD, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_AOS, out_buffer, nullptr); }
    // real -> SoA bins (reference :77)
    void forward(F* in_buffer, std::array<F*, 2> out_buffer) {
        run(ZLFFT_FORWARD, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_SOA, out_buffer[0], out_buffer[1]);
    }
    // AoS bins -> real (reference :86)
    void backward(C* in_buffer, F* out_buffer) { run(ZLFFT_BACKWARD, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_AOS, out_buffer, nullptr); }
    // SoA bins -> real (reference :95)
    void backward(std::array<F*, 2> in_buffer, F* out_buffer) {
        run(ZLFFT_BACKWARD, ZLFFT_SOA, in_buffer[0], in_buffer[1], ZLFFT_AOS, out_buffer, nullptr);
    }
    // real -> N/2+1 squared magnitudes (reference :104)
    void forward_sqr_mag(F* in_buffer, F* out_buffer) {
        run(ZLFFT_FORWARD_SQR_MAG, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_AOS, out_buffer, nullptr);
    }

    [[nodiscard]] zlfft_plan plan() const { return plan_.get(); }

private:
    void run(int op, int il, const void* i0, const void* i1, int ol, void* o0, void* o1) {
        cuda_detail::check(zlfft_exec_host(plan_.get(), op, il, ol, i0, i1, o0, o1));
    }
    cuda_detail::Plan plan_;
};

}  // namespace zldsp::fft
