// Drop-in replacement for zldsp::fft::CFFT<F> (reference: src/zldsp_fft_cfft.hpp:11-118)
// running on the GPU through libzlfft_cuda. Same class name, namespace,
// constructor, getters and the eight forward/backward overloads; buffers are
// host memory and every call is synchronous (the output is valid on return),
// exactly like the reference. Link with -lzlfft_cuda.
#pragma once

#include <array>
#include <complex>

#include "zldsp_fft_common.hpp"

namespace zldsp::fft {

template <typename F>
class CFFT {
    using C = std::complex<F>;

public:
    // reference: src/zldsp_fft_cfft.hpp:19-23
    explicit CFFT(const size_t cfft_order) : plan_(ZLFFT_C2C, cuda_detail::precision<F>(), cfft_order) {}

    // reference: src/zldsp_fft_cfft.hpp:25-31
    [[nodiscard]] size_t get_size() const { return plan_.size(); }
    [[nodiscard]] size_t get_order() const { return plan_.order(); }

    // AoS -> AoS (reference :38, :47)
    void forward(C* in_buffer, C* out_buffer) { run(ZLFFT_FORWARD, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_AOS, out_buffer, nullptr); }
    void backward(C* in_buffer, C* out_buffer) { run(ZLFFT_BACKWARD, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_AOS, out_buffer, nullptr); }
    // AoS -> SoA (reference :56, :65)
    void forward(C* in_buffer, std::array<F*, 2> out_buffer) {
        run(ZLFFT_FORWARD, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_SOA, out_buffer[0], out_buffer[1]);
    }
    void backward(C* in_buffer, std::array<F*, 2> out_buffer) {
        run(ZLFFT_BACKWARD, ZLFFT_AOS, in_buffer, nullptr, ZLFFT_SOA, out_buffer[0], out_buffer[1]);
    }
    // SoA -> AoS (reference :74, :83)
    void forward(std::array<F*, 2> in_buffer, C* out_buffer) {
        run(ZLFFT_FORWARD, ZLFFT_SOA, in_buffer[0], in_buffer[1], ZLFFT_AOS, out_buffer, nullptr);
    }
    void backward(std::array<F*, 2> in_buffer, C* out_buffer) {
        run(ZLFFT_BACKWARD, ZLFFT_SOA, in_buffer[0], in_buffer[1], ZLFFT_AOS, out_buffer, nullptr);
    }
    // SoA -> SoA (reference :92, :101)
    void forward(std::array<F*, 2> in_buffer, std::array<F*, 2> out_buffer) {
        run(ZLFFT_FORWARD, ZLFFT_SOA, in_buffer[0], in_buffer[1], ZLFFT_SOA, out_buffer[0], out_buffer[1]);
    }
    void backward(std::array<F*, 2> in_buffer, std::array<F*, 2> out_buffer) {
        run(ZLFFT_BACKWARD, ZLFFT_SOA, in_buffer[0], in_buffer[1], ZLFFT_SOA, out_buffer[0], out_buffer[1]);
    }

    // The underlying plan, for the batched device-pointer entry point (zlfft_exec_device).
    [[nodiscard]] zlfft_plan plan() const { return plan_.get(); }

private:
    void run(int op, int il, const void* i0, const void* i1, int ol, void* o0, void* o1) {
        cuda_detail::check(zlfft_exec_host(plan_.get(), op, il, ol, i0, i1, o0, o1));
    }
    cuda_detail::Plan plan_;
};

}  // namespace zldsp::fft
