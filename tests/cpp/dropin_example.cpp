// The README usage of the reference, compiled unchanged except for the include
// path, against the GPU drop-in headers. Prints the first bins so the test can
// compare them with the oracle.
#include <cmath>
#include <complex>
#include <cstdio>
#include <vector>

#include "zldsp_fft_cuda/zldsp_fft_cfft.hpp"
#include "zldsp_fft_cuda/zldsp_fft_rfft.hpp"

int main() {
    constexpr size_t order = 10;
    zldsp::fft::CFFT<float> cfft(order);
    std::vector<std::complex<float>> in_buffer(1 << order), out_buffer(1 << order), back(1 << order);
    for (size_t i = 0; i < in_buffer.size(); ++i) in_buffer[i] = {std::sin(0.1f * i), std::cos(0.3f * i)};
    cfft.forward(in_buffer.data(), out_buffer.data());
    cfft.backward(out_buffer.data(), back.data());
    std::vector<float> re(1 << order), im(1 << order);
    cfft.forward(in_buffer.data(), {re.data(), im.data()});
    float err = 0.f;
    for (size_t i = 0; i < in_buffer.size(); ++i) {
        err = std::fmax(err, std::abs(back[i] / float(1 << order) - in_buffer[i]));
        err = std::fmax(err, std::abs(std::complex<float>(re[i], im[i]) - out_buffer[i]));
    }
    zldsp::fft::RFFT<float> rfft(order);
    std::vector<float> real_in(1 << order), real_back(1 << order), sqr((1 << order) / 2 + 1);
    std::vector<std::complex<float>> bins((1 << order) / 2 + 1);
    for (size_t i = 0; i < real_in.size(); ++i) real_in[i] = std::sin(0.05f * i * i);
    rfft.forward(real_in.data(), bins.data());
    rfft.forward_sqr_mag(real_in.data(), sqr.data());
    rfft.backward(bins.data(), real_back.data());
    for (size_t i = 0; i < real_in.size(); ++i) err = std::fmax(err, std::abs(real_back[i] / float(1 << (order - 1)) - real_in[i]));
    std::printf("size=%zu order=%zu maxerr=%g X0=%.9g,%.9g X1=%.9g,%.9g\n", cfft.get_size(), cfft.get_order(), err,
                out_buffer[0].real(), out_buffer[0].imag(), out_buffer[1].real(), out_buffer[1].imag());
    bool threw = false;
    try {
        zldsp::fft::RFFT<float> bad(0);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    std::printf("rfft0_throws=%d\n", threw ? 1 : 0);
    return err < 1e-3f && threw ? 0 : 1;
}
